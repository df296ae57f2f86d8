// ref_harness: drives the UNMODIFIED reference (CAVIAR, compiled from its own
// sources into libcaviar_ref.a by oracle/Makefile) and dumps its FP64 results.
// Test infrastructure only: used by tests/ to pin the C restatement and the
// CUDA path, and by bench.py as the timed reference CPU arm.
//
// Usage:
//   ref_harness <script.casl> <state.bin> forces <out.bin>
//   ref_harness <script.casl> <state.bin> run    <out.bin> <nsteps> [budget_seconds]
//   ref_harness <script.casl> <state.bin> randvel <out.bin> <seed> <amplitude>
//   ref_harness <script.casl> <state.bin> runcall <out.bin>
//
// The CASL script defines the objects (domain box, atom_data basic,
// neighborlist basic, force fields, md_simulator basic) with the reference's
// own keywords but adds no atoms and does not call `run`; the atoms are added
// here from state.bin through Atom_data::add_atom (atom_data.cpp:487-521) so
// that FP64 positions pass bit-exactly (no text round trip).
//
// "forces" repeats Md_simulator::setup (md_simulator.cpp:504-549): owned wrap,
// ghost generation, Neighborlist::init + build(true), zero acceleration, each
// force field's calculate_acceleration.  It dumps accelerations, virialForce,
// the canonical pair set of the Verlet list, the Ewald k-space energy pieces
// and the kinetic energy.
//
// "run" calls Md_simulator::step(i) for i in [0, nsteps) (md_simulator.cpp:
// 376-485) and dumps the final owned state plus per-step kinetic energy and
// virial, and the wall time of the first step (which includes setup) and of
// the remaining steps.  With a budget, it stops after the first step whose end
// exceeds the budget (at least two steps) and reports how many ran.
//
// "randvel" calls Atom_data::add_random_velocity(seed, amplitude) on the loaded
// atoms (uniform velocities from the reference's mt19937, centre-of-mass
// motion removed) and dumps the owned state.
//
// state.bin (little endian):
//   int64 n; then n records of { int32 type; int32 mol; double pos[3]; double vel[3]; }
//
// out.bin: a sequence of named blocks { char name[16]; int64 count; int32 elem_size; pad; data }.

#include "caviar/CAVIAR.h"
#include "caviar/interpreter/all.h"
#include "caviar/objects/atom_data.h"
#include "caviar/objects/domain.h"
#include "caviar/objects/neighborlist.h"
#include "caviar/objects/force_field.h"
#include "caviar/objects/force_field/electrostatic_ewald_k.h"
#include "caviar/objects/md_simulator.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <tuple>
#include <vector>

namespace
{

  struct Out
  {
    FILE *f;
    explicit Out(const char *path) : f(std::fopen(path, "wb"))
    {
      if (!f)
      {
        std::fprintf(stderr, "cannot open %s\n", path);
        std::exit(2);
      }
    }
    ~Out() { std::fclose(f); }
    void block(const char *name, const void *data, int64_t count, int32_t elem)
    {
      char nm[16] = {0};
      std::strncpy(nm, name, 15);
      int32_t pad = 0;
      std::fwrite(nm, 1, 16, f);
      std::fwrite(&count, 8, 1, f);
      std::fwrite(&elem, 4, 1, f);
      std::fwrite(&pad, 4, 1, f);
      if (count > 0)
        std::fwrite(data, (size_t)elem, (size_t)count, f);
    }
    void scalar(const char *name, double v) { block(name, &v, 1, 8); }
  };

  struct Rec
  {
    int32_t type;
    int32_t mol;
    double pos[3];
    double vel[3];
  };

  std::vector<Rec> read_state(const char *path)
  {
    FILE *f = std::fopen(path, "rb");
    if (!f)
    {
      std::fprintf(stderr, "cannot open %s\n", path);
      std::exit(2);
    }
    int64_t n = 0;
    if (std::fread(&n, 8, 1, f) != 1)
      std::exit(2);
    std::vector<Rec> r((size_t)n);
    for (auto &x : r)
    {
      if (std::fread(&x.type, 4, 1, f) != 1 || std::fread(&x.mol, 4, 1, f) != 1 ||
          std::fread(x.pos, 8, 3, f) != 3 || std::fread(x.vel, 8, 3, f) != 3)
        std::exit(2);
    }
    std::fclose(f);
    return r;
  }

  // Canonical pair set of a reference Verlet list: each entry (owned i, j)
  // becomes (id_a, id_b, s) with id_a < id_b and r_b + s*L the image of b
  // that is paired with a (s in {-1,0,1}^3).  Owned-owned entries have s = 0;
  // a ghost's s comes from its offset to its owner.  Duplicates (owned-ghost
  // pairs appear from both ends) are removed and the set is sorted.
  std::vector<std::array<int32_t, 5>> canonical_pairs(caviar::Atom_data *ad, caviar::Neighborlist *nl,
                                                      caviar::Domain *dom)
  {
    const auto &own = ad->atom_struct_owned;
    const auto &gh = ad->atom_struct_ghost;
    const size_t n = own.position.size();
    const double L[3] = {dom->size_global.x, dom->size_global.y, dom->size_global.z};
    std::vector<int64_t> id_to_index;
    for (size_t i = 0; i < n; ++i)
    {
      if ((size_t)own.id[i] >= id_to_index.size())
        id_to_index.resize(own.id[i] + 1, -1);
      id_to_index[own.id[i]] = (int64_t)i;
    }
    std::vector<std::array<int32_t, 5>> out;
    for (size_t i = 0; i < nl->neighlist.size(); ++i)
    {
      for (auto j : nl->neighlist[i])
      {
        int32_t ida = (int32_t)own.id[i];
        int32_t idb;
        int s[3] = {0, 0, 0};
        if (j < n)
        {
          idb = (int32_t)own.id[j];
        }
        else
        {
          const size_t g = j - n;
          idb = (int32_t)gh.id[g];
          const auto &po = own.position[(size_t)id_to_index[idb]];
          const double gp[3] = {gh.position[g].x, gh.position[g].y, gh.position[g].z};
          const double op[3] = {po.x, po.y, po.z};
          for (int d = 0; d < 3; ++d)
            s[d] = (int)std::lround((gp[d] - op[d]) / L[d]);
        }
        if (ida > idb || (ida == idb && std::make_tuple(s[0], s[1], s[2]) < std::make_tuple(-s[0], -s[1], -s[2])))
        {
          std::swap(ida, idb);
          s[0] = -s[0];
          s[1] = -s[1];
          s[2] = -s[2];
        }
        out.push_back({ida, idb, s[0], s[1], s[2]});
      }
    }
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
    return out;
  }

  double now_s()
  {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
  }

} // namespace

int main(int argc, char **argv)
{
  if (argc < 5)
  {
    std::fprintf(stderr, "usage: %s script.casl state.bin forces|run out.bin [nsteps]\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[3];
  const int64_t nsteps = (argc > 5) ? std::atoll(argv[5]) : 0;
  const double budget = (argc > 6) ? std::atof(argv[6]) : 0.0;

  char arg0[] = "ref_harness";
  char arg1[] = "-i";
  std::vector<char> script(argv[1], argv[1] + std::strlen(argv[1]) + 1);
  char *cargv[] = {arg0, arg1, script.data(), nullptr};

  caviar::CAVIAR cav(3, cargv);
  cav.execute();

  auto *oc = cav.object_container;
  if (oc->atom_data.empty() || oc->domain.empty() || oc->md_simulator.empty())
  {
    std::fprintf(stderr, "script must define domain, atom_data and md_simulator\n");
    return 2;
  }
  caviar::Atom_data *ad = oc->atom_data[0];
  caviar::Domain *dom = oc->domain[0];
  caviar::Md_simulator *sim = oc->md_simulator[0];
  caviar::Neighborlist *nl = oc->neighborlist.empty() ? nullptr : oc->neighborlist[0];

  const auto state = read_state(argv[2]);
  for (size_t i = 0; i < state.size(); ++i)
  {
    const auto &r = state[i];
    ad->add_atom((caviar::GlobalID_t)i, (caviar::AtomType_t)r.type,
                 caviar::Vector<double>{r.pos[0], r.pos[1], r.pos[2]},
                 caviar::Vector<double>{r.vel[0], r.vel[1], r.vel[2]});
    ad->atom_struct_owned.molecule_index.back() = r.mol;
  }

  Out out(argv[4]);
  const int64_t n = (int64_t)state.size();

  auto dump_owned = [&](void) {
    const auto &own = ad->atom_struct_owned;
    std::vector<double> buf((size_t)n * 3);
    std::vector<int32_t> ids((size_t)n);
    for (int64_t i = 0; i < n; ++i)
      ids[(size_t)i] = (int32_t)own.id[(size_t)i];
    out.block("id", ids.data(), n, 4);
    auto put = [&](const char *name, const std::vector<caviar::Vector<double>> &v) {
      for (int64_t i = 0; i < n; ++i)
      {
        buf[(size_t)(3 * i)] = v[(size_t)i].x;
        buf[(size_t)(3 * i + 1)] = v[(size_t)i].y;
        buf[(size_t)(3 * i + 2)] = v[(size_t)i].z;
      }
      out.block(name, buf.data(), 3 * n, 8);
    };
    put("pos", own.position);
    put("vel", own.velocity);
    put("acc", own.acceleration);
  };

  if (mode == "forces")
  {
    // Md_simulator::initialize does this before setup (md_simulator.cpp:307);
    // kinetic_energy skips atoms whose mpi_rank is unset (kinetic_energy.cpp:64).
    ad->set_atoms_mpi_rank();
    const double t0 = now_s();
    if (nl)
      nl->init();
    ad->exchange_owned(0);
    ad->exchange_ghost(0);
    if (nl)
      nl->build(true);
    ad->reset_virial();
    ad->reset_owned_acceleration();
    for (auto *f : sim->force_field)
      f->calculate_acceleration();
    const double t1 = now_s();
    dump_owned();
    out.scalar("virial", ad->virialForce);
    out.scalar("ke", ad->kinetic_energy());
    out.scalar("n_ghost", (double)ad->atom_struct_ghost.position.size());
    out.scalar("wall", t1 - t0);
    for (auto *f : sim->force_field)
    {
      auto *ek = dynamic_cast<caviar::force_field::Electrostatic_ewald_k *>(f);
      if (ek)
      {
        out.scalar("ek_kspace", ek->k_space_energy());
        out.scalar("ek_self", ek->self_energy());
        out.scalar("ek_nk", (double)ek->n_k_vectors);
        std::vector<double> sk;
        for (auto &c : ek->potential_k_coef_cmplx)
        {
          sk.push_back(c.real());
          sk.push_back(c.imag());
        }
        out.block("sk", sk.data(), (int64_t)sk.size(), 8);
      }
    }
    if (nl)
    {
      const auto pairs = canonical_pairs(ad, nl, dom);
      out.block("pairs", pairs.data(), (int64_t)pairs.size() * 5, 4);
    }
  }
  else if (mode == "run")
  {
    std::vector<double> ke, vir;
    double t_first = 0, t_rest = 0;
    int64_t done = 0;
    for (int64_t s = 0; s < nsteps; ++s)
    {
      const double t0 = now_s();
      sim->step(s);
      const double t1 = now_s();
      if (s == 0)
        t_first = t1 - t0;
      else
        t_rest += t1 - t0;
      ke.push_back(ad->kinetic_energy());
      vir.push_back(ad->virialForce);
      ++done;
      if (budget > 0 && s >= 1 && t_first + t_rest > budget)
        break;
    }
    dump_owned();
    out.block("ke_trace", ke.data(), (int64_t)ke.size(), 8);
    out.block("vir_trace", vir.data(), (int64_t)vir.size(), 8);
    out.scalar("wall_first", t_first);
    out.scalar("wall_rest", t_rest);
    out.scalar("steps_done", (double)done);
    out.scalar("n_ghost", (double)ad->atom_struct_ghost.position.size());
  }
  else if (mode == "runcall")
  {
    // the simulator's own run() (md_simulator.cpp:235-274, or the B200
    // adapter's override when the script names `md_simulator b200`), over the
    // script's initial_step .. final_step, then the owned state
    const double t0 = now_s();
    sim->run();
    out.scalar("wall", now_s() - t0);
    dump_owned();
  }
  else if (mode == "randvel")
  {
    // the reference's own Atom_data::add_random_velocity (atom_data.cpp:597-616)
    // on the loaded atoms: argv[5] = seed, argv[6] = amplitude
    const unsigned int seed = (argc > 5) ? (unsigned int)std::strtoul(argv[5], nullptr, 10) : 0u;
    const double amplitude = (argc > 6) ? std::atof(argv[6]) : 1.0;
    ad->add_random_velocity(seed, amplitude);
    dump_owned();
  }
  else
  {
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
  }
  return 0;
}
