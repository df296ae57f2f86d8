// cvr_casl.cpp -- the hot-path subset of CAVIAR's CASL scripting language and
// object model, in front of the C ABI (include/caviar_b200.h).
//
// A script written for the reference's objects runs here unchanged as long as
// it only uses the hot-path objects and keywords:
//   domain box <name>          xmin xmax ymin ymax zmin zmax (or lower_global.x ...),
//                              boundary_condition|bc i j k, generate
//                              (reference: src/caviar/objects/domain.cpp:206-266)
//   atom_data basic <name>     ghost_cutoff, k_b, set_domain|domain, add_type_mass t m,
//                              add_type_charge t q, add_xyz_data_file file_name "<f>"
//                              [read_velocity] [last_frame] [replace_data],
//                              set_owned_position|set_owned_velocity i x y z,
//                              add_random_velocity seed amplitude, msd_process (accepted, no effect)
//                              (atom_data.cpp:78-306, 597-616, atom_data/add_xyz_data_file.cpp:22-168)
//   neighborlist basic <name>  set_atom_data|atom_data, set_domain|domain, cutoff,
//                              cutoff_extra_coef, build_cell_list,
//                              make_verlet_list_from_cell_list, rebuild_test, all_atom_test, dt
//                              (neighborlist.cpp:193-251)
//   force_field lj <name>      cutoff, cutoff_list i j v, epsilon i j v, sigma i j v,
//                              epsilon_atom i v, sigma_atom i v, lambda_s i j v,
//                              lambda_e i j v, wca, ignore_intra_molecule, jump_tol v,
//                              monitor_jump (accepted; the reference's per-pair print is not made),
//                              make_off_diagonal_vectors, set_neighborlist|neighborlist,
//                              set_atom_data|atom_data, set_domain|domain (lj.cpp:42-353)
//   force_field electrostatic_ewald_r <name>  cutoff, alpha, k_electrostatic, lambda i j v,
//                              set_neighborlist, set_atom_data (electrostatic_ewald_r.cpp:38-107)
//   force_field electrostatic_ewald_k <name>  alpha, k_max, kx_max, ky_max, kz_max,
//                              k_electrostatic, slab_normal_axis, slab_lz|slab_thickness,
//                              epsilon_dipole, set_atom_data, set_domain (electrostatic_ewald_k.cpp:48-143)
//   force_field electrostatic_ewald_slab_correction <name>  slab_normal_axis, lz, k_max,
//                              kx_max, ky_max, k_electrostatic, set_atom_data, set_domain
//                              (electrostatic_ewald_slab_correction.cpp:44-111)
//   md_simulator basic <name>  set_atom_data, add_force_field|force_field,
//                              add_neighborlist|neighborlist, add_writer|writer,
//                              integrator_type velocity_verlet|velocity_verlet_langevin,
//                              temperature, friction, kb, kbt, dt, initial_step,
//                              final_step, final_step_add, initial_time, final_time,
//                              remove_force_field|neighborlist|writer|constraint,
//                              run (md_simulator.cpp:58-233)
//   writer atom_data <name>    set_atom_data|atom_data, set_domain|domain, energy_step,
//                              temperature_step, pressure_step, volume_step, xyz_step,
//                              file_name_energy|_temperature|_pressure|_volume|_xyz,
//                              xyz_output_id, xyz_output_velocity, xyz_output_acceleration,
//                              open_files, close_files, *_mpi_rank0, *_mpi_per_process
//                              (writer/atom_data.cpp:84-331, dump_energy.cpp, dump_xyz_serial.cpp)
//   constraint berendsen <name>    set_atom_data, temperature, coupling, dt, step,
//                                  lambda_min, lambda_max (constraint/berendsen.cpp:36-96)
//   constraint nose_hoover <name>  set_atom_data, temperature, mass, tau, type, kb, dt
//                                  (constraint/nose_hoover.cpp:39-117); md_simulator add_constraint
// plus the variables `real name value` / `int name value`, comments (#) and
// `exit`.  Keywords of these objects that sit off the hot path (other
// constraints, msd/povray/ghost writers) are
// rejected with a message instead of being ignored.
//
// Writers follow the reference: a line "step time value" (default stream
// format, 6 significant digits) at setup as (0, 0) and after every step i
// with i % <x>_step == 0 as (i, time at the start of the step); energy =
// kinetic energy, temperature and pressure only when atom_data has
// temperature_process / pressure_process (0 otherwise; the pressure is not
// finalised at setup, so its setup line is 0), xyz frames "N / Atom /
// type [id] x y z [v] [a]" with positions wrapped into the box.  File names
// get ".txt" / ".xyz" and are relative to the script's directory.
//
// Extensions for the B200 path (md_simulator): rng reference|philox and seed N
// (the Langevin noise: the reference's own streams, or a counter-based
// generator on the GPU), precision mixed|fp64,
// rebuild_policy displacement|reference, thermo_step N, thermo_file "<f>",
// state_file "<f>" (FP64 binary dump of the final state, id order);
// (atom_data) add_state_file file_name "<f>" [replace_data] (reads that dump
// back: positions and velocities bit for bit), write_state_file "<f>" (the
// same dump of the atoms as loaded so far, acceleration zero); (writer) potential_energy_step
// N and file_name_potential_energy "<f>" (LJ + Ewald potential energy, which
// the reference writer lacks), precision N (significant digits of every
// writer number; 17 makes an xyz frame an exact FP64 restart file).
//
// Errors come back as CVR_ERR_INVALID with "file:line: message"; nothing here
// exits the process (the reference prints and exits, interpreter/error.cpp:27-31).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <random>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/caviar_b200.h"

namespace {

struct CaslError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// ------------------------------------------------------------------ lexer
struct Line {
  std::vector<std::string> tok;
  std::vector<bool> quoted;
  int lineno = 0;
  size_t pos = 0;
  bool done() const { return pos >= tok.size(); }
};

std::vector<Line> lex(const std::string &path) {
  std::ifstream f(path);
  if (!f) throw CaslError("cannot open script " + path);
  std::vector<Line> out;
  std::string raw;
  int no = 0;
  while (std::getline(f, raw)) {
    ++no;
    Line L;
    L.lineno = no;
    size_t k = 0;
    while (k < raw.size()) {
      const char c = raw[k];
      if (c == '#') break;
      if (std::isspace((unsigned char)c)) {
        ++k;
        continue;
      }
      if (c == '"' || c == '\'') {
        const size_t e = raw.find(c, k + 1);
        if (e == std::string::npos) throw CaslError(path + ":" + std::to_string(no) + ": unterminated string");
        L.tok.push_back(raw.substr(k + 1, e - k - 1));
        L.quoted.push_back(true);
        k = e + 1;
        continue;
      }
      size_t e = k;
      while (e < raw.size() && !std::isspace((unsigned char)raw[e]) && raw[e] != '#') ++e;
      L.tok.push_back(raw.substr(k, e - k));
      L.quoted.push_back(false);
      k = e;
    }
    if (!L.tok.empty()) out.push_back(L);
  }
  return out;
}

std::string dir_of(const std::string &p) {
  const size_t s = p.find_last_of('/');
  return (s == std::string::npos) ? std::string(".") : p.substr(0, s);
}

// ------------------------------------------------------------- objects
struct Script;

struct Object {
  std::string name;
  virtual ~Object() = default;
};

struct Domain : Object {
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  int bc[3] = {0, 0, 0};
  bool generated = false;
};

struct Atom_data : Object {
  Domain *domain = nullptr;
  double ghost_cutoff = -1.0, k_b = -1.0;
  bool temperature_process = false, pressure_process = false, msd_process = false;
  std::vector<double> mass, charge;
  std::vector<int32_t> type, mol;
  std::vector<double> pos, vel;
  int64_t n() const { return (int64_t)type.size(); }
};

struct Neighborlist : Object {
  Atom_data *atom_data = nullptr;
  Domain *domain = nullptr;
  double cutoff = 0.0, coef = 1.12347;  // neighborlist.h:134
  bool rebuild_test = false, from_cell_list = false;
  bool all_atom_test = false;  // neighborlist.cpp:161-191, 233-235
};

struct Force_field : Object {
  Atom_data *atom_data = nullptr;
  Neighborlist *neighborlist = nullptr;
  Domain *domain = nullptr;
};

using Mat = std::vector<std::vector<double>>;

void set_elem(Mat &m, int i, int j, double v, double fill) {
  if (i < 0 || j < 0) throw CaslError("negative type index");
  if ((int)m.size() <= i) m.resize(i + 1);
  if ((int)m[i].size() <= j) m[i].resize(j + 1, fill);
  m[i][j] = v;
}

double elem(const Mat &m, int i, int j, double fill) {
  if (i < (int)m.size() && j < (int)m[i].size()) return m[i][j];
  return fill;
}

struct Lj : Force_field {
  double cutoff = 0.0;
  Mat epsilon, sigma, cutoff_list, lambda_s, lambda_e;
  std::vector<double> epsilon_atom, sigma_atom;
  bool by_array = false, by_atom = false, wca = false, cutoff_list_on = false, ignore_intra = false;
  double jump_tol = 0.0;  // lj.cpp:118-127 (jump_fix when set)
  bool monitor_jump = false;
};

struct Ewald_r : Force_field {
  double cutoff = 0.0, alpha = 1.0, k_e = 1.0;
  Mat lambda;
  bool lambda_on = false;
};

struct Ewald_k : Force_field {
  double alpha = 1.0, k_e = 1.0;
  int kmax[3] = {1, 1, 1};
  int slab_axis = -1;  // slab_normal_axis (default z once slab_lz is given, electrostatic_ewald_k.cpp:44-45)
  double slab_lz = 1.0;
  bool slab = false, dipole = false, dipole_once = false;
  double eps_dipole = 0.0;
};

struct Writer : Object {
  Atom_data *atom_data = nullptr;
  Domain *domain = nullptr;
  // writer/atom_data.h:114-165 defaults
  int64_t step[6] = {100, 100, 100, 100, 100, 100};  // energy, temperature, pressure, volume, potential energy, xyz
  bool on[6] = {false, false, false, false, false, false};
  std::string file[6] = {"o_energy", "o_temperature", "o_pressure", "o_volume", "o_potential_energy", "o_xyz"};
  bool xyz_id = false, xyz_vel = false, xyz_acc = false;
  int digits = 6;
  FILE *fp[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  ~Writer() override {
    for (FILE *f : fp)
      if (f) std::fclose(f);
  }
};
enum { W_ENERGY = 0, W_TEMPERATURE, W_PRESSURE, W_VOLUME, W_PE, W_XYZ };

// constraint berendsen / nose_hoover (constraint/berendsen.cpp:25-96, nose_hoover.cpp:25-117)
struct Thermostat : Object {
  bool nose_hoover = false;
  Atom_data *atom_data = nullptr;
  double temperature = -1, coupling = -1, dt = -1, lambda_min = 0.8, lambda_max = 1.25;  // berendsen.h:50-60
  int step = 1;
  int type = 1;                                // nose_hoover.cpp:27-33
  double mass = -1, tau = -1, kb = 1.0;
};

// force_field electrostatic_ewald_slab_correction (electrostatic_ewald_slab_correction.cpp:28-111)
struct Slab_correction : Force_field {
  int axis = 2, kx = 1, ky = 1;
  double lz = 1.0, k_e = 1.0;
};

struct Md_simulator : Object {
  Atom_data *atom_data = nullptr;
  std::vector<Thermostat *> constraint;
  std::vector<Writer *> writer;
  bool initialized = false;  // the reference's setup (and its (0, 0) writer call) happens once
  double time = 0.0;
  bool langevin = false;     // integrator_type velocity_verlet_langevin
  double lgv_temperature = -1, lgv_friction = 0, lgv_kb = -1, lgv_kbt = -1;  // md_simulator.cpp:48-51
  int lgv_rng = CVR_RNG_REFERENCE;
  int64_t lgv_seed = 0;
  std::vector<Force_field *> force_field;
  std::vector<Neighborlist *> neighborlist;
  double dt = -1.0;
  int64_t initial_step = 0, final_step = 0;
  int64_t current_step = 0;  // Md_simulator::current_step: final_step after a run
  double initial_time = 0.0, final_time = 0.0;
  bool vv = false, use_step = false, use_time = false;
  int precision = CVR_PREC_MIXED, policy = CVR_REBUILD_DISPLACEMENT;
  int64_t thermo_step = 0;
  std::string thermo_file, state_file;
};

// ------------------------------------------------------------- interpreter
struct Script {
  std::string path, dir;
  std::map<std::string, std::unique_ptr<Object>> objects;
  std::map<std::string, double> vars;
  Line *cur = nullptr;

  [[noreturn]] void err(const std::string &m) const {
    throw CaslError(path + ":" + std::to_string(cur ? cur->lineno : 0) + ": " + m);
  }
  std::string word() {
    if (cur->done()) err("expected a value");
    return cur->tok[cur->pos++];
  }
  double real() {
    const std::string w = word();
    auto it = vars.find(w);
    if (it != vars.end()) return it->second;
    char *end = nullptr;
    const double v = std::strtod(w.c_str(), &end);
    if (end == w.c_str() || *end) err("expected a real number or variable, got '" + w + "'");
    return v;
  }
  int integer() {
    const double v = real();
    if (v != std::floor(v)) err("expected an integer");
    return (int)v;
  }
  template <typename T>
  T *find(const std::string &nm) {
    auto it = objects.find(nm);
    if (it == objects.end()) err("undefined object '" + nm + "'");
    T *p = dynamic_cast<T *>(it->second.get());
    if (!p) err("object '" + nm + "' has the wrong class");
    return p;
  }

  void create(const std::string &cls, const std::string &type, const std::string &nm) {
    if (objects.count(nm)) err("object name '" + nm + "' already used");
    std::unique_ptr<Object> o;
    if (cls == "domain" && type == "box") o.reset(new Domain);
    else if (cls == "atom_data" && type == "basic") o.reset(new Atom_data);
    else if (cls == "neighborlist" && type == "basic") o.reset(new Neighborlist);
    else if (cls == "force_field" && type == "lj") o.reset(new Lj);
    else if (cls == "force_field" && type == "electrostatic_ewald_r") o.reset(new Ewald_r);
    else if (cls == "force_field" && type == "electrostatic_ewald_k") o.reset(new Ewald_k);
    else if (cls == "force_field" && type == "electrostatic_ewald_slab_correction") o.reset(new Slab_correction);
    else if (cls == "md_simulator" && type == "basic") o.reset(new Md_simulator);
    else if (cls == "writer" && type == "atom_data") o.reset(new Writer);
    else if (cls == "constraint" && (type == "berendsen" || type == "nose_hoover")) {
      auto *t = new Thermostat;
      t->nose_hoover = type == "nose_hoover";
      o.reset(t);
    }
    else err("'" + cls + " " + type + "' is not on the B200 hot path");
    o->name = nm;
    objects[nm] = std::move(o);
  }

  void read_domain(Domain &d) {
    while (!cur->done()) {
      const std::string t = word();
      const char *ax[3][2] = {{"xmin", "xmax"}, {"ymin", "ymax"}, {"zmin", "zmax"}};
      const char *ax2[3][2] = {{"lower_global.x", "upper_global.x"},
                               {"lower_global.y", "upper_global.y"},
                               {"lower_global.z", "upper_global.z"}};
      bool done = false;
      for (int a = 0; a < 3 && !done; ++a) {
        if (t == ax[a][0] || t == ax2[a][0]) d.lo[a] = real(), done = true;
        else if (t == ax[a][1] || t == ax2[a][1]) d.hi[a] = real(), done = true;
      }
      if (done) continue;
      if (t == "boundary_condition" || t == "bc") {
        for (int a = 0; a < 3; ++a) d.bc[a] = integer();
      } else if (t == "generate") {
        d.generated = true;
      } else err("domain: unknown keyword '" + t + "'");
    }
  }

  void add_xyz(Atom_data &a) {
    std::string file;
    bool read_velocity = false, last_frame = false, replace = false;
    while (!cur->done()) {
      const std::string t = word();
      if (t == "file_name") file = word();
      else if (t == "read_velocity") read_velocity = true;
      else if (t == "last_frame") last_frame = true;
      else if (t == "replace_data") replace = true;
      else err("add_xyz_data_file: unknown keyword '" + t + "'");
    }
    if (file.empty()) err("add_xyz_data_file needs file_name");
    const std::string full = (file[0] == '/') ? file : dir + "/" + file;
    std::ifstream f(full);
    if (!f) err("file does not exist : " + full);
    std::vector<std::string> lines;
    std::string l;
    while (std::getline(f, l)) lines.push_back(l);
    // frames: <count> / comment / count lines; last_frame picks the last one
    size_t start = 0;
    if (last_frame) {
      size_t k = 0;
      while (k < lines.size()) {
        std::istringstream is(lines[k]);
        long long m;
        if (!(is >> m) || m <= 0) break;
        start = k;
        k += 2 + (size_t)m;
      }
    }
    std::istringstream hs(lines.size() > start ? lines[start] : "");
    long long m = 0;
    if (!(hs >> m) || m <= 0) err("no atom found in the xyz file. Something is wrong.");
    if (replace && m != a.n()) err("XYZ file is not compatible: Different number of existing atoms");
    for (long long k = 0; k < m; ++k) {
      if (start + 2 + k >= lines.size()) err("xyz file ends early");
      std::istringstream is(lines[start + 2 + (size_t)k]);
      int ty;
      double p[3], v[3] = {0, 0, 0};
      if (!(is >> ty >> p[0] >> p[1] >> p[2])) err("bad xyz line");
      if (read_velocity && !(is >> v[0] >> v[1] >> v[2])) err("bad xyz velocity");
      if (replace) {
        if (ty != a.type[(size_t)k]) err("XYZ file is not compatible: Different atom type order exists.");
        for (int d = 0; d < 3; ++d) {
          a.pos[3 * (size_t)k + d] = p[d];
          a.vel[3 * (size_t)k + d] = v[d];
        }
      } else {
        a.type.push_back(ty);
        a.mol.push_back(-1);
        for (int d = 0; d < 3; ++d) {
          a.pos.push_back(p[d]);
          a.vel.push_back(v[d]);
        }
      }
    }
  }

  // Atom_data::add_random_velocity (atom_data.cpp:597-616): every velocity
  // component uniform in [-amplitude, amplitude] from std::mt19937(seed) in
  // atom order (x, y, z per atom), then the mass-weighted centre-of-mass
  // velocity (owned_velocity_cm, kinetic_energy.cpp:413-457) subtracted from
  // the atoms whose type has a mass.  The same standard-library generator and
  // distribution as the reference build, so the same bits.
  void add_random_velocity(Atom_data &a, unsigned int seed, double amplitude) {
    std::mt19937 mt(seed);
    std::uniform_real_distribution<double> dist(-amplitude, amplitude);
    const int64_t n = a.n();
    a.vel.assign((size_t)n * 3, 0.0);
    for (int64_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) a.vel[3 * (size_t)i + d] = dist(mt);
    auto mass_of = [&](int64_t i) {
      const int t = a.type[(size_t)i];
      return (t >= 0 && t < (int)a.mass.size()) ? a.mass[(size_t)t] : 0.0;
    };
    double vcm[3] = {0.0, 0.0, 0.0}, msum = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      const double m = mass_of(i);
      msum += m;
      for (int d = 0; d < 3; ++d) vcm[d] += a.vel[3 * (size_t)i + d] * m;
    }
    for (int d = 0; d < 3; ++d) vcm[d] = vcm[d] / msum;
    for (int64_t i = 0; i < n; ++i)
      if (mass_of(i) != 0.0)
        for (int d = 0; d < 3; ++d) a.vel[3 * (size_t)i + d] -= vcm[d];
  }

  // The atoms as loaded so far, in the md_simulator state_file format
  // (acceleration zero): a checkpoint of a prepared input state.
  void write_state_file(const Atom_data &a, const std::string &file) {
    const std::string p = (file[0] == '/') ? file : dir + "/" + file;
    FILE *sf = std::fopen(p.c_str(), "wb");
    if (!sf) err("cannot write " + p);
    const int64_t n = a.n();
    std::vector<double> vel = a.vel, acc((size_t)n * 3, 0.0);
    vel.resize((size_t)n * 3, 0.0);
    std::fwrite(&n, 8, 1, sf);
    std::fwrite(a.pos.data(), 8, (size_t)n * 3, sf);
    std::fwrite(vel.data(), 8, (size_t)n * 3, sf);
    std::fwrite(acc.data(), 8, (size_t)n * 3, sf);
    std::fclose(sf);
  }

  // FP64 binary state written by md_simulator state_file: n, pos[3n], vel[3n], acc[3n]
  void add_state_file(Atom_data &a) {
    std::string file;
    bool replace = false;
    while (!cur->done()) {
      const std::string t = word();
      if (t == "file_name") file = word();
      else if (t == "replace_data") replace = true;
      else err("add_state_file: unknown keyword '" + t + "'");
    }
    if (file.empty()) err("add_state_file needs file_name");
    const std::string full = (file[0] == '/') ? file : dir + "/" + file;
    FILE *f = std::fopen(full.c_str(), "rb");
    if (!f) err("file does not exist : " + full);
    int64_t n = 0;
    bool ok = std::fread(&n, 8, 1, f) == 1 && n > 0;
    std::vector<double> p((size_t)std::max<int64_t>(n, 0) * 3), v(p.size());
    ok = ok && std::fread(p.data(), 8, p.size(), f) == p.size() && std::fread(v.data(), 8, v.size(), f) == v.size();
    std::fclose(f);
    if (!ok) err("bad state file " + full);
    if (!replace) err("add_state_file: the file carries no types; load atoms first and use replace_data");
    if (n != a.n()) err("state file is not compatible: different number of existing atoms");
    a.pos = p;
    a.vel = v;
  }

  void read_writer(Writer &w) {
    static const char *stepk[6] = {"energy_step", "temperature_step", "pressure_step", "volume_step",
                                   "potential_energy_step", "xyz_step"};
    static const char *filek[6] = {"file_name_energy", "file_name_temperature", "file_name_pressure",
                                   "file_name_volume", "file_name_potential_energy", "file_name_xyz"};
    while (!cur->done()) {
      const std::string t = word();
      bool done = false;
      for (int k = 0; k < 6 && !done; ++k) {
        if (t == stepk[k]) {
          w.step[k] = integer();
          w.on[k] = w.step[k] > 0;
          done = true;
        } else if (t == filek[k]) {
          w.file[k] = word();
          done = true;
        }
      }
      if (done) continue;
      if (t == "set_atom_data" || t == "atom_data") w.atom_data = find<Atom_data>(word());
      else if (t == "set_domain" || t == "domain") w.domain = find<Domain>(word());
      else if (t == "xyz_output_id") w.xyz_id = integer() != 0;
      else if (t == "xyz_output_velocity") w.xyz_vel = integer() != 0;
      else if (t == "xyz_output_acceleration") w.xyz_acc = integer() != 0;
      else if (t == "precision") {
        w.digits = integer();
        if (w.digits < 1 || w.digits > 17) err("writer precision: 1..17 significant digits");
      } else if (t == "open_files" || t == "close_files") {
        // no effect in the reference either (writer/atom_data.cpp:485-486)
      } else if (t.size() > 10 && (t.compare(t.size() - 10, 10, "_mpi_rank0") == 0 ||
                                   (t.size() > 16 && t.compare(t.size() - 16, 16, "_mpi_per_process") == 0))) {
        integer();  // MPI output switches: one process here
      } else err("writer atom_data: '" + t + "' is not supported on the B200 path");
    }
  }

  void read_thermostat(Thermostat &c) {
    while (!cur->done()) {
      const std::string t = word();
      if (t == "set_atom_data" || t == "atom_data") c.atom_data = find<Atom_data>(word());
      else if (t == "temperature") {
        c.temperature = real();
        if (c.temperature <= 0.0) err("Temperature have to non-negative.");
      } else if (t == "dt") {
        c.dt = real();
        if (c.dt <= 0.0) err("dt have to non-negative.");
      } else if (!c.nose_hoover && t == "coupling") {
        c.coupling = real();
        if (c.coupling <= 0.0) err("coupling have to non-negative.");
      } else if (!c.nose_hoover && t == "step") {
        c.step = integer();
        if (c.step <= 0) err("step have to non-negative.");
      } else if (!c.nose_hoover && (t == "lambda_min" || t == "lambda_max")) {
        const double v = real();
        if (v <= 0.0) err(t + " have to non-negative.");
        (t == "lambda_min" ? c.lambda_min : c.lambda_max) = v;
      } else if (c.nose_hoover && t == "mass") {
        c.mass = real();
        if (c.mass <= 0.0) err("mass have to non-negative.");
      } else if (c.nose_hoover && t == "tau") {
        c.tau = real();
        if (c.tau <= 0.0) err("dt have to non-negative.");
      } else if (c.nose_hoover && t == "type") {
        c.type = integer();
        if (c.type <= 0) err("type have to non-negative.");
      } else if (c.nose_hoover && t == "kb") {
        c.kb = real();
        if (c.kb <= 0.0) err("kb have to non-negative.");
      } else err(std::string(c.nose_hoover ? "constraint nose_hoover" : "constraint berendsen") +
                 ": Unknown variable or command '" + t + "'");
    }
  }

  void read_atom_data(Atom_data &a) {
    while (!cur->done()) {
      const std::string t = word();
      if (t == "ghost_cutoff") a.ghost_cutoff = real();
      else if (t == "k_b") a.k_b = real();
      else if (t == "set_domain" || t == "domain") a.domain = find<Domain>(word());
      else if (t == "add_type_mass") {
        const int i = integer();
        const double v = real();
        if ((int)a.mass.size() <= i) a.mass.resize(i + 1, 0.0);
        a.mass[i] = v;
      } else if (t == "add_type_charge") {
        const int i = integer();
        const double v = real();
        if ((int)a.charge.size() <= i) a.charge.resize(i + 1, 0.0);
        a.charge[i] = v;
      } else if (t == "add_xyz_data_file") {
        add_xyz(a);
      } else if (t == "set_owned_position" || t == "set_owned_velocity") {
        const int i = integer();
        if (i < 0 || i >= a.n()) err(t + ": atom index out of range");
        auto &dst = (t == "set_owned_position") ? a.pos : a.vel;
        for (int d = 0; d < 3; ++d) dst[3 * (size_t)i + d] = real();
      } else if (t == "temperature_process") {
        // atom_data.cpp:147-151; the writer's temperature (and the pressure's kinetic part) is 0 without it
        a.temperature_process = integer() != 0;
      } else if (t == "pressure_process") {
        a.pressure_process = integer() != 0;  // atom_data.cpp:137-146
      } else if (t == "msd_process") {
        // atom_data.cpp:127-136: switches on the reference's displacement
        // counters, read only by its msd writer and by an external virial that
        // its pressure excludes (kinetic_energy.cpp:288); no effect here
        a.msd_process = integer() != 0;
      } else if (t == "add_state_file") {
        add_state_file(a);
      } else if (t == "add_random_velocity") {
        const long long seed = integer();
        double amplitude = real();
        if (amplitude < 0) amplitude = -amplitude;  // atom_data.cpp:280-289
        add_random_velocity(a, (unsigned int)seed, amplitude);
      } else if (t == "write_state_file") {
        write_state_file(a, word());
      } else err("atom_data: '" + t + "' is not on the B200 hot path");
    }
  }

  void read_neighborlist(Neighborlist &nl) {
    while (!cur->done()) {
      const std::string t = word();
      if (t == "set_atom_data" || t == "atom_data") nl.atom_data = find<Atom_data>(word());
      else if (t == "set_domain" || t == "domain") nl.domain = find<Domain>(word());
      else if (t == "cutoff") {
        nl.cutoff = real();
        if (nl.cutoff <= 0.0) err("cutoff have to non-negative.");
      } else if (t == "cutoff_extra_coef") {
        nl.coef = real();
        if (nl.coef < 1.0) err("cutoff_extra_coef must be larger than 1.0");
      } else if (t == "make_verlet_list_from_cell_list" || t == "build_cell_list") {
        nl.from_cell_list = true;
      } else if (t == "rebuild_test") {
        nl.rebuild_test = true;
      } else if (t == "all_atom_test") {
        nl.all_atom_test = true;
      } else if (t == "dt") {
        real();
      } else err("neighborlist: '" + t + "' is not supported on the B200 path");
    }
  }

  void common_ff(Force_field &f, const std::string &t, bool &handled) {
    handled = true;
    if (t == "set_neighborlist" || t == "neighborlist") f.neighborlist = find<Neighborlist>(word());
    else if (t == "set_atom_data" || t == "atom_data") f.atom_data = find<Atom_data>(word());
    else if (t == "set_domain" || t == "domain") f.domain = find<Domain>(word());
    else handled = false;
  }

  void read_lj(Lj &f) {
    while (!cur->done()) {
      const std::string t = word();
      bool h;
      common_ff(f, t, h);
      if (h) continue;
      if (t == "cutoff") {
        f.cutoff = real();
        if (f.cutoff < 0) err("Force field cutoff have to non-negative.");
      } else if (t == "cutoff_list") {
        const int i = integer(), j = integer();
        set_elem(f.cutoff_list, i, j, real(), 0.0);
        f.cutoff_list_on = true;
      } else if (t == "epsilon" || t == "sigma") {
        const int i = integer(), j = integer();
        const double v = real();
        if (v < 0) err("Epsilon have to be non-negative.");
        set_elem(t == "epsilon" ? f.epsilon : f.sigma, i, j, v, 0.0);
        f.by_array = true;
      } else if (t == "lambda_s" || t == "lambda_e") {
        const int i = integer(), j = integer();
        set_elem(t == "lambda_s" ? f.lambda_s : f.lambda_e, i, j, real(), 1.0);
      } else if (t == "epsilon_atom" || t == "sigma_atom") {
        const int i = integer();
        auto &v = (t == "epsilon_atom") ? f.epsilon_atom : f.sigma_atom;
        if ((int)v.size() <= i) v.resize(i + 1, 0.0);
        v[i] = real();
        f.by_atom = true;
      } else if (t == "wca") {
        f.wca = true;
        f.cutoff_list_on = true;
      } else if (t == "ignore_intra_molecule") {
        f.ignore_intra = true;
      } else if (t == "jump_tol") {
        f.jump_tol = real();
        if (f.jump_tol < 0) err("jump_tol have to be non-negative.");
      } else if (t == "monitor_jump") {
        // the reference prints each clamped r^2 to stdout; accepted, no output here
        f.monitor_jump = true;
      } else if (t == "make_off_diagonal_vectors") {
        // no effect on the forces
      } else err("force_field lj: '" + t + "' is not supported on the B200 path");
    }
  }

  void read_ewald_r(Ewald_r &f) {
    while (!cur->done()) {
      const std::string t = word();
      bool h;
      common_ff(f, t, h);
      if (h) continue;
      if (t == "cutoff") f.cutoff = real();  // parsed, unused by the force (electrostatic_ewald_r.cpp:142-226)
      else if (t == "alpha") f.alpha = real();
      else if (t == "k_electrostatic") f.k_e = real();
      else if (t == "lambda") {
        const int i = integer(), j = integer();
        set_elem(f.lambda, i, j, real(), 1.0);
        f.lambda_on = true;
      } else err("force_field electrostatic_ewald_r: '" + t + "' is not supported on the B200 path");
    }
  }

  void read_ewald_k(Ewald_k &f) {
    while (!cur->done()) {
      const std::string t = word();
      bool h;
      common_ff(f, t, h);
      if (h) continue;
      if (t == "alpha") f.alpha = real();
      else if (t == "k_electrostatic") f.k_e = real();
      else if (t == "k_max") f.kmax[0] = f.kmax[1] = f.kmax[2] = integer();
      else if (t == "kx_max") f.kmax[0] = integer();
      else if (t == "ky_max") f.kmax[1] = integer();
      else if (t == "kz_max") f.kmax[2] = integer();
      else if (t == "slab_normal_axis") {
        const std::string v = word();
        f.slab = true;
        if (v == "x") f.slab_axis = 0;
        else if (v == "y") f.slab_axis = 1;
        else if (v == "z") f.slab_axis = 2;
        else err("expected 'x' or 'y' or 'z' for axis.");
      } else if (t == "slab_lz" || t == "slab_thickness") {
        f.slab = true;
        f.slab_lz = real();
        if (f.slab_lz < 0.0) err("slab_lz have to non-negative.");
      } else if (t == "epsilon_dipole") {
        f.eps_dipole = real();
        if (f.eps_dipole < 0) err("'epsilon_dipole' has to be non-negative.");
        f.dipole = true;
      } else if (t == "dipole_once") {
        f.dipole_once = true;  // extension: the textbook term once, not once per k-vector
      } else err("force_field electrostatic_ewald_k: '" + t + "' is not supported on the B200 path");
    }
  }

  void read_slab(Slab_correction &f) {
    while (!cur->done()) {
      const std::string t = word();
      bool h;
      common_ff(f, t, h);
      if (h) continue;
      if (t == "k_max") {
        const int k = integer();
        if (k < 0) err("'k_max' have to non-negative.");
        f.kx = f.ky = k;
      } else if (t == "kx_max") f.kx = integer();
      else if (t == "ky_max") f.ky = integer();
      else if (t == "lz") {
        f.lz = real();
        if (f.lz < 0) err("'lz' has to be non-negative.");
      } else if (t == "slab_normal_axis") {
        const std::string v = word();
        if (v == "x") f.axis = 0;
        else if (v == "y") f.axis = 1;
        else if (v == "z") f.axis = 2;
        else err("expected 'x', 'y' or 'z'.");
      } else if (t == "k_electrostatic") {
        f.k_e = real();
        if (f.k_e < 0) err("k_electrostatic has to be non-negative.");
      } else err("force_field electrostatic_ewald_slab_correction: '" + t + "' is not supported on the B200 path");
    }
  }

  template <typename T>
  void remove_from(std::vector<T *> &v, T *o, const char *what) {
    auto it = std::find(v.begin(), v.end(), o);
    if (it == v.end()) err(std::string("Unknown ") + what + " to remove.");
    v.erase(it);
  }

  void read_md(Md_simulator &m) {
    while (!cur->done()) {
      const std::string t = word();
      if (t == "set_atom_data" || t == "atom_data") m.atom_data = find<Atom_data>(word());
      else if (t == "add_force_field" || t == "force_field") m.force_field.push_back(find<Force_field>(word()));
      else if (t == "add_neighborlist" || t == "neighborlist") m.neighborlist.push_back(find<Neighborlist>(word()));
      else if (t == "add_writer" || t == "writer") m.writer.push_back(find<Writer>(word()));
      else if (t == "add_constraint" || t == "constraint") m.constraint.push_back(find<Thermostat>(word()));
      // md_simulator.cpp:107-150: remove the named object from the simulator's list
      else if (t == "remove_force_field") remove_from(m.force_field, find<Force_field>(word()), "force_field");
      else if (t == "remove_neighborlist") remove_from(m.neighborlist, find<Neighborlist>(word()), "neighborlist");
      else if (t == "remove_writer") remove_from(m.writer, find<Writer>(word()), "writer");
      else if (t == "remove_constraint") remove_from(m.constraint, find<Thermostat>(word()), "constraint");
      else if (t == "integrator_type") {
        const std::string v = word();
        if (v == "velocity_verlet") {
          m.vv = true;
          m.langevin = false;
        } else if (v == "velocity_verlet_langevin") {
          m.vv = true;
          m.langevin = true;
        } else {
          err("integrator_type '" + v + "' is not on the B200 hot path");
        }
      } else if (t == "temperature") {
        m.lgv_temperature = real();
        if (m.lgv_temperature < 0.0) err("Temperature have to non-negative.");
      } else if (t == "friction") {
        m.lgv_friction = real();
        if (m.lgv_friction < 0.0) err("friction have to non-negative.");
      } else if (t == "kb") {
        m.lgv_kb = real();
        if (m.lgv_kb < 0.0) err("kb have to non-negative.");
      } else if (t == "kbt") {
        m.lgv_kbt = real();
      } else if (t == "rng") {
        const std::string v = word();
        if (v == "reference") m.lgv_rng = CVR_RNG_REFERENCE;
        else if (v == "philox") m.lgv_rng = CVR_RNG_PHILOX;
        else err("rng reference|philox");
      } else if (t == "seed") {
        m.lgv_seed = integer();
      } else if (t == "dt") m.dt = real();
      else if (t == "initial_step") m.initial_step = integer(), m.use_step = true;
      else if (t == "final_step") m.final_step = integer(), m.use_step = true;
      else if (t == "final_step_add") {  // md_simulator.cpp:91-97: does not select step mode
        m.final_step += integer();
        m.initial_step = m.current_step;
      }
      else if (t == "initial_time") m.initial_time = real(), m.use_time = true;  // md_simulator.cpp:71-80
      else if (t == "final_time") m.final_time = real(), m.use_time = true;
      else if (t == "precision") {
        const std::string v = word();
        if (v == "mixed") m.precision = CVR_PREC_MIXED;
        else if (v == "fp64") m.precision = CVR_PREC_FP64;
        else err("precision mixed|fp64");
      } else if (t == "rebuild_policy") {
        const std::string v = word();
        if (v == "displacement") m.policy = CVR_REBUILD_DISPLACEMENT;
        else if (v == "reference") m.policy = CVR_REBUILD_REFERENCE;
        else err("rebuild_policy displacement|reference");
      } else if (t == "thermo_step") m.thermo_step = integer();
      else if (t == "thermo_file") m.thermo_file = word();
      else if (t == "state_file") m.state_file = word();
      else if (t == "run") run(m);
      else err("md_simulator: '" + t + "' is not supported on the B200 path");
    }
  }

  // Lj::verify_settings (lj.cpp:149-353): the per-type-pair tables.
  void lj_tables(const Lj &f, int T, std::vector<double> &eps, std::vector<double> &sig, std::vector<double> &cut,
                 bool &use_cut) {
    if (f.by_atom && f.by_array) err("lj: (input_by_atom && input_by_array)");
    eps.assign(T * T, 0.0);
    sig.assign(T * T, 0.0);
    for (int i = 0; i < T; ++i)
      for (int j = 0; j < T; ++j) {
        if (f.by_atom) {
          const double ei = i < (int)f.epsilon_atom.size() ? f.epsilon_atom[i] : 0.0;
          const double ej = j < (int)f.epsilon_atom.size() ? f.epsilon_atom[j] : 0.0;
          const double si = i < (int)f.sigma_atom.size() ? f.sigma_atom[i] : 0.0;
          const double sj = j < (int)f.sigma_atom.size() ? f.sigma_atom[j] : 0.0;
          eps[i * T + j] = (i == j) ? ei : std::sqrt(ei * ej);
          sig[i * T + j] = (i == j) ? si : 0.5 * (si + sj);
        } else {
          eps[i * T + j] = elem(f.epsilon, i, j, 0.0);
          sig[i * T + j] = elem(f.sigma, i, j, 0.0);
        }
      }
    for (int i = 0; i < T; ++i)
      for (int j = 0; j < T; ++j) {
        sig[i * T + j] *= elem(f.lambda_s, i, j, 1.0);
        eps[i * T + j] *= elem(f.lambda_e, i, j, 1.0);
      }
    use_cut = f.cutoff_list_on;
    cut.assign(T * T, 0.0);
    for (int i = 0; i < T; ++i)
      for (int j = 0; j < T; ++j)
        cut[i * T + j] = f.wca ? std::pow(2.0, 1.0 / 6.0) * sig[i * T + j] : elem(f.cutoff_list, i, j, 0.0);
    // the GPU list is full (each pair from both atoms), so the tables must be
    // symmetric; the reference evaluates each pair from one end only
    for (int i = 0; i < T; ++i)
      for (int j = 0; j < i; ++j)
        if (eps[i * T + j] != eps[j * T + i] || sig[i * T + j] != sig[j * T + i] ||
            (use_cut && cut[i * T + j] != cut[j * T + i]))
          err("lj: epsilon, sigma and cutoff_list must be symmetric on the B200 path");
  }

  FILE *wfile(Writer &w, int k) {
    if (!w.fp[k]) {
      std::string f = w.file[k] + (k == W_XYZ ? ".xyz" : ".txt");
      if (f[0] != '/') f = dir + "/" + f;
      w.fp[k] = std::fopen(f.c_str(), "w");
      if (!w.fp[k]) err("cannot write " + f);
    }
    return w.fp[k];
  }

  // Writer::write(i, t) for the scalar outputs (dump_energy.cpp): th is the
  // thermo record of the state after step i (or of the initial state).
  void write_scalars(Md_simulator &m, const Atom_data &a, const Domain &d, int64_t i, double t, const double *th,
                     bool setup) {
    const double V = (d.hi[0] - d.lo[0]) * (d.hi[1] - d.lo[1]) * (d.hi[2] - d.lo[2]);
    const double T = a.temperature_process ? th[CVR_TH_TEMP] : 0.0;
    const double kb = a.k_b > 0 ? a.k_b : 1.0;
    // finalize_pressure_mpi_domain (kinetic_energy.cpp:242-292); not called at setup
    const double P = (a.pressure_process && !setup) ? (double)a.n() * kb * T / V + th[CVR_TH_VIRIAL] / (3.0 * V) : 0.0;
    const double val[5] = {th[CVR_TH_KE], T, P, V,
                           th[CVR_TH_E_LJ] + th[CVR_TH_E_EWR] + th[CVR_TH_E_K] + th[CVR_TH_E_SELF]};
    for (Writer *w : m.writer)
      for (int k = 0; k < 5; ++k)
        if (w->on[k] && i % w->step[k] == 0)
          std::fprintf(wfile(*w, k), "%lld %.*g %.*g\n", (long long)i, w->digits, t, w->digits, val[k]);
  }

  // dump_xyz_serial (dump_xyz_serial.cpp:34-67): positions wrapped into the box
  void write_xyz(Md_simulator &m, const Domain &d, int64_t i, const std::vector<int32_t> &type,
                 std::vector<double> pos, const std::vector<double> &vel, const std::vector<double> &acc) {
    const size_t n = type.size();
    for (size_t q = 0; q < n; ++q)
      for (int a = 0; a < 3; ++a)
        if (d.bc[a]) {
          const double L = d.hi[a] - d.lo[a];
          double &x = pos[3 * q + a];
          x -= L * std::floor((x - d.lo[a]) / L);
        }
    for (Writer *w : m.writer) {
      if (!w->on[W_XYZ] || i % w->step[W_XYZ] != 0) continue;
      FILE *f = wfile(*w, W_XYZ);
      const int g = w->digits;
      std::fprintf(f, "%zu\nAtom\n", n);
      for (size_t q = 0; q < n; ++q) {
        std::fprintf(f, "%d", (int)type[q]);
        if (w->xyz_id) std::fprintf(f, " %zu", q);
        std::fprintf(f, " %.*g %.*g %.*g", g, pos[3 * q], g, pos[3 * q + 1], g, pos[3 * q + 2]);
        if (w->xyz_vel) std::fprintf(f, " %.*g %.*g %.*g", g, vel[3 * q], g, vel[3 * q + 1], g, vel[3 * q + 2]);
        if (w->xyz_acc) std::fprintf(f, " %.*g %.*g %.*g", g, acc[3 * q], g, acc[3 * q + 1], g, acc[3 * q + 2]);
        std::fprintf(f, "\n");
      }
      std::fflush(f);
    }
  }

  // The reference's writer calls (md_simulator.cpp:548, :664): (0, 0) after
  // setup, then (i, time before the step) after every step i.  Runs in chunks
  // that end where an xyz frame is due; one thermo record per step.
  template <typename Check>
  void run_with_writers(Md_simulator &m, const Atom_data &a, const Domain &d, cvr_ctx *ctx, Check &check) {
    const size_t n = (size_t)a.n();
    std::vector<double> pos(3 * n), vel(3 * n), acc(3 * n), th(CVR_N_THERMO);
    int64_t xs = 0;  // smallest xyz step
    for (Writer *w : m.writer)
      if (w->on[W_XYZ]) xs = xs ? std::min(xs, w->step[W_XYZ]) : w->step[W_XYZ];
    if (!m.initialized) {
      check(cvr_compute_forces(ctx, acc.data(), th.data()));
      write_scalars(m, a, d, 0, 0.0, th.data(), true);
      if (xs) {
        check(cvr_get_state(ctx, pos.data(), vel.data(), nullptr));
        write_xyz(m, d, 0, a.type, pos, vel, acc);
      }
      m.time = m.dt * (double)m.initial_step;
      m.initialized = true;
    }
    std::vector<double> rec;
    int64_t i = m.initial_step;
    while (i < m.final_step) {
      int64_t e = std::min(m.final_step, i + 4096);
      if (xs) e = std::min(e, ((i + xs - 1) / xs) * xs + 1);
      const int64_t len = e - i;
      rec.assign((size_t)len * CVR_N_THERMO, 0.0);
      check(cvr_run(ctx, len, 1, rec.data()));
      for (int64_t r = 0; r < len; ++r) {
        write_scalars(m, a, d, i + r, m.time, &rec[(size_t)r * CVR_N_THERMO], false);
        m.time += m.dt;
      }
      if (xs && (e - 1) % xs == 0) {
        check(cvr_get_state(ctx, pos.data(), vel.data(), acc.data()));
        write_xyz(m, d, e - 1, a.type, pos, vel, acc);
      }
      i = e;
    }
    for (Writer *w : m.writer)
      for (FILE *f : w->fp)
        if (f) std::fflush(f);
  }

  void run(Md_simulator &m) {
    Atom_data *a = m.atom_data;
    if (!a) err("md_simulator: set_atom_data first");
    if (!m.vv) err("md_simulator: set 'integrator_type velocity_verlet' (the reference leaves it unset)");
    if (m.dt < 0) err("expected 'dt' input");
    // Md_simulator::verify_settings (md_simulator.cpp:276-282) and setup
    // (:508-512): times become steps as `(int)time / dt` -- the time is
    // truncated to an integer before the division, as the reference does.
    if (m.use_time && m.use_step) err("simulator md: verify_settings: cannot use both 'time' and 'step'.");
    if (!(m.use_time || m.use_step)) err("simulator md: verify_settings: please assign 'time' or 'step' variables.");
    if (m.use_time) {
      m.initial_step = (int)((double)(int)m.initial_time / m.dt);
      m.final_step = (int)((double)(int)m.final_time / m.dt);
    }
    if (m.neighborlist.size() != 1) err("the B200 path takes exactly one neighborlist");
    Neighborlist *nl = m.neighborlist[0];
    Domain *d = a->domain ? a->domain : nl->domain;
    if (!d) err("atom_data: set_domain first");
    if (a->n() == 0) err("no atoms");
    int T = (int)std::max(a->mass.size(), a->charge.size());
    for (int32_t t : a->type) T = std::max(T, t + 1);
    std::vector<double> mass(T, 0.0), charge(T, 0.0);
    for (int t = 0; t < T; ++t) {
      mass[t] = t < (int)a->mass.size() ? a->mass[t] : 0.0;
      charge[t] = t < (int)a->charge.size() ? a->charge[t] : 0.0;
    }
    cvr_ctx *ctx = nullptr;
    int rc = cvr_create(&ctx, d->lo, d->hi, d->bc, T, mass.data(), charge.data(), 0);
    if (rc) err("cvr_create failed (" + std::to_string(rc) + ")");
    auto check = [&](int r) {
      if (r) {
        char buf[512];
        cvr_last_error(ctx, buf, sizeof(buf));
        const std::string msg = buf;
        cvr_destroy(ctx);
        err("B200 path: " + msg);
      }
    };
    check(cvr_set_precision(ctx, m.precision));
    const int policy = nl->rebuild_test ? CVR_REBUILD_EVERY_STEP : m.policy;
    check(cvr_set_neighborlist(ctx, nl->cutoff, nl->coef, a->ghost_cutoff, policy));
    if (nl->all_atom_test) check(cvr_set_all_atom_test(ctx, 1));
    for (Force_field *f : m.force_field) {
      if (auto *lj = dynamic_cast<Lj *>(f)) {
        std::vector<double> eps, sig, cut;
        bool use_cut = false;
        lj_tables(*lj, T, eps, sig, cut, use_cut);
        check(cvr_set_lj(ctx, lj->cutoff, eps.data(), sig.data(), use_cut ? cut.data() : nullptr,
                         lj->ignore_intra ? 1 : 0));
        if (lj->jump_tol > 0) check(cvr_set_lj_jump_tol(ctx, lj->jump_tol));
      } else if (auto *er = dynamic_cast<Ewald_r *>(f)) {
        std::vector<double> lam(T * T, 1.0);
        for (int i = 0; i < T; ++i)
          for (int j = 0; j < T; ++j) lam[i * T + j] = elem(er->lambda, i, j, 1.0);
        check(cvr_set_ewald_r(ctx, er->alpha, er->k_e, er->lambda_on ? lam.data() : nullptr, -1.0));
      } else if (auto *sc = dynamic_cast<Slab_correction *>(f)) {
        check(cvr_set_ewald_slab_correction(ctx, sc->axis, sc->lz, sc->kx, sc->ky, sc->k_e));
      } else if (auto *ek = dynamic_cast<Ewald_k *>(f)) {
        check(cvr_set_ewald_k(ctx, ek->alpha, ek->kmax[0], ek->kmax[1], ek->kmax[2], ek->k_e));
        if (ek->slab || ek->dipole)
          check(cvr_set_ewald_k_geometry(ctx, ek->slab ? (ek->slab_axis < 0 ? 2 : ek->slab_axis) : -1, ek->slab_lz,
                                         ek->dipole ? (ek->dipole_once ? CVR_DIPOLE_ONCE : CVR_DIPOLE_REFERENCE) : 0,
                                         ek->eps_dipole));
      }
    }
    check(cvr_set_integrator(ctx, m.dt, a->k_b > 0 ? a->k_b : 1.0));
    if (m.langevin)
      check(cvr_set_langevin(ctx, m.lgv_temperature, m.lgv_friction, m.lgv_kb, m.lgv_kbt, m.lgv_rng,
                             (uint64_t)m.lgv_seed));
    if (m.constraint.size() > 1) err("the B200 path takes one thermostat constraint");
    for (Thermostat *t : m.constraint) {
      // the reference reads temperature_ (0 unless temperature_process): its Berendsen
      // factor would sit at lambda_max and its Nose-Hoover zeta would turn NaN
      if (!a->temperature_process) err("thermostat constraints need 'atom_data temperature_process 1'");
      if (t->nose_hoover)
        check(cvr_set_nose_hoover(ctx, t->temperature, t->type, t->mass, t->tau, t->kb, t->dt));
      else
        check(cvr_set_berendsen(ctx, t->temperature, t->coupling, t->dt, t->step, t->lambda_min, t->lambda_max));
    }
    bool any_mol = false;
    for (int32_t v : a->mol) any_mol = any_mol || v >= 0;
    check(cvr_set_state(ctx, a->n(), a->pos.data(), a->vel.data(), a->type.data(), any_mol ? a->mol.data() : nullptr));
    const int64_t nsteps = m.final_step - m.initial_step;
    const int64_t every = m.thermo_step > 0 ? m.thermo_step : 0;
    std::vector<double> thermo((size_t)std::max<int64_t>(1, every > 0 ? nsteps / every : 1) * CVR_N_THERMO);
    bool writers = false;
    for (Writer *w : m.writer)
      for (int k = 0; k < 6; ++k) writers = writers || w->on[k];
    if (!writers) {
      check(cvr_run(ctx, nsteps, every, every > 0 ? thermo.data() : nullptr));
      if (!m.initialized) m.time = m.dt * (double)m.initial_step;
      m.initialized = true;
      m.time += m.dt * (double)nsteps;
    } else {
      if (every > 0) err("thermo_step with writers: use the writers' outputs");
      run_with_writers(m, *a, *d, ctx, check);
    }
    check(cvr_get_state(ctx, a->pos.data(), a->vel.data(), nullptr));
    if (!m.thermo_file.empty() && every > 0) {
      const std::string p = (m.thermo_file[0] == '/') ? m.thermo_file : dir + "/" + m.thermo_file;
      FILE *tf = std::fopen(p.c_str(), "w");
      if (!tf) err("cannot write " + p);
      std::fprintf(tf, "# step ke temperature e_lj e_ewald_r e_ewald_k e_self virial pressure builds\n");
      for (int64_t r = 0; r < nsteps / every; ++r) {
        for (int q = 0; q < CVR_N_THERMO; ++q)
          std::fprintf(tf, q ? " %.17g" : "%.17g", thermo[(size_t)r * CVR_N_THERMO + q]);
        std::fprintf(tf, "\n");
      }
      std::fclose(tf);
    }
    if (!m.state_file.empty()) {
      std::vector<double> acc((size_t)a->n() * 3);
      check(cvr_get_state(ctx, nullptr, nullptr, acc.data()));
      const std::string p = (m.state_file[0] == '/') ? m.state_file : dir + "/" + m.state_file;
      FILE *sf = std::fopen(p.c_str(), "wb");
      if (!sf) err("cannot write " + p);
      const int64_t n = a->n();
      std::fwrite(&n, 8, 1, sf);
      std::fwrite(a->pos.data(), 8, (size_t)n * 3, sf);
      std::fwrite(a->vel.data(), 8, (size_t)n * 3, sf);
      std::fwrite(acc.data(), 8, (size_t)n * 3, sf);
      std::fclose(sf);
    }
    cvr_destroy(ctx);
    m.current_step = m.final_step;  // the reference's run loop leaves current_step == final_step
  }

  void execute() {
    std::vector<Line> lines = lex(path);
    for (Line &L : lines) {
      cur = &L;
      const std::string first = word();
      if (first == "exit") break;
      if (first == "real" || first == "int") {
        const std::string nm = word();
        double v = real();
        if (first == "int") v = std::floor(v);
        vars[nm] = v;
        continue;
      }
      if (first == "domain" || first == "atom_data" || first == "neighborlist" || first == "force_field" ||
          first == "md_simulator" || first == "writer" || first == "constraint" || first == "unique") {
        const std::string type = word();
        const std::string nm = word();
        create(first, type, nm);
        cur->pos = cur->tok.size();
        continue;
      }
      auto it = objects.find(first);
      if (it == objects.end()) err("unknown command or object '" + first + "'");
      Object *o = it->second.get();
      if (auto *d = dynamic_cast<Domain *>(o)) read_domain(*d);
      else if (auto *a = dynamic_cast<Atom_data *>(o)) read_atom_data(*a);
      else if (auto *nl = dynamic_cast<Neighborlist *>(o)) read_neighborlist(*nl);
      else if (auto *lj = dynamic_cast<Lj *>(o)) read_lj(*lj);
      else if (auto *er = dynamic_cast<Ewald_r *>(o)) read_ewald_r(*er);
      else if (auto *ek = dynamic_cast<Ewald_k *>(o)) read_ewald_k(*ek);
      else if (auto *sc = dynamic_cast<Slab_correction *>(o)) read_slab(*sc);
      else if (auto *m = dynamic_cast<Md_simulator *>(o)) read_md(*m);
      else if (auto *w = dynamic_cast<Writer *>(o)) read_writer(*w);
      else if (auto *th = dynamic_cast<Thermostat *>(o)) read_thermostat(*th);
    }
  }
};

}  // namespace

extern "C" int cvr_casl_run_file(const char *path, char *err, size_t err_len) {
  if (err && err_len) err[0] = '\0';
  if (!path) return CVR_ERR_INVALID;
  try {
    Script s;
    s.path = path;
    s.dir = dir_of(path);
    s.execute();
  } catch (const std::exception &e) {
    if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
    return CVR_ERR_INVALID;
  }
  return CVR_OK;
}
