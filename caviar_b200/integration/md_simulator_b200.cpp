// md_simulator_b200.cpp -- `md_simulator b200` / `b200_fp64` for the
// reference (CAVIAR): Md_simulator::run (src/caviar/objects/md_simulator.cpp:
// 235-274) done by the B200 path through the C ABI of include/caviar_b200.h.
//
// Compiled against the reference's headers and linked with the reference's
// objects and libcaviar_b200.so (oracle/Makefile target `ref_b200` builds the
// reference harness that way).  Everything before `run` -- the script's
// domain, atom_data, neighborlist, force_field and md_simulator keywords --
// is the reference's own code; run() hands the atoms and settings to one GPU
// context, advances final_step - initial_step velocity-Verlet steps there,
// and writes the final owned positions (wrapped into the box as
// Domain::fix_position leaves them), velocities and accelerations back into
// Atom_data.  A failing call ends the run through the reference's own error
// path (Error::all, which prints and exits, interpreter/error.cpp:27-31).
#include "caviar/objects/md_simulator/b200.h"

#include "caviar/interpreter/error.h"
#include "caviar/interpreter/output.h"
#include "caviar/objects/atom_data.h"
#include "caviar/objects/domain.h"
#include "caviar/objects/force_field.h"
#include "caviar/objects/force_field/electrostatic_ewald_k.h"
#include "caviar/objects/force_field/electrostatic_ewald_r.h"
#include "caviar/objects/force_field/lj.h"
#include "caviar/objects/neighborlist.h"
#include "caviar/utility/interpreter_io_headers.h"

#include "caviar_b200.h"

#include <string>
#include <vector>

CAVIAR_NAMESPACE_OPEN

namespace md_simulator
{

  namespace
  {
    // Neighborlist::all_atom_test is protected (neighborlist.h); a derived
    // class may name it, which yields a pointer to the member of the base.
    struct NeighborlistSettings : Neighborlist
    {
      static bool all_atom_test_of(const Neighborlist *n) { return n->*(&NeighborlistSettings::all_atom_test); }
    };

    // T x T row-major copy of a reference type-pair table (missing entries 0).
    std::vector<double> flat(const std::vector<std::vector<Real_t>> &m, size_t T)
    {
      std::vector<double> out(T * T, 0.0);
      for (size_t i = 0; i < T && i < m.size(); ++i)
        for (size_t j = 0; j < T && j < m[i].size(); ++j)
          out[i * T + j] = m[i][j];
      return out;
    }
  } // namespace

  B200::B200(CAVIAR *fptr) : B200(fptr, CVR_PREC_MIXED) {}

  B200::B200(CAVIAR *fptr, int precision) : Md_simulator{fptr}, precision_{precision}
  {
    FC_OBJECT_INITIALIZE_INFO
  }

  B200::~B200() {}

  B200_fp64::B200_fp64(CAVIAR *fptr) : B200(fptr, CVR_PREC_FP64) {}

  bool B200::run()
  {
    output->info("MD started (B200 path).");
    verify_settings();
    if (dt < 0.0)
      error->all(FC_FILE_LINE_FUNC, "expected 'dt' input");
    if (integrator_type != Integrator_t::Velocity_verlet)
      error->all(FC_FILE_LINE_FUNC, "md_simulator b200: integrator_type velocity_verlet only");
    if (use_time)
    { // Md_simulator::setup (md_simulator.cpp:508-512)
      initial_step = (int)initial_time / dt;
      final_step = (int)final_time / dt;
    }
    if (neighborlist.size() != 1)
      error->all(FC_FILE_LINE_FUNC, "md_simulator b200: exactly one neighborlist");

    Atom_data *ad = atom_data;
    Domain *dom = ad->domain;
    if (!dom)
      error->all(FC_FILE_LINE_FUNC, "md_simulator b200: atom_data has no domain");
    auto &own = ad->atom_struct_owned;
    const int64_t n = (int64_t)own.position.size();
    const auto &tp = ad->atom_type_params;
    size_t T = std::max(tp.mass.size(), tp.charge.size());
    for (auto t : own.type)
      T = std::max(T, (size_t)t + 1);
    std::vector<double> mass(T, 0.0), charge(T, 0.0);
    for (size_t t = 0; t < T; ++t)
    {
      if (t < tp.mass.size())
        mass[t] = tp.mass[t];
      if (t < tp.charge.size())
        charge[t] = tp.charge[t];
    }

    const double lo[3] = {dom->lower_global.x, dom->lower_global.y, dom->lower_global.z};
    const double hi[3] = {dom->upper_global.x, dom->upper_global.y, dom->upper_global.z};
    const int bc[3] = {dom->boundary_condition.x, dom->boundary_condition.y, dom->boundary_condition.z};
    cvr_ctx *ctx = nullptr;
    auto check = [&](int rc) {
      if (rc != CVR_OK)
      {
        char buf[512] = {0};
        if (ctx)
          cvr_last_error(ctx, buf, sizeof(buf));
        const std::string msg = std::string("md_simulator b200: ") + (buf[0] ? buf : "C ABI call failed") +
                                " (status " + std::to_string(rc) + ")";
        if (ctx)
          cvr_destroy(ctx);
        error->all(FC_FILE_LINE_FUNC, msg);
      }
    };
    check(cvr_create(&ctx, lo, hi, bc, (int)T, mass.data(), charge.data(), 0));
    check(cvr_set_precision(ctx, precision_));
    Neighborlist *nl = neighborlist[0];
    // the reference's own rebuild trigger (neighborlist.cpp:91-139)
    check(cvr_set_neighborlist(ctx, nl->cutoff, nl->cutoff_extra_coef, ad->ghost_cutoff, CVR_REBUILD_REFERENCE));
    if (NeighborlistSettings::all_atom_test_of(nl)) // neighborlist.cpp:161-191
      check(cvr_set_all_atom_test(ctx, 1));
    for (auto *f : force_field)
    {
      if (auto *lj = dynamic_cast<force_field::Lj *>(f))
      {
        if (!lj->settings_verified)
        { // lj.cpp:149-353: mixing rules, WCA cutoffs, table sizes
          lj->verify_settings();
          lj->settings_verified = true;
        }
        const std::vector<double> eps = flat(lj->epsilon, T), sig = flat(lj->sigma, T);
        const bool cl = lj->wca || lj->cutoff_list_activated;
        const std::vector<double> cut = cl ? flat(lj->cutoff_list, T) : std::vector<double>();
        check(cvr_set_lj(ctx, lj->cutoff, eps.data(), sig.data(), cl ? cut.data() : nullptr,
                         lj->ignore_intra_molecule ? 1 : 0));
        if (lj->jump_fix) // lj.cpp:118-127, 423-432 (monitor_jump's per-pair print is not made)
          check(cvr_set_lj_jump_tol(ctx, lj->jump_tol));
      }
      else if (auto *er = dynamic_cast<force_field::Electrostatic_ewald_r *>(f))
      {
        const std::vector<double> lam = er->lambda_is_set ? flat(er->lambda, T) : std::vector<double>();
        // cutoff < 0: every list pair, as the reference (electrostatic_ewald_r.cpp:142-226)
        check(cvr_set_ewald_r(ctx, er->alpha, er->k_electrostatic, er->lambda_is_set ? lam.data() : nullptr, -1.0));
      }
      else if (auto *ek = dynamic_cast<force_field::Electrostatic_ewald_k *>(f))
      {
        check(cvr_set_ewald_k(ctx, ek->alpha, ek->kx_max, ek->ky_max, ek->kz_max, ek->k_electrostatic));
      }
      else
        error->all(FC_FILE_LINE_FUNC, "md_simulator b200: force_field " + f->object_class_name +
                                          " is not on this path (lj, electrostatic_ewald_r, electrostatic_ewald_k)");
    }
    check(cvr_set_integrator(ctx, dt, ad->k_b));

    std::vector<int32_t> type(own.type.begin(), own.type.end());
    bool any_mol = false;
    std::vector<int32_t> mol((size_t)n, -1);
    for (size_t i = 0; i < (size_t)n && i < own.molecule_index.size(); ++i)
    {
      mol[i] = own.molecule_index[i];
      any_mol = any_mol || mol[i] >= 0;
    }
    // Vector<double> is {x, y, z}: the owned arrays are AoS doubles, n * 3
    check(cvr_set_state(ctx, n, &own.position[0].x, &own.velocity[0].x, type.data(), any_mol ? mol.data() : nullptr));
    const int64_t nsteps = final_step - initial_step;
    if (nsteps > 0)
      check(cvr_run(ctx, nsteps, 0, nullptr));
    else
      check(cvr_compute_forces(ctx, nullptr, nullptr));
    if (own.acceleration.size() != own.position.size())
      own.acceleration.resize(own.position.size());
    check(cvr_get_state(ctx, &own.position[0].x, &own.velocity[0].x, &own.acceleration[0].x));
    cvr_destroy(ctx);
    current_step = final_step;
    output->info("MD finished (B200 path).");
    return true;
  }

} // md_simulator

CAVIAR_NAMESPACE_CLOSE
