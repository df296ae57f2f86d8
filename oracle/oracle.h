/* oracle.h -- CPU FP64 restatement of CAVIAR's per-timestep particle path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA path is
 * compared against (tests/, __graft_entry__.smoke, bench.py's cpu_baseline
 * leg); the product (caviar_b200/) never links or calls it.
 *
 * Parity pinning: the restatement is checked bit-for-bit against the
 * unmodified reference compiled from its own sources (oracle/_ref, see
 * Makefile and ref_harness.cpp) and against the published Ewald golden
 * forces (tests/golden/).  Every function cites the reference file:line it
 * follows; paths are relative to the reference project root.
 */
#ifndef CAVIAR_ORACLE_H
#define CAVIAR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sys orc_sys;

/* Rebuild policies of the Verlet list.
 *  ORC_REBUILD_DISPLACEMENT: rebuild only when an atom moved more than half
 *    the skin since the last build; positions are wrapped at rebuilds only.
 *  ORC_REBUILD_REFERENCE: the reference's trigger -- any owned wrap, a change
 *    of ghost count, or any owned/ghost displacement above half the skin
 *    (md_simulator.cpp:487-502, neighborlist.cpp:91-139); wrap every step.
 *  ORC_REBUILD_EVERY_STEP: Neighborlist `rebuild_test` (neighborlist.cpp:98-101). */
enum { ORC_REBUILD_DISPLACEMENT = 0, ORC_REBUILD_REFERENCE = 1, ORC_REBUILD_EVERY_STEP = 2 };

orc_sys *orc_create(const double lo[3], const double hi[3], const int bc[3],
                    int n_types, const double *mass, const double *charge);
void orc_destroy(orc_sys *s);

int orc_set_atoms(orc_sys *s, int64_t n, const double *pos, const double *vel,
                  const int32_t *type, const int32_t *mol);
void orc_set_neighborlist(orc_sys *s, double cutoff, double cutoff_extra_coef,
                          double ghost_cutoff, int all_atom_test);
/* eps, sigma: n_types*n_types row-major; cutoff_list may be NULL. jump_tol <= 0 disables. */
void orc_set_lj(orc_sys *s, double cutoff, const double *eps, const double *sigma,
                const double *cutoff_list, int ignore_intra_molecule, double jump_tol);
/* lambda may be NULL; cutoff < 0 keeps the reference's behaviour (no cutoff test). */
void orc_set_ewald_r(orc_sys *s, double alpha, double k_electrostatic, const double *lambda,
                     double cutoff);
void orc_set_ewald_k(orc_sys *s, double alpha, int kx_max, int ky_max, int kz_max,
                     double k_electrostatic);
void orc_set_integrator(orc_sys *s, double dt, double k_b, int rebuild_policy);

/* Md_simulator::setup (md_simulator.cpp:504-549): wrap, ghosts, list, forces. */
int orc_setup(orc_sys *s);
/* One velocity-Verlet step (md_simulator.cpp:555-668). */
int orc_step(orc_sys *s);
/* Build the list at the current positions (setup's wrap+ghost+build(true)) without forces. */
int orc_build_list(orc_sys *s);
/* Forces at the current positions with the current list (re_calculate_acc's force part). */
int orc_compute_forces(orc_sys *s);

/* Canonical pair set (id_a < id_b, shift of b), 5 int32 per pair, sorted.
 * Returns the pair count; out may be NULL to only count. */
int64_t orc_pairs(orc_sys *s, int32_t *out);
int orc_get_state(const orc_sys *s, double *pos, double *vel, double *acc);
int64_t orc_n_kvec_used(const orc_sys *s);
/* S(k) of the used k-vectors from the last force call: 2 doubles (re, im) each. */
int orc_get_sk(const orc_sys *s, double *out);

/* Scalars, in this order:
 *  0 virial (virialForce: LJ + Ewald-r, each pair once)
 *  1 kinetic energy (COM-removed when all axes are periodic, kinetic_energy.cpp:58-72)
 *  2 LJ energy of the linear force-shifted pair potential (the restatement's own)
 *  3 Ewald real-space energy over the list pairs (the restatement's own)
 *  4 Ewald k-space energy (electrostatic_ewald_k/energy.cpp:61-107)
 *  5 Ewald self energy (energy.cpp:31-50)
 *  6 number of list builds so far
 *  7 number of ghosts at the last ghost exchange
 *  8 degrees of freedom (kinetic_energy.cpp:680-718)
 */
#define ORC_N_SCALARS 9
int orc_get_scalars(orc_sys *s, double *out);
/* Evaluate energies (scalars 2..5) at the current positions and list. */
int orc_energy(orc_sys *s);

/* ---------------------------------------------------------------- replicas
 * Small periodic boxes (L < 2 rl, which the reference's one-ghost-image
 * scheme cannot represent): minimum-image all-pairs LJ (linear force shift,
 * cutoff rc_lj) + Ewald real space with cutoff rc_r (<= L/2), Ewald k space
 * over the reference's k-set (first (2k)^3 vectors of [-k,k]^3 \ {0}), FP64.
 * pos/vel/acc: n*3; type: n; box: L (cube [0, L)).  Writes acc and, when
 * energy is non-NULL, {e_lj, e_ewald_r, e_ewald_k, e_self, virial}. */
void orc_replica_forces(int64_t n, const double *pos, const int32_t *type, double L, int n_types,
                        const double *mass, const double *charge, const double *eps, const double *sigma,
                        double rc_lj, double alpha, double rc_r, int kmax, double k_e, double *acc,
                        double *energy);
/* nsteps velocity-Verlet steps (kick, drift, wrap into [0, L), force, kick). */
void orc_replica_run(int64_t n, double *pos, double *vel, double *acc, const int32_t *type, double L, int n_types,
                     const double *mass, const double *charge, const double *eps, const double *sigma,
                     double rc_lj, double alpha, double rc_r, int kmax, double k_e, double dt, int64_t nsteps);

/* ----------------------------------------------------------------- adjoint
 * FP64 gradient of the trajectory loss J = (1/M) sum_{t=1..M} U(r_t) of M
 * velocity-Verlet steps on one periodic cube (minimum image, cutoffs <= L/2):
 * LJ (linear force shift, cutoff rc_lj), Ewald real space with an explicit
 * cutoff rc_r, Ewald k space over the reference's k-set, self energy.
 * eps/sigma: nt*nt symmetric; gradients of a shared off-diagonal value are
 * written to both entries.  Forces here are F (not F/m). */
#define ORC_ADJ_TMAX 4
typedef struct orc_adj orc_adj;
orc_adj *orc_adj_create(int64_t n, double L, int nt, const double *mass, const double *charge, const double *eps,
                        const double *sigma, double rc_lj, double alpha, double rc_r, int kmax, double k_e, double dt,
                        const int32_t *type);
void orc_adj_destroy(orc_adj *a);
void orc_adj_set_params(orc_adj *a, const double *eps, const double *sigma, const double *charge);
/* energy: {lj, ewald_r, ewald_k, self}; dU_*: dU/dtheta.  Outputs nullable. */
void orc_adj_forces(orc_adj *a, const double *pos, double *force, double *energy, double *dU_eps, double *dU_sig,
                    double *dU_q);
/* w = (dF/dr)^T u and u . dF/dtheta. */
void orc_adj_force_vjp(orc_adj *a, const double *pos, const double *u, double *w, double *g_eps, double *g_sig,
                       double *g_q);
double orc_adj_loss(orc_adj *a, const double *pos0, const double *vel0, int64_t M, double *pos_out, double *vel_out);
/* Checkpoints (r, v) every K steps; the reverse sweep re-runs each segment. */
double orc_adj_loss_grad(orc_adj *a, const double *pos0, const double *vel0, int64_t M, int64_t K, double *g_pos,
                         double *g_vel, double *g_eps, double *g_sig, double *g_q);

#ifdef __cplusplus
}
#endif
#endif
