/* caviar_b200.h -- C ABI of the B200 (sm_100a) MD timestep hot path.
 *
 * One opaque context per periodic system.  The context owns every device
 * buffer and a CUDA stream; host pointers passed in are borrowed for the call
 * only.  Every function returns CVR_OK (0) or a CVR_ERR_* code and never
 * exits the process; cvr_last_error() gives the message.  A context is not
 * thread safe: use one per host thread.
 *
 * Each entry point replaces one piece of the reference's object interface
 * (CAVIAR, paths relative to its project root).  The reference shares state
 * between objects through Atom_data's public vectors; here that state lives
 * in the context, in HBM.
 */
#ifndef CAVIAR_B200_H
#define CAVIAR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define CVR_OK 0
#define CVR_ERR_INVALID 1   /* bad argument (reference: error->all on read/verify) */
#define CVR_ERR_CUDA 2      /* CUDA runtime error */
#define CVR_ERR_NAN 3       /* NaN acceleration (md_simulator.cpp:584-590) */
#define CVR_ERR_STATE 4     /* wrong call order, e.g. cvr_run before cvr_set_state */
#define CVR_ERR_GEOMETRY 5  /* box/cutoff combination the path cannot represent */
#define CVR_ERR_CAPACITY 6  /* neighbour list or cell capacity exceeded and regrow failed */
#define CVR_ERR_NOMEM 7     /* device allocation failed */

/* ------------------------------------------------------------ option values */
#define CVR_PREC_MIXED 0    /* FP32 pair/k-space math; FP64 positions, S(k), energy/virial sums */
#define CVR_PREC_FP64 1     /* everything FP64 (the comparison form) */

#define CVR_REBUILD_DISPLACEMENT 0 /* rebuild when an atom moved > skin/2 since the last build */
#define CVR_REBUILD_REFERENCE 1    /* also on any owned wrap or ghost-set change (neighborlist.cpp:91-139) */
#define CVR_REBUILD_EVERY_STEP 2   /* Neighborlist rebuild_test (neighborlist.cpp:98-101) */

/* Thermo record written by cvr_run / cvr_get_scalars, in this order. */
#define CVR_TH_STEP 0
#define CVR_TH_KE 1        /* kinetic energy, COM removed when all axes are periodic (kinetic_energy.cpp:58-72) */
#define CVR_TH_TEMP 2      /* 2 KE / (k_b dof)  (kinetic_energy.cpp:193-202) */
#define CVR_TH_E_LJ 3      /* LJ energy of the linear force-shifted potential (lj.cpp:439-448) */
#define CVR_TH_E_EWR 4     /* Ewald real-space energy over the list pairs */
#define CVR_TH_E_K 5       /* Ewald k-space energy (electrostatic_ewald_k/energy.cpp:61-107) */
#define CVR_TH_E_SELF 6    /* Ewald self energy (energy.cpp:31-50) */
#define CVR_TH_VIRIAL 7    /* virialForce: LJ + Ewald-r, each pair once (lj.cpp:451-453) */
#define CVR_TH_PRESSURE 8  /* N k_b T / V + virial / 3V (kinetic_energy.cpp:242-300) */
#define CVR_TH_BUILDS 9    /* Verlet-list builds so far */
#define CVR_N_THERMO 10

typedef struct cvr_ctx cvr_ctx;

/* Domain box + Atom_data type table.
 * Replaces: Domain::read xmin..zmax/boundary_condition/generate (domain.cpp:206-266),
 *           Atom_data add_type_mass / add_type_charge (atom_data.cpp:224-245, 574-595).
 * lo, hi: box corners; bc: 1 periodic, 0 not; mass, charge: n_types each (host).
 * device: CUDA ordinal. */
int cvr_create(cvr_ctx **out, const double lo[3], const double hi[3], const int bc[3], int n_types,
               const double *mass, const double *charge, int device);
void cvr_destroy(cvr_ctx *ctx);

/* Neighborlist basic: cutoff, cutoff_extra_coef (rl = cutoff * coef), and
 * Atom_data ghost_cutoff; rebuild policy (CVR_REBUILD_*).
 * Replaces: Neighborlist::read (neighborlist.cpp:193-251), init (:313-406),
 *           update_is_needed (:91-139). */
int cvr_set_neighborlist(cvr_ctx *ctx, double cutoff, double cutoff_extra_coef, double ghost_cutoff,
                         int rebuild_policy);

/* force_field lj: cutoff; epsilon, sigma: n_types*n_types row-major; cutoff_list:
 * n_types*n_types or NULL; ignore_intra_molecule: 0/1.
 * Replaces: Lj::read (lj.cpp:42-147), verify_settings (:149-353),
 *           calculate_acceleration (:355-483). */
int cvr_set_lj(cvr_ctx *ctx, double cutoff, const double *epsilon, const double *sigma,
               const double *cutoff_list, int ignore_intra_molecule);

/* Neighborlist all_atom_test (neighborlist.cpp:161-191, 233-235, 517-519): a
 * debugging mode of the reference whose list holds every owned pair once and
 * every owned atom with every ghost image, with no distance test (LJ keeps
 * its cutoff test; the Ewald real-space sum, which has none, runs over all of
 * them).  Forces come from an all-pairs kernel over the direct displacements
 * and the ghost images of this step's wrapped positions (rebuilt every
 * step); cvr_get_pairs returns that pair set (for at most 4096 atoms, else
 * CVR_ERR_CAPACITY).  At most CVR_ALL_ATOM_MAX atoms (O(n^2) work).  on = 0
 * returns to the Verlet list. */
#define CVR_ALL_ATOM_MAX 65536
int cvr_set_all_atom_test(cvr_ctx *ctx, int on);

/* force_field lj jump_tol v (lj.cpp:118-127, 423-432): a debugging clamp of
 * the reference; after the cutoff test, a pair closer than sqrt(jump_tol)
 * gets the LJ force coefficient (and LJ virial and energy) of r^2 = jump_tol,
 * applied to its true displacement.  0 turns it off (the default).
 * Replaces: Lj::read jump_tol and the clamp in Lj::calculate_acceleration. */
int cvr_set_lj_jump_tol(cvr_ctx *ctx, double jump_tol);

/* force_field electrostatic_ewald_r: alpha, k_electrostatic; lambda: n_types^2
 * same-molecule scaling or NULL; cutoff < 0 keeps the reference's behaviour of
 * summing every list pair (electrostatic_ewald_r.cpp:142-226 has no cutoff test).
 * Replaces: Electrostatic_ewald_r::read (:38-88), calculate_acceleration (:115-317). */
int cvr_set_ewald_r(cvr_ctx *ctx, double alpha, double k_electrostatic, const double *lambda, double cutoff);

/* force_field electrostatic_ewald_k: alpha, kx/ky/kz_max, k_electrostatic.
 * Uses the reference's k-set: the first (2kx)(2ky)(2kz) vectors of the
 * [-kmax,kmax]^3 \ {0} enumeration (initialize.cpp:184-222).
 * Replaces: Electrostatic_ewald_k::read (:48-143), initialize (initialize.cpp:31-92),
 *           calculate_potential_k_coef_cmplx (:117-146), calculate_acceleration (:161-294). */
int cvr_set_ewald_k(cvr_ctx *ctx, double alpha, int kx_max, int ky_max, int kz_max, double k_electrostatic);

/* Electrostatic_ewald_k geometry keywords (electrostatic_ewald_k.cpp:87-126,
 * initialize.cpp:49-115): slab_axis 0/1/2 (slab_normal_axis x/y/z, -1 off)
 * replaces that axis' length by slab_lz in the k-vectors and the volume;
 * dipole_mode != 0 (epsilon_dipole set) adds the surrounding-medium term
 * F_i += q_i E, E = -(sum_j q_j r_j) k_e 4 pi / (V (1 + 2 epsilon_dipole)),
 * and 0.5 (k_e 4 pi / (V (1 + 2 eps))) |M|^2 to the k-space energy.
 * CVR_DIPOLE_REFERENCE adds the force term once per k-vector, as the
 * reference does (inside its k loop, electrostatic_ewald_k.cpp:197-223);
 * CVR_DIPOLE_ONCE adds it once. */
#define CVR_DIPOLE_REFERENCE 1
#define CVR_DIPOLE_ONCE 2
int cvr_set_ewald_k_geometry(cvr_ctx *ctx, int slab_axis, double slab_lz, int dipole_mode, double epsilon_dipole);

/* force_field electrostatic_ewald_slab_correction (electrostatic_ewald_slab_correction.cpp:44-181
 * and its initialize/field/energy files): the slab correction term for a
 * system periodic in two directions, with the reference's keywords
 * slab_normal_axis (0/1/2; -1 turns it off), lz (>= the box along that axis),
 * kx_max, ky_max (1..8 here) and k_electrostatic.  Its field includes the
 * reference's dipole term, which uses the normal dipole moment of the previous
 * force call (the first call has none); its energy is added to
 * thermo[CVR_TH_E_K]. */
int cvr_set_ewald_slab_correction(cvr_ctx *ctx, int slab_axis, double lz, int kx_max, int ky_max, double k_e);

/* md_simulator basic: dt; atom_data k_b.
 * Replaces: Md_simulator::read dt / integrator_type velocity_verlet (md_simulator.cpp:58-233). */
int cvr_set_integrator(cvr_ctx *ctx, double dt, double k_b);

/* Langevin velocity Verlet, the reference's `integrator_type
 * velocity_verlet_langevin` (md_simulator.cpp:670-811) with its keywords
 * temperature, friction, kb, kbt (md_simulator.cpp:198-222): per step one
 * Gaussian vector eta per atom, v += dt/2 a + b eta, r += c v, forces,
 * v = a_c v + b eta + dt/2 a, a_c = (2 - g dt)/(2 + g dt),
 * b = sqrt(kbt g dt / 2) (or kb T in place of kbt), c = 2 dt / (2 + g dt).
 * rng: CVR_RNG_REFERENCE draws eta from the reference's own three streams
 * (std::mt19937 seeded 1, 2, 3 with std::normal_distribution, on the host,
 * the same numbers the reference uses); CVR_RNG_PHILOX draws it on the GPU
 * from a counter-based generator keyed by (seed, step, atom). */
#define CVR_RNG_REFERENCE 0
#define CVR_RNG_PHILOX 1
int cvr_set_langevin(cvr_ctx *c, double temperature, double friction, double kb, double kbt, int rng,
                     uint64_t seed);

/* Verlet-list search kernel (a tuning and testing knob; both kernels build
 * the same pair set, Neighborlist::update_verlet_list_from_cell_list,
 * neighborlist.cpp:515-573): CVR_LIST_AUTO picks by system size (a warp per
 * atom up to 65536 atoms, else a thread per atom), CVR_LIST_THREAD one
 * thread per atom, CVR_LIST_WARP one warp per atom.  Takes effect at the
 * next list build. */
/* k-space force kernel of the mixed form (a tuning and testing knob; both
 * compute the reference's k-space force, electrostatic_ewald_k.cpp:197-234):
 * CVR_KFORCE_AUTO takes the tensor cores (tcgen05 TF32 MMAs with hi/lo
 * split operands, FP32-level sums) when k_max_z <= 11 and k_max <= 11 on
 * every axis, else the CUDA-core kernel; CVR_KFORCE_CUDA_CORES always the
 * latter.  The FP64 form always uses the CUDA-core kernel. */
#define CVR_KFORCE_AUTO 0
#define CVR_KFORCE_CUDA_CORES 1
int cvr_set_kspace_force_kernel(cvr_ctx *ctx, int kind);

#define CVR_LIST_AUTO 0
#define CVR_LIST_THREAD 1
#define CVR_LIST_WARP 2
int cvr_set_list_kernel(cvr_ctx *ctx, int kind);

/* CVR_PREC_MIXED (default) or CVR_PREC_FP64.  No reference counterpart
 * (the reference is FP64 only).  In the mixed form, a cubic box whose listed
 * pairs stay below L/2 apart and that has at most 256 cells per axis gets
 * fixed-point pair displacements: positions as round(r 2^32 / L) mod 2^32,
 * the minimum image as a wrapping int32 difference (resolution L / 2^32). */
int cvr_set_precision(cvr_ctx *ctx, int precision);

/* Thermostat applied after the velocity update of each velocity-Verlet step,
 * where the reference calls Constraint::apply_thermostat
 * (md_simulator.cpp:619-627).  One at a time; not with the Langevin integrator.
 * cvr_set_berendsen: `constraint berendsen` (constraint/berendsen.cpp:44-131):
 *   every `step` steps v *= clamp(sqrt(1 + (dt/coupling)(T0/T - 1)), lambda_min, lambda_max)
 *   (the reference's defaults: step 1, lambda_min 0.8, lambda_max 1.25).
 * cvr_set_nose_hoover: `constraint nose_hoover` (constraint/nose_hoover.cpp:36-180):
 *   zeta += dt zeta_dot, type 1: zeta_dot = (-kb n_df T / mass)(T0/T - 1),
 *   type 2: zeta_dot = (-1/tau)(T0/T - 1); then a -= zeta v.
 * T is the instantaneous temperature after the step's velocity update. */
int cvr_set_berendsen(cvr_ctx *c, double temperature, double coupling, double dt, int step, double lambda_min,
                      double lambda_max);
int cvr_set_nose_hoover(cvr_ctx *c, double temperature, int type, double mass, double tau, double kb, double dt);
int cvr_clear_thermostat(cvr_ctx *c);

/* Atoms from HOST memory: pos, vel: n*3 (x,y,z per atom, = Vector<double> AoS);
 * type: n; mol: n molecule indices or NULL (-1 = none).  Atom i gets id i.
 * The arrays are read before the call returns.  On a context that keeps its
 * atom count and settings, the next run's setup (list build, first forces)
 * runs inside this call, beside the velocity copy; a list overflow there is
 * reported here.
 * Replaces: Atom_data::add_atom (atom_data.cpp:487-521) / add_xyz_data_file
 *           (atom_data/add_xyz_data_file.cpp:22-168). */
int cvr_set_state(cvr_ctx *ctx, int64_t n, const double *pos, const double *vel, const int32_t *type,
                  const int32_t *mol);

/* Build the Verlet list at the current positions (force = 1), or only if the
 * rebuild policy says so (force = 0).  *rebuilt (nullable) = 1 if it did.
 * Replaces: Neighborlist::build (neighborlist.cpp:66-88). */
int cvr_build_neighbors(cvr_ctx *ctx, int force, int *rebuilt);

/* Accelerations of every enabled force field at the current positions and
 * list, plus energies and virial.  acc: n*3 host (nullable), in id order;
 * thermo: CVR_N_THERMO host (nullable).
 * Replaces: Md_simulator::re_calculate_acc's force part (md_simulator.cpp:370-373),
 *           Force_field::energy (force_field.h:36-50). */
int cvr_compute_forces(cvr_ctx *ctx, double *acc, double *thermo);

/* Advance nsteps velocity-Verlet steps (the first call also does setup:
 * list + forces).  Every thermo_every steps (0 = never) a CVR_N_THERMO record
 * is appended to thermo (host, nullable; capacity nsteps/thermo_every records).
 * Replaces: Md_simulator::run / step (md_simulator.cpp:235-274, 382-485),
 *           integrate_velocity_verlet (:555-668), setup (:504-549). */
int cvr_run(cvr_ctx *ctx, int64_t nsteps, int64_t thermo_every, double *thermo);

/* Current state to HOST memory in id order (each nullable): pos, vel, acc n*3.
 * Positions are wrapped into the box the way Domain::fix_position does. */
int cvr_get_state(cvr_ctx *ctx, double *pos, double *vel, double *acc);

/* Canonical pair set of the current list: 5 int32 per pair
 * (id_a < id_b, image shift sx, sy, sz of b), sorted.  Returns the count
 * (< 0 on error); out may be NULL to count only.
 * Replaces: reading Neighborlist::neighlist (neighborlist.h:88) + ghost ids. */
int64_t cvr_get_pairs(cvr_ctx *ctx, int32_t *out);

/* S(k) of the used k-vectors from the last force evaluation: 2 doubles
 * (re, im) per vector (host).  Returns the count (< 0 on error).
 * Replaces: reading Electrostatic_ewald_k::potential_k_coef_cmplx (electrostatic_ewald_k.h:83). */
int64_t cvr_get_sk(cvr_ctx *ctx, double *out);

/* Last thermo record (CVR_N_THERMO doubles, host). */
int cvr_get_scalars(cvr_ctx *ctx, double *thermo);

/* Diagnostics. */
int cvr_last_error(const cvr_ctx *ctx, char *buf, size_t len);
int64_t cvr_launch_count(const cvr_ctx *ctx);     /* kernels launched by this context so far */
void *cvr_get_stream(const cvr_ctx *ctx);         /* the cudaStream_t the context launches on */
/* out[0..len): n, cells x, y, z, list capacity per atom, list builds, lanes
 * per atom, k-vectors, stencil radius, largest neighbour count, error bits,
 * step, total list entries (index 12 costs a device-to-host copy), 1 if the
 * mixed form's pair kernel uses fixed-point displacements (cubic box, see
 * cvr_set_precision), 1 if the k-space force runs on the tensor cores (see
 * cvr_set_kspace_force_kernel). */
int cvr_get_info(const cvr_ctx *ctx, int64_t *out, int len);

/* Arithmetic-pipe peak of `device` for the compute side of the roofline (no
 * reference counterpart): a kernel of independent fused multiply-adds only
 * (FP32, or FP64 when fp64 != 0) filling every SM, `iters` rounds of 128 FMAs
 * per thread, best of 5 launches timed with CUDA events; *tflops = 2 flops
 * per FMA / time, *ms = that launch's time.  Synchronous. */
int cvr_measure_fma_peak(int device, int fp64, int iters, double *tflops, double *ms);

/* Kernel timing: when on, CUDA events bracket every launch of the named
 * kernel class on the context's stream; cvr_kernel_time returns the summed
 * milliseconds and the launch count since the last reset. */
#define CVR_KT_PAIR 0      /* LJ + Ewald real-space pair force */
#define CVR_KT_KSPACE 1    /* S(k) + k-space force */
#define CVR_KT_INTEGRATE 2 /* velocity-Verlet kernels */
#define CVR_KT_BUILD 3     /* binning + Verlet-list build */
#define CVR_N_KT 4
int cvr_set_kernel_timing(cvr_ctx *ctx, int on);
int cvr_kernel_time(cvr_ctx *ctx, int kind, double *ms, int64_t *launches);

/* -------------------------------------------------------- batched replicas */
/* Many small independent periodic boxes advanced together: one persistent
 * CTA per replica for all steps, every replica in one CUDA graph launch, the
 * threads per CTA of each size class picked by timing candidates on the
 * state (autotuner).  No reference counterpart: the reference runs one system
 * per process and its one-ghost-image scheme cannot hold boxes smaller than
 * twice the list radius (exchange_ghost_single_md_domain.cpp:59-99).
 * Physics per replica: LJ with the reference's linear force shift
 * (lj.cpp:439-448) up to rc_lj, Ewald real space (electrostatic_ewald_r.cpp:196-198)
 * up to rc_r, both <= L/2 (minimum image), Ewald k space over the reference's
 * k-set (initialize.cpp:184-222, electrostatic_ewald_k.cpp:197-234), velocity
 * Verlet.  Mixed precision: FP32 pair and k-space math on hi/lo FP32
 * coordinates, FP64 positions, velocities, S(k) and energies.
 * Limits: 2048 atoms per replica, 4 types, k_max <= 6. */
typedef struct cvr_batch cvr_batch;
#define CVR_BATCH_N_OUT 8 /* per replica: ke, e_lj, e_ewald_r, e_ewald_k, e_self, virial, temperature, steps */
/* n_atoms, box_len: n_rep each (cubes [0, L)); mass, charge: n_types. */
int cvr_batch_create(cvr_batch **out, int n_rep, const int64_t *n_atoms, const double *box_len, int n_types,
                     const double *mass, const double *charge, int device);
void cvr_batch_destroy(cvr_batch *b);
/* eps, sigma: n_types^2; rc_lj, rc_r: n_rep each (<= L/2); alpha; k_max; k_e; dt. */
int cvr_batch_set_forces(cvr_batch *b, const double *eps, const double *sigma, const double *rc_lj,
                         const double *rc_r, double alpha, int kmax, double k_e, double dt);
/* All replicas' atoms concatenated in replica order: pos, vel n*3 (host), type n. */
int cvr_batch_set_state(cvr_batch *b, const double *pos, const double *vel, const int32_t *type);
/* nsteps steps of every replica in one graph launch (the first call tunes the
 * launch shapes); out (host, nullable): n_rep * CVR_BATCH_N_OUT at the end. */
int cvr_batch_run(cvr_batch *b, int64_t nsteps, double *out);
/* pos, vel, acc (each nullable) n*3; acc = FP32 force / mass of the current positions (after a run). */
int cvr_batch_get_state(cvr_batch *b, double *pos, double *vel, double *acc);
/* n_rep, atoms, classes, then per class: replicas, largest replica, threads per CTA, atom groups per k-run. */
int cvr_batch_info(const cvr_batch *b, int64_t *out, int len);
int cvr_batch_last_error(const cvr_batch *b, char *buf, size_t len);
void *cvr_batch_stream(const cvr_batch *b);

/* ---------------------------------------------------------------- adjoint */
/* Gradient of the trajectory loss J = (1/M) sum_{t=1..M} U(r_t) of M
 * velocity-Verlet steps (md_simulator.cpp:555-668) with respect to the
 * initial positions and velocities, eps/sigma per type pair and per-type
 * charges.  No reference counterpart (the reference has no gradients).
 * One periodic cube [0, L)^3, minimum image (rc_lj, rc_r <= L/2), at most 2
 * types; U = LJ with the reference's linear force shift (lj.cpp:439-448) +
 * Ewald real space with cutoff rc_r (electrostatic_ewald_r.cpp:196-198) +
 * Ewald k space over the reference's k-set (initialize.cpp:184-222) + self
 * energy (electrostatic_ewald_k/energy.cpp:31-50).  CVR_PREC_MIXED: FP32 pair
 * and k-space terms, FP64 sums, state and cotangents; CVR_PREC_FP64: all FP64.
 * Parameter vectors theta: eps[T*T], sigma[T*T], charge[T]; the gradient of a
 * shared off-diagonal value is written to both of its entries.
 * Forces here are F (not F/m); pos/vel/force/u/w arrays are n*3 (host). */
typedef struct cvr_adj cvr_adj;
int cvr_adj_create(cvr_adj **out, int64_t n, double box_len, int n_types, const double *mass, int precision,
                   int device);
void cvr_adj_destroy(cvr_adj *a);
/* charge[T], eps[T*T], sigma[T*T] symmetric; k_max <= 10. */
int cvr_adj_set_params(cvr_adj *a, const double *charge, const double *eps, const double *sigma, double rc_lj,
                       double alpha, double rc_r, int kmax, double k_e, double dt);
/* The initial state of the loss (and the positions of the force calls). */
int cvr_adj_set_state(cvr_adj *a, const double *pos, const double *vel, const int32_t *type);
/* Forces at the state's positions; energy[4] = {lj, ewald_r, ewald_k, self}; dU = dU/dtheta.  Outputs nullable. */
int cvr_adj_forces(cvr_adj *a, double *force, double *energy, double *dU);
/* The hand-written VJP: w = (dF/dr)^T u and g = u . dF/dtheta at the state's positions. */
int cvr_adj_force_vjp(cvr_adj *a, const double *u, double *w, double *g);
/* J of nsteps steps (forward only); final pos/vel nullable. */
int cvr_adj_loss(cvr_adj *a, int64_t nsteps, double *loss, double *pos_out, double *vel_out);
/* J and dJ/d(pos0, vel0, theta), checkpoints every checkpoint_every steps. */
int cvr_adj_loss_grad(cvr_adj *a, int64_t nsteps, int64_t checkpoint_every, double *loss, double *g_pos,
                      double *g_vel, double *g_theta);
int cvr_adj_last_error(const cvr_adj *a, char *buf, size_t len);
void *cvr_adj_stream(const cvr_adj *a);

/* ------------------------------------------------------------------ CASL */
/* Run a CASL script that uses the hot-path objects with the reference's own
 * keywords (domain box, atom_data basic, neighborlist basic, force_field lj /
 * electrostatic_ewald_r / electrostatic_ewald_k, md_simulator basic, real/int
 * variables); `sim run` advances the system on the GPU.  Extensions on
 * md_simulator: precision mixed|fp64, rebuild_policy displacement|reference,
 * thermo_step N, thermo_file "f", state_file "f" (binary: int64 n, then n*3
 * FP64 positions, velocities, accelerations in id order).  Off-path objects
 * and keywords are rejected with a message in err.
 * Replaces: CAVIAR::execute -> Input::read for these objects
 * (src/caviar/CAVIAR.cpp:70-88, interpreter/input.cpp:128-199). */
int cvr_casl_run_file(const char *path, char *err, size_t err_len);

/* ---------------------------------------------------------- no allocation */
/* Capacity, in complex doubles (16 B each), of the fixed device array behind
 * cvr_structure_factor_noalloc: 262144 = 4 MiB per GPU that loads the library. */
#define CVR_NOALLOC_SK_SCRATCH 262144

/* Ewald structure factor S(k) = sum_j q_j exp(i k.r_j), k = 2 pi (nx/Lx, ny/Ly, nz/Lz)
 * over the reference's k-set (the first (2kx)(2ky)(2kz) vectors of the
 * [-kmax, kmax]^3 \ {0} enumeration), for callers that cannot allocate device
 * memory: it calls no cudaMalloc, cudaFree or allocating library routine.
 * No counterpart in the reference (there S(k) lives inside Electrostatic_ewald_k).
 *
 * Callers that need it run inside a host program whose allocator owns the
 * GPU's memory (a framework's caching allocator, an engine that reserves its
 * pool up front), are plug-ins forbidden to allocate after start-up, or cannot
 * afford the device-wide synchronisation of cudaMalloc/cudaFree mid-run.
 *
 * pos: DEVICE, n*3 doubles (x, y, z per atom); q: DEVICE, n charges;
 * box_len: HOST, 3 box lengths; sk: DEVICE, 2*(2kx)(2ky)(2kz) doubles (re, im)
 * written in k-set order; stream: cudaStream_t (NULL = default stream);
 * err/err_len: optional host buffer for a message.  Launches on the current
 * device and returns without synchronising.
 *
 * Scratch: the chunk partial sums use one fixed device array of
 * CVR_NOALLOC_SK_SCRATCH complex doubles per GPU, held until process exit.
 * Limit: k_max <= 30 per axis (at most 216000 k-vectors, which always fit);
 * a larger k_max, n <= 0 or n > 2^30 -> CVR_ERR_INVALID before any launch.
 * The first call on each device looks up that array's device address and
 * keeps it for the process; make it before any stream capture, and do not
 * call again on a device after cudaDeviceReset.  All calls share the array and it keeps the last
 * call's contents (every partial is written before it is read, so nothing
 * needs clearing); calls whose kernels overlap on the GPU race on it. */
int cvr_structure_factor_noalloc(const double *pos, const double *q, int64_t n, const double box_len[3],
                                 int kx_max, int ky_max, int kz_max, double *sk, void *stream, char *err,
                                 size_t err_len);

#ifdef __cplusplus
}
#endif
#endif
