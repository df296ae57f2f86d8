// cvr_abi.cu -- host orchestration behind the C ABI of include/caviar_b200.h.
//
// One context = one periodic system resident in HBM.  A step is a fixed
// sequence of stream launches:
//   kick_drift -> [bin_count, scan x3, bin_scatter, rank, permute, build_list]
//   -> pair (LJ + Ewald r) -> [sk_partial, sk_reduce, kforce] -> kick -> [thermo]
// The bracketed build kernels exit at once unless kick_drift raised the
// rebuild flag, so the host never waits on the device inside a run.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <array>
#include <random>
#include <tuple>
#include <vector>

#include "../../include/caviar_b200.h"
#include "cvr_build.cuh"
#include "cvr_device.cuh"
#include "cvr_force.cuh"
#include "cvr_kforce_tc.cuh"

// Stencil radius in cells: cells are at least rl / R wide, so every pair
// within rl is at most R cells apart on each axis (R = 1 was measured: the
// pair kernel gathers better, the list search costs more, the step is slower).
#ifndef CVR_STENCIL_R
#define CVR_STENCIL_R 2
#endif

using namespace cvr;

namespace {

#ifndef CVR_KCH
#define CVR_KCH 64
#endif
#ifndef CVR_KMG
#define CVR_KMG 3
#endif
constexpr int KCH = CVR_KCH;  // atoms per S(k) chunk
constexpr int KMG = CVR_KMG;  // m-values per S(k) thread
constexpr int KMZ = 16;    // k-force: Z[m] held in registers up to this many m-values (kmax_z < 16)
#ifndef CVR_KF_WMAX
#define CVR_KF_WMAX 8
#endif
constexpr int KF_WMAX = CVR_KF_WMAX;  // k-force: most warps per block of 32 atoms
constexpr int KRW = 16;    // warps of the S(k) chunk reduction
constexpr size_t KF_COEF_SMEM = 72 * 1024;  // k-force: shared memory for staged column coefficients

struct DBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

struct KT {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  size_t used = 0;
  double ms = 0;
  int64_t launches = 0;
};

}  // namespace

struct cvr_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // side stream of the S(k) chain (phase tables, chunk partials, reduction),
  // which runs beside the pair kernel; joined before the k-space force
  cudaStream_t kstream = nullptr;
  cudaEvent_t k_fork = nullptr, k_join = nullptr;
  // domain + types
  double lo[3], hi[3], L[3];
  int bc[3];
  int n_types = 0;
  std::vector<double> mass, charge;
  // neighbour list
  bool nl_set = false;
  double cutoff = 0, coef = 1.12347, gc = 0;
  int policy = CVR_REBUILD_DISPLACEMENT;
  // LJ
  bool lj_on = false;
  double lj_cut = 0;
  std::vector<double> eps, sig, cutl;
  int ignore_intra = 0;
  // Ewald r
  bool ewr_on = false;
  double ewr_alpha = 1, ewr_ke = 1, ewr_cut = -1;
  std::vector<double> lam;
  // Ewald k
  bool ewk_on = false;
  double ewk_alpha = 1, ewk_ke = 1;
  int kmax[3] = {1, 1, 1};
  int slab_axis = -1;     // Ewald k-space slab geometry: this axis' length is slab_lz (initialize.cpp:49-79)
  double slab_lz = 1.0;
  int dipole_mode = 0;    // 0 off, CVR_DIPOLE_REFERENCE (n_k times), CVR_DIPOLE_ONCE
  double eps_dipole = 0;
  // force_field electrostatic_ewald_slab_correction
  bool sc_on = false;
  int sc_axis = 2, sc_kx = 1, sc_ky = 1;
  double sc_lz = 1.0, sc_ke = 1.0;
  double *d_sc_partial{}, *d_sc_chi{}, *d_sc_state{};
  int sc_parts = 0;
  double *d_dipole{};     // E[3], M[3]
  double *d_dip_part{};
  int dip_parts = 0;
  // integrator
  double dt = 0.001, k_b = 1.0;
  int precision = CVR_PREC_MIXED;
  // state
  int64_t n = 0;
  bool have_state = false, list_valid = false, setup_done = false, use_mol = false;
  int64_t step = 0;
  int R = CVR_STENCIL_R, nc[3] = {1, 1, 1}, ncells = 1;
  double w[3] = {1, 1, 1};
  int tpa = 1, log2_tpa = 0, cap = 0, n_pad = 0;
  int fixed = 0;  // mixed form: fixed-point pair displacements (choose_fixed)
  bool refreshed = false;  // refresh() has run for the current settings and atom count
  int list_kernel = CVR_LIST_AUTO;  // list search kernel (cvr_set_list_kernel)
  // k space
  int nk = 0, nxy = 0, kM = 1, kp = 2;
  std::vector<int4> kint;
  std::vector<double> fk;
  std::vector<int2> kxy, kpm;
  double e_self = 0, total_mass = 0, q2_sum = 0;  // q2_sum = sum of q_i^2 over the atoms
  double jump_tol = 0;                              // LJ jump_tol (lj.cpp:118-127), <= 0 off
  bool all_atom = false;                            // neighborlist all_atom_test (neighborlist.cpp:161-191)
  // device memory
  std::vector<std::pair<void **, size_t>> atom_bufs;
  // per atom
  double *x{}, *y{}, *z{}, *vx{}, *vy{}, *vz{};
  void *ax{}, *ay{}, *az{}, *x4{};
  float4 *xb{};
  int *cell{}, *id{}, *type{}, *mol{};
  int8_t *gcls{};
  double *tx{}, *ty{}, *tz{}, *tvx{}, *tvy{}, *tvz{};
  int *tid{}, *ttype{}, *tmol{}, *tcell{}, *slot_atom{}, *perm{};
  double *stage{};
  int *stage_i{};
  int *ncount{};
  // snapshot for replay after a list overflow
  std::vector<std::pair<void *, void *>> snap_pairs;
  std::vector<size_t> snap_bytes;
  // cells
  int *cell_count{}, *cell_start{}, *cell_fill{}, *block_sums{};
  unsigned long long *d_type_hist{};  // atoms per type of the last cvr_set_state (+ out-of-range count)
  // list
  uint32_t *nlist{};
  size_t nlist_bytes = 0;
  // flags: [flag, err, max_count, n_builds, build_epoch, clamp_mark]
  int *flags{};
  double *d_mass_inv{}, *d_mass{}, *d_charge{};
  void *d_coef{};
  // partials
  double *ev_part{}, *ke_part{}, *ek_part{};
  int n_ev_blocks = 0, n_ke_blocks = 0, n_ek_blocks = 0;
  double *d_thermo{};
  size_t thermo_cap = 0;
  // k space device
  double *d_fk{};
  int2 *d_kxy{}, *d_kpm{};
  // S(k) columns actually summed (one of each mirror pair) and each column's source
  std::vector<int2> kxyc;
  std::vector<int> ksrc;
  int2 *d_kxyc{};
  int *d_ksrc{};
  std::vector<int> kmir;  // per summed column: the column taken from it, or -1
  int *d_kmir{};
  int ncomp = 0;
  double2 *d_kpartial{}, *d_sk{};
  void *d_ptab{}, *d_kcoef{};
  int nchunks = 0;
  int kf_warps = 1;  // k-force warps per block of 32 atoms
  int kf_tc = 1;     // k-force columns per staged tile of one warp
  // tensor-core k-space force (mixed form): coefficient image and its tiles
  float *d_kimg{};
  int kimg_tiles = 0;
  int kforce_kind = CVR_KFORCE_AUTO;  // cvr_set_kspace_force_kernel
  // diagnostics
  std::string err;
  int64_t launches = 0;
  double last_thermo[CVR_N_THERMO] = {0};
  bool timing = false;
  KT kt[CVR_N_KT];
  // CUDA graphs of one step (plain, thermo); rebuilt when buffers move
  bool use_graphs = true;
  int64_t epoch = 0, graph_epoch = -1;
  // [deferred kick of the previous step in the head][tail: 0 kick deferred,
  // 1 kick, 2 kick + thermo record]
  cudaGraphExec_t g_step[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int64_t graph_kernels[2] = {0, 0};
  long long *counters{};
  long long counter_src[2] = {0, 0};
  // Langevin integrator (md_simulator.cpp:670-811)
  int integrator = 0;  // 0 velocity Verlet, 1 velocity Verlet Langevin
  double lgv_temperature = -1, lgv_friction = 0, lgv_kb = -1, lgv_kbt = -1;
  int lgv_rng = CVR_RNG_REFERENCE;
  uint64_t lgv_seed = 0;
  // the reference's three streams (md_simulator.cpp:45-47): std::mt19937 seeded 1, 2, 3, unit normals
  std::mt19937 gen[3];
  std::normal_distribution<double> ndist[3];
  double *d_eta{};                          // [3][n], caller's atom order
  double *h_eta[2] = {nullptr, nullptr};    // pinned staging, double-buffered
  cudaEvent_t eta_done[2] = {nullptr, nullptr};
  int64_t eta_n = 0;                        // atoms the noise buffers are sized for
  // thermostat applied after each velocity-Verlet step (0 none, 1 Berendsen, 2 Nose-Hoover)
  ThermostatArgs tstat{};
  double *d_tscal{};  // [0] Berendsen factor, [1] Nose-Hoover zeta (carried across calls)
  std::vector<void *> all_allocs;
};

// ------------------------------------------------------------------ helpers
namespace {

int fail(cvr_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

#define CVR_CUDA(ctx, call)                                                                        \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail((ctx), CVR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int dalloc(cvr_ctx *c, T **p, size_t count) {
  if (*p) {
    cudaFree(*p);
    auto it = std::find(c->all_allocs.begin(), c->all_allocs.end(), (void *)*p);
    if (it != c->all_allocs.end()) c->all_allocs.erase(it);
    *p = nullptr;
  }
  if (count == 0) count = 1;
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, count * sizeof(T));
  if (e != cudaSuccess) return fail(c, CVR_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  cudaMemsetAsync(q, 0, count * sizeof(T), c->stream);
  c->all_allocs.push_back(q);
  *p = (T *)q;
  c->epoch++;
  return CVR_OK;
}

inline int grid_for(int64_t n, int block) { return (int)((n + block - 1) / block); }

template <typename real>
DevState<real> dev_state(cvr_ctx *c) {
  DevState<real> s{};
  s.n = (int)c->n;
  s.n_pad = c->n_pad;
  s.cap = c->cap;
  s.tpa = c->tpa;
  // all_atom_test: wrap and reclassify every step (the reference regenerates
  // its ghosts every step and its list covers all of them)
  s.policy = c->all_atom ? CVR_REBUILD_EVERY_STEP : c->policy;
  s.n_types = c->n_types;
  for (int d = 0; d < 3; ++d) {
    s.box.lo[d] = c->lo[d];
    s.box.hi[d] = c->hi[d];
    s.box.L[d] = c->L[d];
    s.box.gclo[d] = c->lo[d] + c->gc;  // x_llow = lower_global.x + ghost_cutoff
    s.box.gchi[d] = c->hi[d] - c->gc;  // x_lupp = upper_global.x - ghost_cutoff
    s.box.bc[d] = c->bc[d];
    s.box.ctr[d] = c->lo[d] + 0.5 * c->L[d];
    s.box.Lf[d] = (float)c->L[d];
    s.cells.nc[d] = c->nc[d];
    s.cells.w[d] = c->w[d];
    s.cells.inv_w[d] = 1.0 / c->w[d];
  }
  s.cells.ncells = c->ncells;
  s.cells.R = c->R;
  s.cells.S = 2 * c->R + 1;
  const double rl = c->cutoff * c->coef;  // cutoff_extra = cutoff * cutoff_extra_coef
  s.rl_sq = rl * rl;
  // Guard band of the FP32 prefilter: each box-centred FP32 coordinate is off
  // by at most 2^-24 (|L|/2 + rl) after rounding, a difference by twice that,
  // so |d|^2 is off by at most 2 rl sqrt(3) (2 eps); the band is 16x that
  // bound (and never below 1e-5 relative).
  double half = 0;
  for (int d = 0; d < 3; ++d) half = std::max(half, 0.5 * c->L[d] + rl);
  const double eps_coord = 2.0 * std::ldexp(half, -24);
  const double band = std::max(1e-5, 16.0 * 2.0 * rl * std::sqrt(3.0) * eps_coord / (rl * rl));
  s.rl_sq_lo = (float)(s.rl_sq * (1.0 - band));
  s.rl_sq_hi = (float)(s.rl_sq * (1.0 + band));
  s.regular_images = 1;
  for (int d = 0; d < 3; ++d)
    if (c->bc[d] == 1 && !(c->gc >= rl && c->gc <= 0.5 * c->L[d])) s.regular_images = 0;
  const double half_skin = 0.5 * (rl - c->cutoff);  // threshold_distance_sq = 0.25 (rl - rc)^2
  s.thr_sq = (float)(half_skin * half_skin);
  s.fixed = c->fixed;
  s.fx_scale = c->fixed ? std::ldexp(1.0, 32) / c->L[0] : 0.0;
  s.x = c->x;
  s.y = c->y;
  s.z = c->z;
  s.vx = c->vx;
  s.vy = c->vy;
  s.vz = c->vz;
  s.ax = (real *)c->ax;
  s.ay = (real *)c->ay;
  s.az = (real *)c->az;
  s.x4 = (typename V4<real>::t *)c->x4;
  s.xb = c->xb;
  s.cell = c->cell;
  s.id = c->id;
  s.type = c->type;
  s.mol = c->mol;
  s.gcls = c->gcls;
  s.tx = c->tx;
  s.ty = c->ty;
  s.tz = c->tz;
  s.tvx = c->tvx;
  s.tvy = c->tvy;
  s.tvz = c->tvz;
  s.tid = c->tid;
  s.ttype = c->ttype;
  s.tmol = c->tmol;
  s.tcell = c->tcell;
  s.cell_count = c->cell_count;
  s.cell_start = c->cell_start;
  s.cell_fill = c->cell_fill;
  s.slot_atom = c->slot_atom;
  s.perm = c->perm;
  s.block_sums = c->block_sums;
  s.nlist = c->nlist;
  s.ncount = c->ncount;
  s.flag = c->flags;
  s.err = c->flags + 1;
  s.max_count = c->flags + 2;
  s.n_builds = c->flags + 3;
  s.build_epoch = c->flags + 4;
  s.clamp_mark = c->flags + 5;
  s.mass_inv = c->d_mass_inv;
  s.mass = c->d_mass;
  return s;
}

// Event-bracketed launches for cvr_kernel_time.
struct Bracket {
  cvr_ctx *c;
  int kind;
  cudaEvent_t stop = nullptr;
  Bracket(cvr_ctx *c_, int kind_) : c(c_), kind(kind_) {
    if (!c->timing) return;
    KT &k = c->kt[kind];
    if (k.used == k.ev.size()) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      k.ev.emplace_back(a, b);
    }
    cudaEventRecord(k.ev[k.used].first, c->stream);
    stop = k.ev[k.used].second;
    k.used++;
    k.launches++;
  }
  ~Bracket() {
    if (stop) cudaEventRecord(stop, c->stream);
  }
};

void collect_timing(cvr_ctx *c) {
  if (!c->timing) return;
  cudaStreamSynchronize(c->stream);
  for (auto &k : c->kt) {
    for (size_t u = 0; u < k.used; ++u) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, k.ev[u].first, k.ev[u].second) == cudaSuccess) k.ms += ms;
    }
    k.used = 0;
  }
}

// -------------------------------------------------------------- geometry
int setup_cells(cvr_ctx *c) {
  const double rl = c->cutoff * c->coef;
  if (!(rl > 0)) return fail(c, CVR_ERR_INVALID, "neighbour list cutoff must be positive");
  int64_t nct = 1;
  for (int d = 0; d < 3; ++d) {
    // cells at least rl/R wide (with a relative margin), so pairs within rl are <= R cells apart
    int k = (int)std::floor(c->L[d] * c->R / (rl * (1.0 + 1e-10)));
    k = std::max(1, std::min(k, 1024));
    c->nc[d] = k;
    c->w[d] = c->L[d] / k;
    nct *= k;
  }
  if (nct > (int64_t)1 << 26) return fail(c, CVR_ERR_GEOMETRY, "too many cells");
  c->ncells = (int)nct;
  return CVR_OK;
}

// Fixed-point pair displacements (mixed form): positions as u = r 2^32 / L
// mod 2^32, the displacement of a listed pair as the wrapping int32
// difference.  Taken when
//  * the box is cubic (one scale for all axes, folded into the coefficients);
//  * every listed pair stays below L/2 apart until the next build: at most
//    rl + 2 (skin/2) = 2 rl - rc, since each atom moves at most skin/2 before
//    the displacement trigger rebuilds the list (so the integer wrap is the
//    image the list entry names; a non-periodic axis never wraps a listed pair);
//  * the fixed-point step L / 2^32 is no coarser than the FP32 spacing of the
//    cell-local coordinates it replaces (|r| < w/2 with w = L / nc: 2^-24 w),
//    i.e. at most 256 cells per axis.
// Otherwise the cell-local FP32 form is used.
void choose_fixed(cvr_ctx *c) {
  c->fixed = 0;
  if (c->precision == CVR_PREC_FP64 || c->all_atom) return;
  const double rl = c->cutoff * c->coef;
  if (!(c->L[0] == c->L[1] && c->L[1] == c->L[2])) return;
  if (!(0.5 * c->L[0] > (2.0 * rl - c->cutoff) * (1.0 + 1e-6))) return;
  for (int d = 0; d < 3; ++d)
    if (c->nc[d] > 256) return;
  c->fixed = 1;
}

int upload_tables(cvr_ctx *c) {
  const int T = c->n_types;
  const bool dbl = c->precision == CVR_PREC_FP64;
  std::vector<PairCoef<double>> cd(T * T);
  for (int a = 0; a < T; ++a)
    for (int b = 0; b < T; ++b) {
      PairCoef<double> &p = cd[a * T + b];
      p = PairCoef<double>{};
      p.lam = 1.0;
      p.rc2 = -1.0;
      if (c->lj_on) {
        const double e = c->eps[a * T + b], s = c->sig[a * T + b];
        const double rc = c->cutl.empty() ? c->lj_cut : c->cutl[a * T + b];
        const double rc2 = rc * rc;
        if (e != 0.0 && rc > 0) {  // lj.cpp:435-436 skips eps = 0
          const double rcinv = 1.0 / rc2;
          const double c2 = s * s * rcinv, c6 = c2 * c2 * c2, c12 = c6 * c6;
          p.sig2 = s * s;
          p.eps24 = 24.0 * e;
          p.eps48 = 48.0 * e;
          p.K = 4.0 * e * (12.0 * c12 * rcinv - 6.0 * c6 * rcinv);
          p.rc2 = rc2;
          const double g = 4.0 * e * (12.0 * c12 - 6.0 * c6);
          p.e4 = 4.0 * e;
          p.C1 = g / (2.0 * rc2);
          p.C0 = -4.0 * e * (c12 - c6) - 0.5 * g;
        }
      }
      if (c->ewr_on) {
        p.qq = c->ewr_ke * c->charge[a] * c->charge[b];
        if (!c->lam.empty()) p.lam = c->lam[a * T + b];
      }
      p.jump2 = (c->lj_on && c->jump_tol > 0) ? c->jump_tol : 0.0;
    }
  if (dbl) {
    if (int r = dalloc(c, (PairCoef<double> **)&c->d_coef, T * T)) return r;
    CVR_CUDA(c, cudaMemcpyAsync(c->d_coef, cd.data(), T * T * sizeof(PairCoef<double>), cudaMemcpyHostToDevice, c->stream));
  } else {
    // fixed-point form: lengths in units of h = L / 2^32 (r2 -> r2 / h^2; the
    // force coefficient c -> c h^2, so c * du summed and times 1/h is the force)
    const double h = c->fixed ? c->L[0] / std::ldexp(1.0, 32) : 1.0, h2 = h * h;
    std::vector<PairCoef<float>> cf(T * T);
    for (int t = 0; t < T * T; ++t) {
      const auto &p = cd[t];
      cf[t] = PairCoef<float>{(float)(p.sig2 / h2), (float)p.eps24, (float)p.eps48, (float)(p.K * h2),
                              (float)(p.rc2 > 0 ? p.rc2 / h2 : p.rc2),
                              (float)(p.qq / h), (float)p.e4, (float)p.C0, (float)(p.C1 * h2), (float)p.lam,
                              (float)(p.jump2 / h2)};
    }
    if (int r = dalloc(c, (PairCoef<float> **)&c->d_coef, T * T)) return r;
    CVR_CUDA(c, cudaMemcpyAsync(c->d_coef, cf.data(), T * T * sizeof(PairCoef<float>), cudaMemcpyHostToDevice, c->stream));
  }
  std::vector<double> mi(T), m(T);
  for (int t = 0; t < T; ++t) {
    m[t] = c->mass[t];
    mi[t] = (c->mass[t] == 0.0) ? 0.0 : 1.0 / c->mass[t];  // atom_data.cpp:582-585
  }
  if (int r = dalloc(c, &c->d_mass_inv, T)) return r;
  if (int r = dalloc(c, &c->d_mass, T)) return r;
  if (int r = dalloc(c, &c->d_charge, T)) return r;
  CVR_CUDA(c, cudaMemcpyAsync(c->d_mass_inv, mi.data(), T * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(c->d_mass, m.data(), T * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(c->d_charge, c->charge.data(), T * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return CVR_OK;
}

// k-vectors of the reference (initialize.cpp:184-222): kx, ky, kz nested over
// [-kmax, kmax], zero skipped, f_k = exp(-k^2/(4 alpha^2)) / k^2; only the
// first (2kx)(2ky)(2kz) are used.
// k-space box length of axis d: the domain's, or slab_lz on the slab axis
double klen(const cvr_ctx *c, int d) { return d == c->slab_axis ? c->slab_lz : c->L[d]; }
double kvolume(const cvr_ctx *c) { return klen(c, 0) * klen(c, 1) * klen(c, 2); }

int setup_kspace(cvr_ctx *c) {
  c->kint.clear();
  c->fk.clear();
  c->kxy.clear();
  c->kpm.clear();
  if (!c->ewk_on) {
    c->nk = 0;
    return CVR_OK;
  }
  const double two_pi = 6.28318530717958647692;
  const double lx_inv = 1.0 / klen(c, 0), ly_inv = 1.0 / klen(c, 1), lz_inv = 1.0 / klen(c, 2);
  const double alpha_sq = c->ewk_alpha * c->ewk_alpha;
  const double four_alpha2_inv = 1.0 / (4.0 * alpha_sq);
  const int64_t used = (int64_t)(2 * c->kmax[0]) * (2 * c->kmax[1]) * (2 * c->kmax[2]);
  for (int a = -c->kmax[0]; a <= c->kmax[0]; ++a)
    for (int b = -c->kmax[1]; b <= c->kmax[1]; ++b)
      for (int q = -c->kmax[2]; q <= c->kmax[2]; ++q) {
        if ((int64_t)c->kint.size() >= used) break;
        const double k0 = two_pi * a * lx_inv, k1 = two_pi * b * ly_inv, k2 = two_pi * q * lz_inv;
        const double ksq = k0 * k0 + k1 * k1 + k2 * k2;
        if (ksq == 0) continue;
        c->kint.push_back(make_int4(a, b, q, 0));
        c->fk.push_back((1.0 / ksq) * std::exp(-ksq * four_alpha2_inv));
      }
  c->nk = (int)c->kint.size();
  // (nx, ny) columns in order of first use; per column and m = 0..kmax_z the
  // k indices of (nx, ny, +m) and (nx, ny, -m) (-1: not in the set)
  c->kxy.clear();
  std::vector<int> col_of(c->nk);
  {
    std::map<std::pair<int, int>, int> col;
    for (int k = 0; k < c->nk; ++k) {
      const int4 v = c->kint[k];
      auto it = col.find({v.x, v.y});
      if (it == col.end()) {
        it = col.emplace(std::make_pair(v.x, v.y), (int)c->kxy.size()).first;
        c->kxy.push_back(make_int2(v.x, v.y));
      }
      col_of[k] = it->second;
    }
  }
  c->nxy = (int)c->kxy.size();
  c->kM = c->kmax[2] + 1;
  c->kpm.assign((size_t)c->kM * c->nxy, make_int2(-1, -1));
  for (int k = 0; k < c->nk; ++k) {
    const int z = c->kint[k].z;
    int2 &e = c->kpm[(size_t)std::abs(z) * c->nxy + col_of[k]];
    (z >= 0 ? e.x : e.y) = k;
  }
  // For real charges S(-nx, -ny, +-m) = conj(S(nx, ny, -+m)) (the phase
  // products of the mirror are the exact conjugates), so of two columns that
  // mirror each other only the first in column order is summed; k_sk_reduce
  // conjugates it for the other.  Columns without their mirror in the
  // (truncated) k-set are summed themselves.
  {
    std::map<std::pair<int, int>, int> col_index;
    for (int q = 0; q < c->nxy; ++q) col_index[{c->kxy[q].x, c->kxy[q].y}] = q;
    c->kxyc.clear();
    c->kmir.clear();
    c->ksrc.assign(c->nxy, 0);
    std::vector<int> comp_of(c->nxy, -1);
    for (int q = 0; q < c->nxy; ++q) {
      const auto it = col_index.find({-c->kxy[q].x, -c->kxy[q].y});
      const int mq = (it == col_index.end()) ? -1 : it->second;
      if (mq >= 0 && mq < q && mq != q) {
        c->ksrc[q] = comp_of[mq] | (1 << 30);  // taken from the earlier mirror
        c->kmir[comp_of[mq]] = q;
      } else {
        comp_of[q] = (int)c->kxyc.size();
        c->ksrc[q] = comp_of[q];
        c->kxyc.push_back(c->kxy[q]);
        c->kmir.push_back(-1);
      }
    }
    c->ncomp = (int)c->kxyc.size();
  }
  c->kp = std::max(c->kmax[0], std::max(c->kmax[1], c->kmax[2])) + 1;
  if (int r = dalloc(c, &c->d_fk, c->nk)) return r;
  if (int r = dalloc(c, &c->d_kxyc, c->ncomp)) return r;
  if (int r = dalloc(c, &c->d_ksrc, c->nxy)) return r;
  if (int r = dalloc(c, &c->d_kmir, c->ncomp)) return r;
  if (int r = dalloc(c, &c->d_kxy, c->nxy)) return r;
  if (int r = dalloc(c, &c->d_kpm, c->kpm.size())) return r;
  if (int r = dalloc(c, &c->d_sk, c->nk)) return r;
  const size_t rb = (c->precision == CVR_PREC_FP64) ? 8 : 4;
  if (int r = dalloc(c, (unsigned char **)&c->d_kcoef, (size_t)c->nxy * c->kM * 8 * rb)) return r;
  CVR_CUDA(c, cudaMemcpyAsync(c->d_fk, c->fk.data(), c->nk * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(c->d_kxy, c->kxy.data(), c->nxy * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(c->d_kxyc, c->kxyc.data(), c->ncomp * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(c->d_ksrc, c->ksrc.data(), c->nxy * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(c->d_kmir, c->kmir.data(), c->ncomp * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(c->d_kpm, c->kpm.data(), c->kpm.size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
  c->n_ek_blocks = grid_for(c->kM * c->nxy, 32);
  if (int r = dalloc(c, &c->ek_part, c->n_ek_blocks)) return r;
  // the tensor-core k-space force holds 2 M <= KTC_K z components and
  // kmax + 1 <= KTC_KPMAX phase rows per axis; its coefficient image is
  // zero wherever k_sk_reduce does not write (padding)
  c->kimg_tiles = 0;
  if (c->precision != CVR_PREC_FP64 && 2 * c->kM <= KTC_K && c->kp <= KTC_KPMAX && c->ncomp <= KTC_MAXCOLS) {
    c->kimg_tiles = grid_for(c->ncomp, KTC_COLS);
    if (int r = dalloc(c, &c->d_kimg, (size_t)c->kimg_tiles * 2 * KTC_TILE_FLOATS)) return r;
  }
  return CVR_OK;
}

// Whether the k-space force runs on the tensor cores (mixed form).
bool kforce_tc(const cvr_ctx *c) {
  return c->precision != CVR_PREC_FP64 && c->kimg_tiles > 0 && c->d_kimg && c->kforce_kind == CVR_KFORCE_AUTO;
}

int alloc_atoms(cvr_ctx *c, int64_t n) {
  const bool dbl = c->precision == CVR_PREC_FP64;
  const size_t rs = dbl ? 8 : 4;
  c->n = n;
  c->n_pad = (int)((n + 31) / 32 * 32);
  int r = 0;
#define A(ptr, cnt) \
  if ((r = dalloc(c, &c->ptr, (cnt)))) return r;
  A(x, n) A(y, n) A(z, n) A(vx, n) A(vy, n) A(vz, n);
  A(tx, n) A(ty, n) A(tz, n) A(tvx, n) A(tvy, n) A(tvz, n);
  A(xb, n) A(cell, n) A(id, n) A(type, n) A(mol, n) A(gcls, n);
  A(tid, n) A(ttype, n) A(tmol, n) A(tcell, n) A(slot_atom, n) A(perm, n);
  A(ncount, n) A(stage, 6 * n) A(stage_i, 2 * n);
#undef A
  if ((r = dalloc(c, (unsigned char **)&c->ax, n * rs))) return r;
  if ((r = dalloc(c, (unsigned char **)&c->ay, n * rs))) return r;
  if ((r = dalloc(c, (unsigned char **)&c->az, n * rs))) return r;
  if ((r = dalloc(c, (unsigned char **)&c->x4, n * 4 * rs))) return r;
  // per-atom arrays that a replay after a list overflow restores
  c->snap_pairs.clear();
  c->snap_bytes.clear();
  auto add = [&](void *p, size_t b) {
    c->snap_pairs.emplace_back(p, nullptr);
    c->snap_bytes.push_back(b);
  };
  add(c->x, n * 8); add(c->y, n * 8); add(c->z, n * 8);
  add(c->vx, n * 8); add(c->vy, n * 8); add(c->vz, n * 8);
  add(c->ax, n * rs); add(c->ay, n * rs); add(c->az, n * rs);
  add(c->x4, n * 4 * rs); add(c->xb, n * 16); add(c->cell, n * 4); add(c->id, n * 4);
  add(c->type, n * 4); add(c->mol, n * 4); add(c->gcls, n);
  // partial-sum buffers
  c->n_ke_blocks = grid_for(n, 256);
  if ((r = dalloc(c, &c->ke_part, (size_t)c->n_ke_blocks * 4))) return r;
  return CVR_OK;
}

int alloc_cells(cvr_ctx *c) {
  int r;
  if ((r = dalloc(c, &c->cell_count, c->ncells + 1))) return r;
  if ((r = dalloc(c, &c->cell_start, c->ncells + 1))) return r;
  if ((r = dalloc(c, &c->cell_fill, c->ncells + 1))) return r;
  if ((r = dalloc(c, &c->block_sums, grid_for(c->ncells, 1024) + 1))) return r;
  return CVR_OK;
}

int alloc_list(cvr_ctx *c, int cap) {
  const int ilv = 1 << c->log2_tpa;
  c->cap = (cap + ilv - 1) / ilv * ilv;
  const size_t entries = (size_t)c->cap * c->n_pad;  // cap is a multiple of the interleave
  int r;
  if ((r = dalloc(c, &c->nlist, entries))) return r;
  c->nlist_bytes = entries * 4;
  const int blocks = grid_for(c->n * c->tpa, 128);
  c->n_ev_blocks = blocks;
  if ((r = dalloc(c, &c->ev_part, (size_t)blocks * 3))) return r;
  return CVR_OK;
}

// ------------------------------------------------------------- launches
// The list search kernel: by default systems up to 65,536 atoms take the
// warp kernel, larger ones one thread per atom (LJ fluid, mixed step: warp
// 34.2 vs thread 38.5 us at 32,000 atoms, 59.5 vs 50.7 us at 108,000).
int list_kernel_kind(const cvr_ctx *c) {
  if (c->list_kernel != CVR_LIST_AUTO) return c->list_kernel;
  return (c->n <= 65536) ? CVR_LIST_WARP : CVR_LIST_THREAD;
}

bool phase_in_drift(const cvr_ctx *c);
template <typename real>
KArgs<real> kargs(cvr_ctx *c);

template <typename real>
void launch_build(cvr_ctx *c, int count_only) {
  Bracket br(c, CVR_KT_BUILD);
  DevState<real> s = dev_state<real>(c);
  const int n = (int)c->n;
  const int nb_scan = grid_for(c->ncells, 1024);
  k_bin_count<real><<<grid_for(n, 256), 256, 0, c->stream>>>(s);
  k_scan_local<<<nb_scan, 1024, 0, c->stream>>>(s.flag, c->cell_count, c->cell_start, c->block_sums, c->ncells);
  k_scan_sums<<<1, 1024, 0, c->stream>>>(s.flag, c->block_sums, nb_scan, c->cell_start + c->ncells, s.build_epoch);
  k_scan_add<<<nb_scan, 1024, 0, c->stream>>>(s.flag, c->cell_start, c->block_sums, c->ncells);
  k_bin_scatter<real><<<grid_for(n, 256), 256, 0, c->stream>>>(s);
  k_rank<real><<<grid_for(n, 256), 256, 0, c->stream>>>(s);
  k_permute<real><<<grid_for(std::max<int64_t>(n, c->ncells), 256), 256, 0, c->stream>>>(s);
  const int kind = list_kernel_kind(c);
  if (kind == CVR_LIST_WARP) {
    k_build_list_warp<real><<<grid_for((int64_t)n * 32, 128), 128, 0, c->stream>>>(s, count_only, c->log2_tpa);
  } else {
    k_build_list<real><<<grid_for(n, 128), 128, 0, c->stream>>>(s, count_only, c->log2_tpa);
  }
  c->launches += 8;
  if (phase_in_drift(c)) {  // the atoms moved in memory: the step's phase tables follow them
    k_phase<real><<<grid_for(3 * (int64_t)c->n, 256), 256, 0, c->stream>>>(s, kargs<real>(c), s.flag);
    c->launches++;
  }
}

template <typename real, int TPA, bool LJ, bool EWR, bool EV, bool ONE_TYPE, bool FIXED>
void launch_pair_t(cvr_ctx *c, int book) {
  DevState<real> s = dev_state<real>(c);
  // fixed-point form: lengths in units of h = L / 2^32 (see upload_tables)
  const double h = FIXED ? c->L[0] / std::ldexp(1.0, 32) : 1.0;
  EwrArgs<real> ew;
  ew.alpha = (real)(c->ewr_alpha * h);
  ew.alpha2 = (real)(c->ewr_alpha * c->ewr_alpha * h * h);
  ew.two_alpha_spi = (real)(2.0 * c->ewr_alpha * 0.56418958354775628695 * h);  // 2 alpha / sqrt(pi)
  ew.cut2 = (real)(c->ewr_cut >= 0 ? c->ewr_cut * c->ewr_cut / (h * h) : -1.0);
  const int blocks = grid_for(c->n * TPA, 128);
  k_pair<real, TPA, LJ, EWR, EV, ONE_TYPE, FIXED><<<blocks, 128, 0, c->stream>>>(
      s, (const PairCoef<real> *)c->d_coef, (real)(1.0 / h), ew, c->ignore_intra, c->use_mol ? 1 : 0, c->ev_part,
      book, c->counters);
  c->launches++;
}

template <typename real, bool LJ, bool EWR, bool EV, bool FIXED>
void launch_pair_tpa_f(cvr_ctx *c, int book) {
  // one type pair, no molecule tests, no jump_tol clamp: LJ constants in registers
  const bool one = LJ && !EWR && c->n_types == 1 && !c->use_mol && !(c->jump_tol > 0);
  switch (c->tpa) {
    case 1:
      one ? launch_pair_t<real, 1, LJ, EWR, EV, true, FIXED>(c, book) : launch_pair_t<real, 1, LJ, EWR, EV, false, FIXED>(c, book);
      break;
    case 8:
      one ? launch_pair_t<real, 8, LJ, EWR, EV, true, FIXED>(c, book) : launch_pair_t<real, 8, LJ, EWR, EV, false, FIXED>(c, book);
      break;
    default:
      one ? launch_pair_t<real, 32, LJ, EWR, EV, true, FIXED>(c, book)
          : launch_pair_t<real, 32, LJ, EWR, EV, false, FIXED>(c, book);
      break;
  }
}

template <typename real, bool LJ, bool EWR, bool EV>
void launch_pair_tpa(cvr_ctx *c, int book) {
  if constexpr (sizeof(real) == 4) {
    if (c->fixed) return launch_pair_tpa_f<real, LJ, EWR, EV, true>(c, book);
  }
  launch_pair_tpa_f<real, LJ, EWR, EV, false>(c, book);
}

// all_atom_test: every owned pair and every ghost image (k_pair_all), in
// length units (the fixed-point form is off in this mode).
template <typename real, bool LJ, bool EWR, bool EV>
void launch_pair_all_t(cvr_ctx *c) {
  DevState<real> s = dev_state<real>(c);
  EwrArgs<real> ew;
  ew.alpha = (real)c->ewr_alpha;
  ew.alpha2 = (real)(c->ewr_alpha * c->ewr_alpha);
  ew.two_alpha_spi = (real)(2.0 * c->ewr_alpha * 0.56418958354775628695);
  ew.cut2 = (real)(c->ewr_cut >= 0 ? c->ewr_cut * c->ewr_cut : -1.0);
  // n_ev_blocks >= the blocks that hold atoms; the rest store zero partials
  k_pair_all<real, LJ, EWR, EV><<<c->n_ev_blocks, 128, 0, c->stream>>>(
      s, (const PairCoef<real> *)c->d_coef, ew, c->ignore_intra, c->use_mol ? 1 : 0, c->ev_part);
  c->launches++;
}

template <typename real, bool EV>
void launch_pair_all(cvr_ctx *c) {
  if (c->lj_on && c->ewr_on)
    launch_pair_all_t<real, true, true, EV>(c);
  else if (c->lj_on)
    launch_pair_all_t<real, true, false, EV>(c);
  else
    launch_pair_all_t<real, false, true, EV>(c);
}

// book: the pair kernel takes over the end-of-step bookkeeping of a step
// whose kick is deferred (only where defer_kick allows it).
template <typename real>
void launch_pair(cvr_ctx *c, bool ev, bool book = false) {
  Bracket br(c, CVR_KT_PAIR);
  const int b = book ? 1 : 0;
  if (c->all_atom && (c->lj_on || c->ewr_on)) {
    ev ? launch_pair_all<real, true>(c) : launch_pair_all<real, false>(c);
  } else if (c->lj_on && c->ewr_on) {
    ev ? launch_pair_tpa<real, true, true, true>(c, b) : launch_pair_tpa<real, true, true, false>(c, b);
  } else if (c->lj_on) {
    ev ? launch_pair_tpa<real, true, false, true>(c, b) : launch_pair_tpa<real, true, false, false>(c, b);
  } else if (c->ewr_on) {
    ev ? launch_pair_tpa<real, false, true, true>(c, b) : launch_pair_tpa<real, false, true, false>(c, b);
  } else {
    // no pair force field: accelerations start from zero
    const size_t rs = sizeof(real);
    cudaMemsetAsync(c->ax, 0, c->n * rs, c->stream);
    cudaMemsetAsync(c->ay, 0, c->n * rs, c->stream);
    cudaMemsetAsync(c->az, 0, c->n * rs, c->stream);
    if (ev) cudaMemsetAsync(c->ev_part, 0, (size_t)c->n_ev_blocks * 3 * sizeof(double), c->stream);
  }
}

template <typename real>
KArgs<real> kargs(cvr_ctx *c) {
  KArgs<real> a{};
  a.nk = c->nk;
  a.nxy = c->nxy;
  a.xyc = c->d_kxyc;
  a.ksrc = c->d_ksrc;
  a.ncomp = c->ncomp;
  a.kmir = c->d_kmir;
  a.M = c->kM;
  for (int d = 0; d < 3; ++d) {
    a.kmax[d] = c->kmax[d];
    a.inv_L[d] = 1.0 / klen(c, d);
    a.two_pi_over_L[d] = (real)(6.28318530717958647692 / klen(c, d));
  }
  a.kp = c->kp;
  a.xy = c->d_kxy;
  a.kpm = c->d_kpm;
  a.fk = c->d_fk;
  a.ptab = (typename R2<real>::t *)c->d_ptab;
  a.partial = c->d_kpartial;
  a.sk = c->d_sk;
  a.kcoef = (real *)c->d_kcoef;
  a.e_partials = c->ek_part;
  a.four_pi_over_v = 12.56637061435917295384 / kvolume(c);
  a.charge = c->d_charge;
  a.k_e = c->ewk_ke;
  a.nchunks = c->nchunks;
  a.kimg = (sizeof(real) == 4 && kforce_tc(c)) ? c->d_kimg : nullptr;
  return a;
}

// dynamic shared memory of the S(k) kernel (a chunk's phase tables and
// charges) and of the k-force kernel (the warps' coefficient tiles and
// column indices, 32 atoms' phase tables, the warps' partial forces)
template <typename real>
size_t sk_smem(const cvr_ctx *c) {
  const int rw = 2 * c->kp + ((c->kM + KMG - 1) / KMG) * KMG;
  return (size_t)KCH * rw * sizeof(typename R2<real>::t) + KCH * sizeof(real);
}
template <typename real>
size_t kf_smem(const cvr_ctx *c) {
  const size_t tiles = (size_t)c->kf_warps * c->kf_tc;
  return tiles * c->kM * 8 * sizeof(real) + ((tiles + 1) & ~(size_t)1) * sizeof(int2) +
         (size_t)32 * 3 * c->kp * sizeof(typename R2<real>::t) + (size_t)c->kf_warps * 96 * sizeof(real);
}

// k-force kernel instance for the context's m-count: Z in registers for
// M = 1..KMZ (one instance per M), else from shared memory.
template <typename real, int MZ>
struct KForceTable {
  static void launch(cvr_ctx *c, const DevState<real> &s, const KArgs<real> &a, double kick_h) {
    if (c->kM == MZ)
      k_kforce<real, MZ><<<grid_for(c->n, 32), dim3(32, c->kf_warps), kf_smem<real>(c), c->stream>>>(
          s, a, c->kf_tc, kick_h, c->counters);
    else
      KForceTable<real, MZ - 1>::launch(c, s, a, kick_h);
  }
  static void attrs(cvr_ctx *c) {
    cudaFuncSetAttribute(k_kforce<real, MZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)std::max<size_t>(kf_smem<real>(c), 48 * 1024));
    KForceTable<real, MZ - 1>::attrs(c);
  }
};
template <typename real>
struct KForceTable<real, 0> {
  static void launch(cvr_ctx *c, const DevState<real> &s, const KArgs<real> &a, double kick_h) {
    k_kforce<real, 0><<<grid_for(c->n, 32), dim3(32, c->kf_warps), kf_smem<real>(c), c->stream>>>(
        s, a, c->kf_tc, kick_h, c->counters);
  }
  static void attrs(cvr_ctx *c) {
    cudaFuncSetAttribute(k_kforce<real, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)std::max<size_t>(kf_smem<real>(c), 48 * 1024));
  }
};
// kick_h != 0: with the step's second half kick (v += kick_h a) fused.
template <typename real>
void launch_kforce(cvr_ctx *c, const DevState<real> &s, const KArgs<real> &a, double kick_h = 0.0) {
  if constexpr (sizeof(real) == 4) {
    if (a.kimg) {
      // two blocks (a cluster) per 128 atoms
      k_kforce_tc<<<2 * grid_for(c->n, KTC_ATOMS), KTC_THREADS, KTC_SMEM, c->stream>>>(s, a, c->kimg_tiles, kick_h,
                                                                                      c->counters);
      return;
    }
  }
  KForceTable<real, KMZ>::launch(c, s, a, kick_h);
}

// S(k) of the current positions: phase tables (unless the position update
// already wrote them), chunk partials, reduction (S(k), energy partials,
// force coefficients), on stream st.
template <typename real>
void launch_sk(cvr_ctx *c, cudaStream_t st, bool tables_fresh = false) {
  DevState<real> s = dev_state<real>(c);
  KArgs<real> a = kargs<real>(c);
  if (!tables_fresh) {
    k_phase<real><<<grid_for(3 * (int64_t)c->n, 256), 256, 0, st>>>(s, a, nullptr);
    c->launches++;
  }
  dim3 g1(grid_for(((c->kM + KMG - 1) / KMG) * c->ncomp, 128), c->nchunks);
  k_sk_partial<real, KMG, KCH><<<g1, 128, sk_smem<real>(c), st>>>(s, a);
  k_sk_reduce<real, KRW><<<c->n_ek_blocks, KRW * 32, 0, st>>>(s, a);
  c->launches += 2;
}

// Whether the velocity-Verlet position update writes the S(k) phase tables
// (k space on): then every list build rewrites them after reordering atoms,
// and a step's S(k) chain starts at the chunk partials.
bool phase_in_drift(const cvr_ctx *c) { return c->ewk_on && c->nk > 0 && c->integrator == 0 && c->d_ptab; }

// Whether a plain (no thermo record) velocity-Verlet step fuses its second
// half kick into the k-space force kernel: nothing else may touch the
// accelerations or velocities after that kernel (slab correction, dipole
// term, thermostat), and per-kernel timing keeps the kick separate.
bool kick_in_kforce(const cvr_ctx *c, bool th) {
  return !th && c->ewk_on && c->nk > 0 && c->integrator == 0 && !c->tstat.kind && !c->sc_on &&
         !c->dipole_mode && !c->timing;
}

// Whether a plain velocity-Verlet step inside a run may defer its second
// half kick to the next step's k_kick_drift (which applies it first, with
// the same acceleration: the same operations, one pass over v and a less):
// the pair kernel is the step's only force and takes over the kick's flag
// reset and step count; the run's last step and every step with a thermo
// record keep their kick.
bool defer_kick(const cvr_ctx *c) {
  return !(c->ewk_on && c->nk > 0) && (c->lj_on || c->ewr_on) && !c->all_atom && c->integrator == 0 &&
         !c->tstat.kind && !c->sc_on && !(c->ewk_on && c->dipole_mode) && !c->timing;
}

template <typename real>
int launch_kspace(cvr_ctx *c) {
  if (!c->ewk_on || c->nk == 0) return CVR_OK;
  Bracket br(c, CVR_KT_KSPACE);
  launch_sk<real>(c, c->stream);
  DevState<real> s = dev_state<real>(c);
  KArgs<real> a = kargs<real>(c);
  launch_kforce<real>(c, s, a);
  c->launches += 1;
  return CVR_OK;
}

template <typename real>
void set_smem_attrs(cvr_ctx *c) {
  if (sizeof(real) == 4) cudaFuncSetAttribute(k_kforce_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, KTC_SMEM);
  cudaFuncSetAttribute(k_sk_partial<real, KMG, KCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)std::max<size_t>(sk_smem<real>(c), 48 * 1024));
  KForceTable<real, KMZ>::attrs(c);
}

template <typename real>
void launch_thermo(cvr_ctx *c, double *out) {
  ThermoArgs t{};
  t.ke_part = c->ke_part;
  t.n_ke = c->n_ke_blocks;
  t.ev_part = c->ev_part;
  t.n_ev = c->n_ev_blocks;
  t.ek_part = c->ek_part;
  t.n_ek = (c->ewk_on && c->nk > 0) ? c->n_ek_blocks : 0;
  t.volume = c->L[0] * c->L[1] * c->L[2];
  t.k_b = c->k_b;
  t.n_atoms = (double)c->n;
  t.ek_coef = 2.0 * 3.14159265358979323846 * c->ewk_ke / kvolume(c);  // (2 pi / V) k_e sum f_k |S_k|^2
  if (c->sc_on && c->d_sc_state) t.slab_e = c->d_sc_state + 1;
  if (c->ewk_on && c->dipole_mode && c->d_dipole) {
    t.dipole = c->d_dipole;
    t.dipole_coef = c->ewk_ke * 12.56637061435917295384 / kvolume(c) / (1.0 + 2.0 * c->eps_dipole);
  }
  t.e_self = c->e_self;
  const int bcsum = c->bc[0] + c->bc[1] + c->bc[2];
  const int n_r_df = (bcsum == 0) ? 6 : (bcsum == 3 ? 3 : 6 - bcsum);  // atom_data.cpp:322-349
  t.com_removed = (n_r_df >= 1 && n_r_df <= 3) ? 1 : 0;
  t.dof = 3.0 * (double)c->n - n_r_df;
  t.total_mass = c->total_mass;
  t.n_builds = c->flags + 3;
  t.counters = c->counters;
  t.out = out;
  k_thermo<<<1, THERMO_THREADS, 0, c->stream>>>(t);
  c->launches++;
}

template <typename real>
int do_build(cvr_ctx *c, bool force) {
  DevState<real> s = dev_state<real>(c);
  if (force) {
    const int one = 1;
    CVR_CUDA(c, cudaMemcpyAsync(c->flags, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  }
  if (c->cap == 0) {
    // size the list: count pass, then allocate
    CVR_CUDA(c, cudaMemsetAsync(c->flags + 2, 0, sizeof(int), c->stream));
    launch_build<real>(c, 1);
    int mc = 0;
    CVR_CUDA(c, cudaMemcpyAsync(&mc, c->flags + 2, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CVR_CUDA(c, cudaStreamSynchronize(c->stream));
    if (int r = alloc_list(c, std::max(8, (int)std::ceil(mc * 1.3) + 8))) return r;
    const int one = 1;
    CVR_CUDA(c, cudaMemcpyAsync(c->flags, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  }
  CVR_CUDA(c, cudaMemsetAsync(c->flags + 2, 0, sizeof(int), c->stream));
  launch_build<real>(c, 0);
  return CVR_OK;
}

int read_flags(cvr_ctx *c, int out[4]) {
  CVR_CUDA(c, cudaMemcpyAsync(out, c->flags, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaStreamSynchronize(c->stream));
  return CVR_OK;
}

SlabArgs slab_args(cvr_ctx *c) {
  SlabArgs a{};
  a.axis = c->sc_axis;
  a.kx = c->sc_kx;
  a.ky = c->sc_ky;
  a.nv = 4 * c->sc_kx + 4 * c->sc_ky + 8 * c->sc_kx * c->sc_ky + 1;
  a.nch = grid_for(c->n, SLAB_CH);
  // initialize.cpp:33-76: in-plane lengths, slab_sum_e_coef, dipole coefficient
  const int lxa = c->sc_axis == 0 ? 1 : (c->sc_axis == 1 ? 0 : 0);
  const int lya = c->sc_axis == 0 ? 2 : (c->sc_axis == 1 ? 2 : 1);
  a.lx = c->L[lxa];
  a.ly = c->L[lya];
  a.lz = c->sc_lz;
  a.ke = c->sc_ke;
  const double four_pi = 12.56637061435917295384, two_pi = 6.28318530717958647692;
  a.sum_e_coef = -four_pi / (a.lx * a.ly);
  a.dipole_coef = c->sc_ke * four_pi / (a.lx * a.ly * a.lz);
  // make_slab_k_vectors (initialize.cpp:96-143)
  for (int i = 0; i < a.kx; ++i) {
    a.kxv[i] = two_pi * (i + 1) / a.lx;
    a.kxc[i] = 1.0 / (a.kxv[i] * (std::exp(a.kxv[i] * a.lz) - 1.0));
  }
  for (int j = 0; j < a.ky; ++j) {
    a.kyv[j] = two_pi * (j + 1) / a.ly;
    a.kyc[j] = 1.0 / (a.kyv[j] * (std::exp(a.kyv[j] * a.lz) - 1.0));
  }
  for (int i = 0; i < a.kx; ++i)
    for (int j = 0; j < a.ky; ++j) {
      const double kp = std::sqrt(a.kxv[i] * a.kxv[i] + a.kyv[j] * a.kyv[j]);
      a.kpv[i * a.ky + j] = kp;
      a.kpc[i * a.ky + j] = 1.0 / (kp * (std::exp(kp * a.lz) - 1.0));
    }
  a.charge = c->d_charge;
  a.partial = c->d_sc_partial;
  a.chi = c->d_sc_chi;
  a.state = c->d_sc_state;
  return a;
}

template <typename real>
int launch_slab(cvr_ctx *c) {
  SlabArgs a = slab_args(c);
  if (!c->d_sc_partial || c->sc_parts < a.nch * a.nv) {
    if (int r = dalloc(c, &c->d_sc_partial, (size_t)a.nch * a.nv)) return r;
    if (int r = dalloc(c, &c->d_sc_chi, (size_t)a.nv)) return r;
    c->sc_parts = a.nch * a.nv;
    a = slab_args(c);
  }
  DevState<real> s = dev_state<real>(c);
  k_slab_chi_partial<real><<<a.nch, 128, 0, c->stream>>>(s, a);
  k_slab_chi_reduce<<<1, 256, 0, c->stream>>>(a);
  k_slab_field<real><<<grid_for(c->n, 128), 128, 0, c->stream>>>(s, a);
  k_slab_store_moment<<<1, 1, 0, c->stream>>>(a);
  c->launches += 4;
  return CVR_OK;
}

template <typename real>
int forces_now(cvr_ctx *c, bool ev, bool tables_fresh = false, double kick_h = 0.0, bool book = false) {
  if (c->ewk_on && c->nk > 0 && !c->timing) {
    // The S(k) chain reads only positions and charges and the pair kernel
    // writes only the accelerations and its energy partials, so the chain
    // runs on the side stream beside the pair kernel (parallel branches in
    // a captured step graph); the k-space force, which adds to the pair
    // kernel's accelerations, waits for both.  With kernel timing on, the
    // kernels run one after the other so that each class keeps its own
    // event bracket.
    CVR_CUDA(c, cudaEventRecord(c->k_fork, c->stream));
    CVR_CUDA(c, cudaStreamWaitEvent(c->kstream, c->k_fork, 0));
    launch_sk<real>(c, c->kstream, tables_fresh);
    CVR_CUDA(c, cudaEventRecord(c->k_join, c->kstream));
    launch_pair<real>(c, ev);
    CVR_CUDA(c, cudaStreamWaitEvent(c->stream, c->k_join, 0));
    DevState<real> s = dev_state<real>(c);
    KArgs<real> a = kargs<real>(c);
    launch_kforce<real>(c, s, a, kick_h);
    c->launches += 1;
  } else {
    // book is set only where defer_kick allows it (no k space)
    launch_pair<real>(c, ev, book);
    if (int r = launch_kspace<real>(c)) return r;
  }
  if (c->sc_on)
    if (int r = launch_slab<real>(c)) return r;
  if (c->ewk_on && c->dipole_mode) {
    const int nb = grid_for(c->n, 256);
    if (!c->d_dipole) {
      if (int r = dalloc(c, &c->d_dipole, 6)) return r;
    }
    if (!c->d_dip_part || c->dip_parts < nb) {
      if (int r = dalloc(c, &c->d_dip_part, (size_t)nb * 3)) return r;
      c->dip_parts = nb;
    }
    DevState<real> s = dev_state<real>(c);
    const double coef = c->ewk_ke * 12.56637061435917295384 / kvolume(c) / (1.0 + 2.0 * c->eps_dipole);
    k_dipole_partial<real><<<nb, 256, 0, c->stream>>>(s, c->d_charge, c->d_dip_part);
    k_dipole_field<<<1, 256, 0, c->stream>>>(c->d_dip_part, nb, coef, c->d_dipole);
    const double mult = c->dipole_mode == CVR_DIPOLE_ONCE ? 1.0 : (double)c->nk;
    k_dipole_apply<real><<<nb, 256, 0, c->stream>>>(s, c->d_charge, c->d_dipole, mult);
    c->launches += 3;
  }
  return CVR_OK;
}

int regrow(cvr_ctx *c);

// List build and first forces before a run.  A state denser than the one the
// list was sized for (a new state on a kept context) overflows it: the list
// grows from the largest count seen and the build is redone.
template <typename real>
int setup_run(cvr_ctx *c) {
  for (int attempt = 0; attempt < 4; ++attempt) {
    if (int r = do_build<real>(c, true)) return r;
    CVR_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(int), c->stream));
    if (int r = forces_now<real>(c, false)) return r;
    int f[4];
    if (int r = read_flags(c, f)) return r;
    if (f[1] & ERR_OVERFLOW) {
      if (int r = regrow(c)) return r;
      continue;
    }
    if (f[1] & ERR_KSPACE_TC) return fail(c, CVR_ERR_CUDA, "tensor-core k-space force: a wait ran out");
    c->list_valid = true;
    c->setup_done = true;
    return CVR_OK;
  }
  return fail(c, CVR_ERR_CAPACITY, "neighbour list overflow at setup");
}

// Grow the list after an overflow: capacity from the largest count seen.
int regrow(cvr_ctx *c) {
  int f[4];
  if (int r = read_flags(c, f)) return r;
  const int want = std::max(c->cap * 5 / 4, (int)std::ceil(f[2] * 1.3) + 8);
  if (int r = alloc_list(c, want)) return r;
  const int zero = 0;
  CVR_CUDA(c, cudaMemcpyAsync(c->flags + 1, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  return CVR_OK;
}

int snapshot(cvr_ctx *c, bool restore) {
  for (size_t k = 0; k < c->snap_pairs.size(); ++k) {
    auto &p = c->snap_pairs[k];
    if (!p.second) {
      void *q = nullptr;
      cudaError_t e = cudaMalloc(&q, c->snap_bytes[k]);
      if (e != cudaSuccess) return fail(c, CVR_ERR_NOMEM, "snapshot allocation failed");
      c->all_allocs.push_back(q);
      p.second = q;
    }
    if (restore)
      CVR_CUDA(c, cudaMemcpyAsync(p.first, p.second, c->snap_bytes[k], cudaMemcpyDeviceToDevice, c->stream));
    else
      CVR_CUDA(c, cudaMemcpyAsync(p.second, p.first, c->snap_bytes[k], cudaMemcpyDeviceToDevice, c->stream));
  }
  return CVR_OK;
}

// The kernels of one step after the position update: list build (gated by
// the device flag), forces, second kick, optional thermo record.
LangevinArgs langevin_args(cvr_ctx *c) {
  LangevinArgs lg{};
  const double g = c->lgv_friction, dt = c->dt;
  lg.a = (2.0 - g * dt) / (2.0 + g * dt);  // md_simulator.cpp:337-344
  lg.b = c->lgv_kbt > 0 ? std::sqrt(c->lgv_kbt * g * 0.5 * dt) : std::sqrt(c->lgv_kb * c->lgv_temperature * g * 0.5 * dt);
  lg.c = 2.0 * dt / (2.0 + g * dt);
  lg.eta = c->d_eta;
  lg.generate = c->lgv_rng == CVR_RNG_PHILOX ? 1 : 0;
  lg.seed = c->lgv_seed;
  lg.step = c->counters;
  return lg;
}

// deferred: the step's kick is left to the next step's k_kick_drift (only
// where defer_kick allows it, never with a thermo record).
template <typename real>
int launch_step_tail(cvr_ctx *c, bool th, bool deferred = false) {
  DevState<real> s = dev_state<real>(c);
  const bool fused_kick = kick_in_kforce(c, th);
  if (int r = forces_now<real>(c, th, phase_in_drift(c), fused_kick ? 0.5 * c->dt : 0.0, deferred)) return r;
  const int nb = grid_for(c->n, 256);
  if (!fused_kick && !deferred) {
    Bracket br(c, CVR_KT_INTEGRATE);
    if (c->integrator == 1) {
      const LangevinArgs lg = langevin_args(c);
      if (th)
        k_lgv_kick<real, true><<<nb, 256, 0, c->stream>>>(s, c->dt, lg, c->ke_part, c->counters);
      else
        k_lgv_kick<real, false><<<nb, 256, 0, c->stream>>>(s, c->dt, lg, c->ke_part, c->counters);
    } else if (th || c->tstat.kind) {
      k_kick<real, true><<<nb, 256, 0, c->stream>>>(s, c->dt, c->ke_part, c->counters);
    } else {
      k_kick<real, false><<<nb, 256, 0, c->stream>>>(s, c->dt, c->ke_part, c->counters);
    }
    if (c->tstat.kind && c->integrator == 0) {
      ThermostatArgs t = c->tstat;
      const int bcsum = c->bc[0] + c->bc[1] + c->bc[2];
      const int n_r_df = (bcsum == 0) ? 6 : (bcsum == 3 ? 3 : 6 - bcsum);  // atom_data.cpp:322-349
      t.com_removed = (n_r_df >= 1 && n_r_df <= 3) ? 1 : 0;
      t.dof = 3.0 * (double)c->n - n_r_df;
      t.total_mass = c->total_mass;
      t.k_b = c->k_b;
      t.ke_part = c->ke_part;
      t.n_ke = c->n_ke_blocks;
      t.counters = c->counters;
      t.scal = c->d_tscal;
      k_thermostat_coef<<<1, 256, 0, c->stream>>>(t);
      if (th)
        k_thermostat_apply<real, true><<<nb, 256, 0, c->stream>>>(s, t.kind, c->d_tscal, c->ke_part);
      else
        k_thermostat_apply<real, false><<<nb, 256, 0, c->stream>>>(s, t.kind, c->d_tscal, c->ke_part);
      c->launches += 2;
    }
    c->launches++;
  }
  if (th) launch_thermo<real>(c, c->d_thermo);
  return CVR_OK;
}

// pending: the previous step deferred its second half kick to this kernel.
template <typename real>
void launch_kick_drift(cvr_ctx *c, bool pending = false) {
  Bracket br(c, CVR_KT_INTEGRATE);
  const double pre_h = pending ? 0.5 * c->dt : 0.0;
  if (c->integrator == 1)
    k_lgv_kick_drift<real><<<grid_for(c->n, 256), 256, 0, c->stream>>>(dev_state<real>(c), c->dt, langevin_args(c));
  else if (phase_in_drift(c))
    k_kick_drift<real, true><<<grid_for((int64_t)c->n * KD_PHASE_SUB, 256), 256, 0, c->stream>>>(
        dev_state<real>(c), c->dt, kargs<real>(c), pre_h);
  else
    k_kick_drift<real, false>
        <<<grid_for(c->n, 256), 256, 0, c->stream>>>(dev_state<real>(c), c->dt, KArgs<real>{}, pre_h);
  c->launches++;
}

// The reference's noise of one step: for every atom in index order, one
// draw from each of the three streams (md_simulator.cpp:688-698), into a
// pinned buffer, then copied to the device ahead of the step's kernels.
int stage_reference_eta(cvr_ctx *c, int slot) {
  const int64_t n = c->n;
  if (!c->h_eta[slot]) {
    if (cudaMallocHost(&c->h_eta[slot], 3 * (size_t)n * sizeof(double)) != cudaSuccess)
      return fail(c, CVR_ERR_NOMEM, "pinned noise buffer");
    cudaEventCreateWithFlags(&c->eta_done[slot], cudaEventDisableTiming);
  } else {
    CVR_CUDA(c, cudaEventSynchronize(c->eta_done[slot]));  // its previous copy has finished
  }
  double *h = c->h_eta[slot];
  for (int a = 0; a < 3; ++a)
    for (int64_t i = 0; i < n; ++i) h[a * n + i] = c->ndist[a](c->gen[a]);
  CVR_CUDA(c, cudaMemcpyAsync(c->d_eta, h, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaEventRecord(c->eta_done[slot], c->stream));
  return CVR_OK;
}

void destroy_graphs(cvr_ctx *c) {
  for (auto &gh : c->g_step)
    for (auto &g : gh)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  c->graph_epoch = -1;
}

// One CUDA graph per step kind (head: with or without the previous step's
// deferred kick; tail: kick deferred, kick, kick + thermo record):
//   [kick_drift, set condition] -> IF(rebuild flag) {list build} -> [forces, kick, thermo]
// The deferred-kick kinds are made only where defer_kick allows them.
// The build nodes sit in the body of a conditional node whose value a one-thread
// kernel sets from the device flag, so a step without a rebuild launches none
// of them.  Kernel parameters are baked in: the graphs are rebuilt whenever a
// device buffer moves (epoch).
template <typename real>
int build_graphs(cvr_ctx *c) {
  destroy_graphs(c);
  const int64_t launches0 = c->launches;
  const bool dk = defer_kick(c);
  for (int kind = 0; kind < 6; ++kind) {
    const int head = kind / 3, tail = kind % 3;
    if ((head == 1 || tail == 0) && !dk) continue;
    cudaGraph_t g = nullptr, pre = nullptr, post = nullptr, body_out = nullptr;
    CVR_CUDA(c, cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    CVR_CUDA(c, cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    CVR_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    launch_kick_drift<real>(c, head == 1);
    k_set_rebuild_condition<<<1, 1, 0, c->stream>>>(c->flags, h);
    CVR_CUDA(c, cudaStreamEndCapture(c->stream, &pre));
    cudaGraphNode_t n_pre, n_cond, n_post;
    CVR_CUDA(c, cudaGraphAddChildGraphNode(&n_pre, g, nullptr, 0, pre));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    CVR_CUDA(c, cudaGraphAddNode(&n_cond, g, &n_pre, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CVR_CUDA(c, cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_build<real>(c, 0);
    CVR_CUDA(c, cudaStreamEndCapture(c->stream, &body_out));
    CVR_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int r = launch_step_tail<real>(c, tail == 2, tail == 0);
    CVR_CUDA(c, cudaStreamEndCapture(c->stream, &post));
    if (r) return r;
    CVR_CUDA(c, cudaGraphAddChildGraphNode(&n_post, g, &n_cond, 1, post));
    CVR_CUDA(c, cudaGraphInstantiate(&c->g_step[head][tail], g, cudaGraphInstantiateFlagUseNodePriority));
    cudaGraphDestroy(pre);
    cudaGraphDestroy(post);
    cudaGraphDestroy(g);
  }
  // kernels per step outside the conditional body, for the launch count
  const int64_t captured = c->launches - launches0;  // both graphs + 8 build kernels each
  c->launches = launches0;
  c->graph_kernels[0] = 0;
  (void)captured;
  c->graph_epoch = c->epoch;
  return CVR_OK;
}

template <typename real>
int run_impl(cvr_ctx *c, int64_t nsteps, int64_t every, double *thermo) {
  if (!c->setup_done)
    if (int r = setup_run<real>(c)) return r;
  const int64_t nrec = (every > 0) ? nsteps / every : 0;
  if ((size_t)nrec > c->thermo_cap) {
    if (int r = dalloc(c, &c->d_thermo, (size_t)std::max<int64_t>(nrec, 1) * CVR_N_THERMO)) return r;
    c->thermo_cap = (size_t)nrec;
  }
  if (int r = snapshot(c, false)) return r;
  int f0[4];
  if (int r = read_flags(c, f0)) return r;
  const int64_t step0 = c->step;
  std::mt19937 gen0[3];
  std::normal_distribution<double> nd0[3];
  if (c->integrator == 1 && c->tstat.kind)
    return fail(c, CVR_ERR_INVALID, "a thermostat constraint with the Langevin integrator is not supported");
  if (c->integrator == 1) {
    if (!(c->lgv_kbt > 0) && !(c->lgv_kb > 0 && c->lgv_temperature > 0))
      return fail(c, CVR_ERR_INVALID, "expected ('temperature'  & 'kb') or 'kbt' input");
    if (!c->d_eta || c->eta_n != c->n) {
      if (int r = dalloc(c, &c->d_eta, 3 * (size_t)c->n)) return r;
      for (int k = 0; k < 2; ++k)
        if (c->h_eta[k]) {
          cudaEventSynchronize(c->eta_done[k]);
          cudaFreeHost(c->h_eta[k]);
          cudaEventDestroy(c->eta_done[k]);
          c->h_eta[k] = nullptr;
          c->eta_done[k] = nullptr;
        }
      c->eta_n = c->n;
    }
  }
  for (int attempt = 0; attempt < 4; ++attempt) {
    c->counter_src[0] = step0;
    c->counter_src[1] = 0;
    CVR_CUDA(c, cudaMemcpyAsync(c->counters, c->counter_src, sizeof(c->counter_src), cudaMemcpyHostToDevice,
                                c->stream));
    // the reference's noise streams are made on the host step by step: no graphs then
    const bool host_noise = c->integrator == 1 && c->lgv_rng == CVR_RNG_REFERENCE;
    const bool graphs = c->use_graphs && !c->timing && !host_noise;
    if (attempt == 0) {
      for (int a = 0; a < 3; ++a) {
        gen0[a] = c->gen[a];
        nd0[a] = c->ndist[a];
      }
    } else {
      for (int a = 0; a < 3; ++a) {
        c->gen[a] = gen0[a];
        c->ndist[a] = nd0[a];
      }
    }
    const bool dk = defer_kick(c);
    if (graphs && (c->graph_epoch != c->epoch || (dk && !c->g_step[1][0])))
      if (int r = build_graphs<real>(c)) return r;
    const int64_t launches0 = c->launches;
    bool pending = false;  // the previous step deferred its second half kick
    int64_t n_kick = 0;    // steps ending with a plain (no thermo) kick
    for (int64_t k = 0; k < nsteps; ++k) {
      const bool th = every > 0 && ((k + 1) % every == 0);
      const int tail = th ? 2 : ((dk && k + 1 < nsteps) ? 0 : 1);
      n_kick += tail == 1;
      if (graphs) {
        CVR_CUDA(c, cudaGraphLaunch(c->g_step[pending ? 1 : 0][tail], c->stream));
      } else {
        if (host_noise)
          if (int r = stage_reference_eta(c, (int)(k & 1))) return r;
        launch_kick_drift<real>(c, pending);
        launch_build<real>(c, 0);
        if (int r = launch_step_tail<real>(c, th, tail == 0)) return r;
      }
      pending = tail == 0;
    }
    int f[4];
    if (int r = read_flags(c, f)) return r;
    collect_timing(c);
    if (graphs) {
      // kernel nodes executed: per step kick_drift + condition + forces +
      // kick (fused into the k-space force, or deferred to the next step's
      // kick_drift, on plain steps when possible) + thermo record; 8 per
      // rebuild (9 when the build rewrites phase tables)
      const int ks = (c->ewk_on && c->nk > 0) ? (phase_in_drift(c) ? 3 : 4) : 0;
      const int tail = (c->lj_on || c->ewr_on ? 1 : 0) + ks + ((c->tstat.kind && c->integrator == 0) ? 2 : 0) +
                       (c->sc_on ? 4 : 0) + ((c->ewk_on && c->dipole_mode) ? 3 : 0);
      const int kick_plain = kick_in_kforce(c, false) ? 0 : 1;
      c->launches = launches0 + nsteps * (2 + tail) + n_kick * kick_plain + nrec * 2 +
                    (8 + (phase_in_drift(c) ? 1 : 0)) * (int64_t)(f[3] - f0[3]);
    }
    if (f[1] & ERR_NAN) return fail(c, CVR_ERR_NAN, "NaN acceleration");
    if (f[1] & ERR_KSPACE_TC) return fail(c, CVR_ERR_CUDA, "tensor-core k-space force: a wait ran out");
    if (f[1] & ERR_OVERFLOW) {
      // replay the call from the snapshot with a larger list
      if (int r = snapshot(c, true)) return r;
      if (int r = regrow(c)) return r;
      CVR_CUDA(c, cudaMemcpyAsync(c->flags + 3, &f0[3], sizeof(int), cudaMemcpyHostToDevice, c->stream));
      if (int r = do_build<real>(c, true)) return r;
      CVR_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(int), c->stream));
      if (int r = forces_now<real>(c, false)) return r;
      continue;
    }
    c->step = step0 + nsteps;
    if (nrec > 0) {
      if (thermo)
        CVR_CUDA(c, cudaMemcpyAsync(thermo, c->d_thermo, (size_t)nrec * CVR_N_THERMO * sizeof(double),
                                    cudaMemcpyDeviceToHost, c->stream));
      CVR_CUDA(c, cudaMemcpyAsync(c->last_thermo, c->d_thermo + (nrec - 1) * CVR_N_THERMO,
                                  CVR_N_THERMO * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      CVR_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(c, CVR_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return CVR_OK;
  }
  return fail(c, CVR_ERR_CAPACITY, "neighbour list overflow persists after regrowing");
}

template <typename real>
int compute_impl(cvr_ctx *c, double *acc, double *thermo) {
  if (!c->list_valid) {
    if (int r = do_build<real>(c, true)) return r;
    CVR_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(int), c->stream));
    c->list_valid = true;
  }
  if (int r = forces_now<real>(c, true)) return r;
  DevState<real> s = dev_state<real>(c);
  k_ke<real><<<c->n_ke_blocks, 256, 0, c->stream>>>(s, c->ke_part);
  c->launches++;
  if (c->thermo_cap == 0) {
    if (int r = dalloc(c, &c->d_thermo, CVR_N_THERMO)) return r;
    c->thermo_cap = 1;
  }
  c->counter_src[0] = c->step;
  c->counter_src[1] = 0;
  CVR_CUDA(c, cudaMemcpyAsync(c->counters, c->counter_src, sizeof(c->counter_src), cudaMemcpyHostToDevice, c->stream));
  launch_thermo<real>(c, c->d_thermo);
  CVR_CUDA(c, cudaMemcpyAsync(c->last_thermo, c->d_thermo, CVR_N_THERMO * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  if (acc) {
    k_gather_state<real><<<grid_for(c->n, 256), 256, 0, c->stream>>>(s, nullptr, nullptr, c->stage);
    c->launches++;
    CVR_CUDA(c, cudaMemcpyAsync(acc, c->stage, c->n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  int f[4];
  if (int r = read_flags(c, f)) return r;
  collect_timing(c);
  if (f[1] & ERR_OVERFLOW) {
    if (int r = regrow(c)) return r;
    c->list_valid = false;
    return compute_impl<real>(c, acc, thermo);
  }
  if (thermo) std::memcpy(thermo, c->last_thermo, sizeof(c->last_thermo));
  c->setup_done = true;
  return CVR_OK;
}

}  // namespace


// ------------------------------------------------------------------ C ABI
namespace {

int choose_tpa(int64_t n) {
  // enough lanes to fill 148 SMs (about 6e5 threads) without starving lanes
  if (n * 32 <= 600000) return 32;
  if (n * 8 <= 600000) return 8;
  return 1;
}

int ensure_ready(cvr_ctx *c) {
  if (!c->have_state) return fail(c, CVR_ERR_STATE, "cvr_set_state has not been called");
  if (!c->nl_set) return fail(c, CVR_ERR_STATE, "cvr_set_neighborlist has not been called");
  return CVR_OK;
}

// Re-derive everything that depends on the settings (cells, tables, k-set).
// Ewald self energy -(alpha / sqrt(pi)) k_e sum q^2 (electrostatic_ewald_k/energy.cpp:49).
double self_energy(const cvr_ctx *c) {
  return c->ewk_on ? -0.56418958354775628695 * c->ewk_alpha * c->q2_sum * c->ewk_ke : 0.0;
}

int refresh(cvr_ctx *c) {
  if (!c->have_state || !c->nl_set) return CVR_OK;
  c->epoch++;  // settings may change what the step graphs bake in
  c->refreshed = false;
  c->e_self = self_energy(c);
  if (int r = setup_cells(c)) return r;
  if (int r = alloc_cells(c)) return r;
  choose_fixed(c);
  if (int r = upload_tables(c)) return r;
  if (int r = setup_kspace(c)) return r;
  if (c->ewk_on && c->nk > 0) {
    c->nchunks = grid_for(c->n, KCH);
    if (int r = dalloc(c, &c->d_kpartial, (size_t)c->nchunks * c->kM * c->nxy * 2)) return r;
    const size_t c2b = (c->precision == CVR_PREC_FP64) ? 16 : 8;
    if (int r = dalloc(c, (unsigned char **)&c->d_ptab, (size_t)3 * c->kp * c->n * c2b)) return r;
    // k-force launch shape: warps per block of 32 atoms until ~24 warps per
    // SM exist (at most 16, at most one per column)
    const int atom_blocks = grid_for(c->n, 32);
    c->kf_warps = std::max(1, std::min(std::min(KF_WMAX, c->ncomp), (24 * 148 + atom_blocks - 1) / atom_blocks));
    // columns per warp staged in tiles of equal size within KF_COEF_SMEM
    {
      const int per_warp = (c->ncomp + c->kf_warps - 1) / c->kf_warps;
      const int tc_max = std::max<int>(1, (int)(KF_COEF_SMEM / ((size_t)c->kf_warps * c->kM * 8 * (c2b / 2))));
      const int ntiles = (per_warp + tc_max - 1) / tc_max;
      c->kf_tc = (per_warp + ntiles - 1) / ntiles;
    }
    if (c->precision == CVR_PREC_FP64)
      set_smem_attrs<double>(c);
    else
      set_smem_attrs<float>(c);
  }
  c->list_valid = false;
  c->setup_done = false;
  c->refreshed = true;
  return CVR_OK;
}

// all_atom_test: every owned pair (no shift) and every owned atom with every
// ghost image (atom a at shift s = -zone on the axes of a non-empty subset of
// a's ghost zones), in the canonical orientation, from the build's ghost-zone
// classes (the reference's list, neighborlist.cpp:161-191).
int pairs_all_atom(cvr_ctx *c, std::vector<std::array<int32_t, 5>> &out) {
  const int64_t n = c->n;
  // n (n - 1) / 2 owned pairs plus n per ghost image: host memory grows as n^2
  if (n > 4096) return fail(c, CVR_ERR_CAPACITY, "the all_atom_test pair set is exported for at most 4096 atoms");
  std::vector<int> ids(n);
  std::vector<int8_t> g(n);
  CVR_CUDA(c, cudaMemcpyAsync(ids.data(), c->id, n * 4, cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(g.data(), c->gcls, n, cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaStreamSynchronize(c->stream));
  out.clear();
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = i + 1; j < n; ++j)
      out.push_back({std::min(ids[i], ids[j]), std::max(ids[i], ids[j]), 0, 0, 0});
  for (int64_t a = 0; a < n; ++a) {
    const int v[3] = {g[a] % 3 - 1, (g[a] / 3) % 3 - 1, g[a] / 9 - 1};
    for (int m = 1; m < 8; ++m) {
      int sh[3];
      bool ok = true;
      for (int d = 0; d < 3; ++d) {
        const bool on = (m >> d) & 1;
        if (on && v[d] == 0) ok = false;
        sh[d] = on ? -v[d] : 0;
      }
      if (!ok) continue;
      for (int64_t i = 0; i < n; ++i) {
        int p = ids[i], q = ids[a], s3[3] = {sh[0], sh[1], sh[2]};
        bool flip = p > q;
        if (p == q) flip = std::make_tuple(s3[0], s3[1], s3[2]) < std::make_tuple(-s3[0], -s3[1], -s3[2]);
        if (flip) {
          std::swap(p, q);
          for (int d = 0; d < 3; ++d) s3[d] = -s3[d];
        }
        out.push_back({p, q, s3[0], s3[1], s3[2]});
      }
    }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return CVR_OK;
}

template <typename real>
int pairs_impl(cvr_ctx *c, std::vector<std::array<int32_t, 5>> &out) {
  if (c->all_atom) return pairs_all_atom(c, out);
  const int64_t n = c->n;
  std::vector<int> cnt(n), ids(n), cells(n);
  std::vector<uint32_t> lst((size_t)c->cap * c->n_pad);
  CVR_CUDA(c, cudaMemcpyAsync(cnt.data(), c->ncount, n * 4, cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(ids.data(), c->id, n * 4, cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(cells.data(), c->cell, n * 4, cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(lst.data(), c->nlist, lst.size() * 4, cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaStreamSynchronize(c->stream));
  const int tpa = 1 << c->log2_tpa;  // list interleave (quads when one lane per atom)
  const size_t stride = (size_t)c->n_pad * tpa;
  auto fdiv = [](int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); };
  out.clear();
  out.reserve((size_t)n * 40);
  for (int64_t k = 0; k < n; ++k) {
    const int ck = cells[k];
    const int cxyz[3] = {ck % c->nc[0], (ck / c->nc[0]) % c->nc[1], ck / (c->nc[0] * c->nc[1])};
    for (int e = 0; e < cnt[k]; ++e) {
      const uint32_t v = lst[(size_t)(e / tpa) * stride + (size_t)k * tpa + (e % tpa)];
      const int j = (int)(v & INDEX_MASK);
      const int dd[3] = {(int)((v >> CODE_SHIFT) & 7u) - c->R, (int)((v >> (CODE_SHIFT + 3)) & 7u) - c->R,
                         (int)((v >> (CODE_SHIFT + 6)) & 7u) - c->R};
      int sh[3];
      for (int d = 0; d < 3; ++d) sh[d] = fdiv(cxyz[d] + dd[d], c->nc[d]);
      int a = ids[k], b = ids[j];
      bool flip = a > b;
      if (a == b) flip = std::make_tuple(sh[0], sh[1], sh[2]) < std::make_tuple(-sh[0], -sh[1], -sh[2]);
      if (flip) {
        std::swap(a, b);
        for (int d = 0; d < 3; ++d) sh[d] = -sh[d];
      }
      out.push_back({a, b, sh[0], sh[1], sh[2]});
    }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return CVR_OK;
}

}  // namespace

#define DISPATCH(c, fn, ...) ((c)->precision == CVR_PREC_FP64 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

extern "C" {

int cvr_create(cvr_ctx **out, const double lo[3], const double hi[3], const int bc[3], int n_types,
               const double *mass, const double *charge, int device) {
  if (!out) return CVR_ERR_INVALID;
  *out = nullptr;
  if (!lo || !hi || !bc || !mass || n_types <= 0 || n_types > MAX_TYPES) return CVR_ERR_INVALID;
  for (int d = 0; d < 3; ++d)
    if (!(hi[d] > lo[d]) || (bc[d] != 0 && bc[d] != 1)) return CVR_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return CVR_ERR_CUDA;
  cvr_ctx *c = new cvr_ctx();
  for (int a = 0; a < 3; ++a) c->gen[a].seed((unsigned)(a + 1));  // md_simulator.cpp:45-47
  c->device = device;
  for (int d = 0; d < 3; ++d) {
    c->lo[d] = lo[d];
    c->hi[d] = hi[d];
    c->L[d] = hi[d] - lo[d];  // size_global = upper_global - lower_global (domain.cpp:470-477)
    c->bc[d] = bc[d];
  }
  c->n_types = n_types;
  c->mass.assign(mass, mass + n_types);
  c->charge.assign(n_types, 0.0);
  if (charge) c->charge.assign(charge, charge + n_types);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return CVR_ERR_CUDA;
  }
  // the S(k) side stream at the highest priority: its chain (phases, partials,
  // reduction) gates the k-space force, while the pair kernel beside it has
  // slack; step graphs keep the captured priorities (UseNodePriority)
  int prio_least = 0, prio_greatest = 0;
  cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  if (cudaStreamCreateWithPriority(&c->kstream, cudaStreamNonBlocking, prio_greatest) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->k_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->k_join, cudaEventDisableTiming) != cudaSuccess) {
    if (c->kstream) cudaStreamDestroy(c->kstream);
    if (c->k_fork) cudaEventDestroy(c->k_fork);
    cudaStreamDestroy(c->stream);
    delete c;
    return CVR_ERR_CUDA;
  }
  if (dalloc(c, &c->flags, 6) != CVR_OK || dalloc(c, &c->counters, 2) != CVR_OK ||
      dalloc(c, &c->d_type_hist, MAX_TYPES + 1) != CVR_OK) {
    cudaEventDestroy(c->k_fork);
    cudaEventDestroy(c->k_join);
    cudaStreamDestroy(c->kstream);
    cudaStreamDestroy(c->stream);
    delete c;
    return CVR_ERR_NOMEM;
  }
  *out = c;
  return CVR_OK;
}

void cvr_destroy(cvr_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  destroy_graphs(c);
  for (void *p : c->all_allocs) cudaFree(p);
  for (int k = 0; k < 2; ++k) {
    if (c->h_eta[k]) cudaFreeHost(c->h_eta[k]);
    if (c->eta_done[k]) cudaEventDestroy(c->eta_done[k]);
  }
  for (auto &k : c->kt)
    for (auto &e : k.ev) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  cudaStreamSynchronize(c->kstream);
  cudaEventDestroy(c->k_fork);
  cudaEventDestroy(c->k_join);
  cudaStreamDestroy(c->kstream);
  cudaStreamDestroy(c->stream);
  delete c;
}

int cvr_set_neighborlist(cvr_ctx *c, double cutoff, double coef, double ghost_cutoff, int policy) {
  if (!c) return CVR_ERR_INVALID;
  if (!(cutoff > 0)) return fail(c, CVR_ERR_INVALID, "cutoff have to non-negative.");  // neighborlist.cpp:210
  if (!(coef >= 1.0)) return fail(c, CVR_ERR_INVALID, "cutoff_extra_coef must be larger than 1.0");
  if (policy < 0 || policy > 2) return fail(c, CVR_ERR_INVALID, "unknown rebuild policy");
  cudaSetDevice(c->device);
  c->cutoff = cutoff;
  c->coef = coef;
  c->gc = (ghost_cutoff > 0) ? ghost_cutoff : cutoff * coef;
  c->policy = policy;
  c->nl_set = true;
  return refresh(c);
}

int cvr_set_lj(cvr_ctx *c, double cutoff, const double *eps, const double *sig, const double *cutl, int ignore_intra) {
  if (!c || !eps || !sig) return CVR_ERR_INVALID;
  if (cutoff < 0) return fail(c, CVR_ERR_INVALID, "Force field cutoff have to non-negative.");
  const int T = c->n_types;
  for (int t = 0; t < T * T; ++t) {
    if (eps[t] < 0) return fail(c, CVR_ERR_INVALID, "Epsilon have to be non-negative.");
    if (sig[t] < 0) return fail(c, CVR_ERR_INVALID, "Sigma have to be non-negative.");
    if (cutl && cutl[t] < 0) return fail(c, CVR_ERR_INVALID, "cutoff_list have to be non-negative.");
  }
  cudaSetDevice(c->device);
  c->lj_on = true;
  c->lj_cut = cutoff;
  c->eps.assign(eps, eps + T * T);
  c->sig.assign(sig, sig + T * T);
  c->cutl.clear();
  if (cutl) c->cutl.assign(cutl, cutl + T * T);
  c->ignore_intra = ignore_intra ? 1 : 0;
  return refresh(c);
}

int cvr_set_all_atom_test(cvr_ctx *c, int on) {
  if (!c) return CVR_ERR_INVALID;
  if (on && c->n > CVR_ALL_ATOM_MAX) return fail(c, CVR_ERR_INVALID, "all_atom_test is for small systems");
  cudaSetDevice(c->device);
  c->all_atom = on != 0;
  return refresh(c);
}

int cvr_set_lj_jump_tol(cvr_ctx *c, double jump_tol) {
  if (!c) return CVR_ERR_INVALID;
  if (!(jump_tol >= 0)) return fail(c, CVR_ERR_INVALID, "jump_tol have to be non-negative.");
  cudaSetDevice(c->device);
  c->jump_tol = jump_tol;
  return refresh(c);
}

int cvr_set_ewald_r(cvr_ctx *c, double alpha, double ke, const double *lambda, double cutoff) {
  if (!c) return CVR_ERR_INVALID;
  if (alpha < 0) return fail(c, CVR_ERR_INVALID, "alpha have to non-negative.");
  if (ke < 0) return fail(c, CVR_ERR_INVALID, "k_electrostatic has to be non-negative.");
  cudaSetDevice(c->device);
  c->ewr_on = true;
  c->ewr_alpha = alpha;
  c->ewr_ke = ke;
  c->ewr_cut = cutoff;
  c->lam.clear();
  if (lambda) c->lam.assign(lambda, lambda + c->n_types * c->n_types);
  return refresh(c);
}

int cvr_set_ewald_k(cvr_ctx *c, double alpha, int kx, int ky, int kz, double ke) {
  if (!c) return CVR_ERR_INVALID;
  if (alpha < 0) return fail(c, CVR_ERR_INVALID, "alpha have to non-negative.");
  if (kx < 0 || ky < 0 || kz < 0) return fail(c, CVR_ERR_INVALID, "'k_max' have to non-negative.");
  if (kx >= MAX_KMAX || ky >= MAX_KMAX || kz >= MAX_KMAX) return fail(c, CVR_ERR_INVALID, "k_max above 30 is not supported");
  if (ke < 0) return fail(c, CVR_ERR_INVALID, "'k_electrostatic' has to be non-negative.");
  cudaSetDevice(c->device);
  c->ewk_on = true;
  c->ewk_alpha = alpha;
  c->kmax[0] = kx;
  c->kmax[1] = ky;
  c->kmax[2] = kz;
  c->ewk_ke = ke;
  return refresh(c);
}

int cvr_set_ewald_k_geometry(cvr_ctx *c, int slab_axis, double slab_lz, int dipole_mode, double epsilon_dipole) {
  if (!c) return CVR_ERR_INVALID;
  if (slab_axis < -1 || slab_axis > 2) return fail(c, CVR_ERR_INVALID, "expected 'x' or 'y' or 'z' for axis.");
  if (slab_axis >= 0 && !(slab_lz > 0)) return fail(c, CVR_ERR_INVALID, "slab_lz have to non-negative.");
  if (dipole_mode != 0 && dipole_mode != CVR_DIPOLE_REFERENCE && dipole_mode != CVR_DIPOLE_ONCE)
    return fail(c, CVR_ERR_INVALID, "unknown dipole mode");
  if (dipole_mode && !(epsilon_dipole >= 0)) return fail(c, CVR_ERR_INVALID, "'epsilon_dipole' has to be non-negative.");
  cudaSetDevice(c->device);
  c->slab_axis = slab_axis;
  c->slab_lz = slab_lz;
  c->dipole_mode = dipole_mode;
  c->eps_dipole = epsilon_dipole;
  c->epoch++;
  return refresh(c);
}

int cvr_set_ewald_slab_correction(cvr_ctx *c, int slab_axis, double lz, int kx_max, int ky_max, double k_e) {
  if (!c) return CVR_ERR_INVALID;
  if (slab_axis < 0) {
    c->sc_on = false;
    c->epoch++;
    return CVR_OK;
  }
  if (slab_axis > 2) return fail(c, CVR_ERR_INVALID, "expected 'x', 'y' or 'z'.");
  if (kx_max < 0 || ky_max < 0) return fail(c, CVR_ERR_INVALID, "'k_max' have to non-negative.");
  if (kx_max < 1 || ky_max < 1 || kx_max > SLAB_KMAX || ky_max > SLAB_KMAX)
    return fail(c, CVR_ERR_INVALID, "slab correction: kx_max and ky_max in [1, 8] on the B200 path");
  if (!(lz >= 0)) return fail(c, CVR_ERR_INVALID, "'lz' has to be non-negative.");
  if (!(k_e >= 0)) return fail(c, CVR_ERR_INVALID, "k_electrostatic has to be non-negative.");
  if (c->L[slab_axis] > lz) return fail(c, CVR_ERR_GEOMETRY, "expected 'hz > lz' for slab geometry");
  cudaSetDevice(c->device);
  if (!c->d_sc_state) {
    if (int r = dalloc(c, &c->d_sc_state, 2)) return r;  // zero: no moment before the first call
  }
  c->sc_on = true;
  c->sc_axis = slab_axis;
  c->sc_lz = lz;
  c->sc_kx = kx_max;
  c->sc_ky = ky_max;
  c->sc_ke = k_e;
  c->epoch++;
  return CVR_OK;
}

int cvr_set_integrator(cvr_ctx *c, double dt, double k_b) {
  if (!c) return CVR_ERR_INVALID;
  if (!(dt >= 0)) return fail(c, CVR_ERR_INVALID, "expected 'dt' input");
  if (!(k_b > 0)) return fail(c, CVR_ERR_INVALID, "k_b is not set.");
  if (dt != c->dt || k_b != c->k_b) c->epoch++;  // the step graphs bake dt and k_b in
  c->dt = dt;
  c->k_b = k_b;
  return CVR_OK;
}

int cvr_set_langevin(cvr_ctx *c, double temperature, double friction, double kb, double kbt, int rng,
                     uint64_t seed) {
  if (!c) return CVR_ERR_INVALID;
  if (temperature < 0 && temperature != -1) return fail(c, CVR_ERR_INVALID, "Temperature have to non-negative.");
  if (!(friction >= 0)) return fail(c, CVR_ERR_INVALID, "friction have to non-negative.");
  if (rng != CVR_RNG_REFERENCE && rng != CVR_RNG_PHILOX) return fail(c, CVR_ERR_INVALID, "unknown noise generator");
  if (!(kbt > 0) && !(kb > 0 && temperature > 0))
    return fail(c, CVR_ERR_INVALID, "expected ('temperature'  & 'kb') or 'kbt' input");
  c->integrator = 1;
  c->lgv_temperature = temperature;
  c->lgv_friction = friction;
  c->lgv_kb = kb;
  c->lgv_kbt = kbt;
  c->lgv_rng = rng;
  c->lgv_seed = seed;
  c->epoch++;  // the step graphs bake the integrator's kernels in
  return CVR_OK;
}

namespace {
int thermostat_buffer(cvr_ctx *c) {
  if (!c->d_tscal) {
    if (int r = dalloc(c, &c->d_tscal, 2)) return r;
    const double init[2] = {1.0, 0.0};
    CVR_CUDA(c, cudaMemcpyAsync(c->d_tscal, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  }
  return CVR_OK;
}
}  // namespace

int cvr_set_berendsen(cvr_ctx *c, double temperature, double coupling, double dt, int step, double lambda_min,
                      double lambda_max) {
  if (!c) return CVR_ERR_INVALID;
  if (!(temperature > 0)) return fail(c, CVR_ERR_INVALID, "Temperature have to non-negative.");
  if (!(coupling > 0)) return fail(c, CVR_ERR_INVALID, "coupling is not set.");
  if (!(dt > 0)) return fail(c, CVR_ERR_INVALID, "dt is not set.");
  if (step <= 0) return fail(c, CVR_ERR_INVALID, "step have to non-negative.");
  if (!(lambda_min > 0) || !(lambda_max > 0)) return fail(c, CVR_ERR_INVALID, "lambda_min, lambda_max > 0");
  if (int r = thermostat_buffer(c)) return r;
  c->tstat = ThermostatArgs{};
  c->tstat.kind = 1;
  c->tstat.T0 = temperature;
  c->tstat.tau = coupling;
  c->tstat.dt = dt;
  c->tstat.every = step;
  c->tstat.lambda_min = lambda_min;
  c->tstat.lambda_max = lambda_max;
  c->epoch++;  // the step graphs bake the thermostat in
  return CVR_OK;
}

int cvr_set_nose_hoover(cvr_ctx *c, double temperature, int type, double mass, double tau, double kb, double dt) {
  if (!c) return CVR_ERR_INVALID;
  if (!(temperature > 0)) return fail(c, CVR_ERR_INVALID, "Temperature have to non-negative.");
  if (!(dt > 0)) return fail(c, CVR_ERR_INVALID, "dt is not set.");
  if (type == 1 && !(mass > 0)) return fail(c, CVR_ERR_INVALID, "mass is not set.");
  if (type == 2 && !(tau > 0)) return fail(c, CVR_ERR_INVALID, "tau is not set.");
  if (type != 1 && type != 2)
    return fail(c, CVR_ERR_INVALID, "this Nose-Hoover type is not implemented.  Expected type 1 or 2");
  if (!(kb > 0)) return fail(c, CVR_ERR_INVALID, "kb have to non-negative.");
  if (int r = thermostat_buffer(c)) return r;
  c->tstat = ThermostatArgs{};
  c->tstat.kind = 2;
  c->tstat.T0 = temperature;
  c->tstat.dt = dt;
  c->tstat.nh_type = type;
  c->tstat.nh_mass = mass;
  c->tstat.nh_tau = tau;
  c->tstat.nh_kb = kb;
  const double zero = 0.0;
  CVR_CUDA(c, cudaMemcpyAsync(c->d_tscal + 1, &zero, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  c->epoch++;
  return CVR_OK;
}

int cvr_clear_thermostat(cvr_ctx *c) {
  if (!c) return CVR_ERR_INVALID;
  c->tstat = ThermostatArgs{};
  c->epoch++;
  return CVR_OK;
}

int cvr_set_kspace_force_kernel(cvr_ctx *c, int kind) {
  if (!c) return CVR_ERR_INVALID;
  if (kind != CVR_KFORCE_AUTO && kind != CVR_KFORCE_CUDA_CORES) return fail(c, CVR_ERR_INVALID, "unknown k-space force kernel");
  if (kind != c->kforce_kind) c->epoch++;  // the step graphs bake the kernel and its arguments in
  c->kforce_kind = kind;
  return CVR_OK;
}

int cvr_set_list_kernel(cvr_ctx *c, int kind) {
  if (!c) return CVR_ERR_INVALID;
  if (kind < CVR_LIST_AUTO || kind > CVR_LIST_WARP) return fail(c, CVR_ERR_INVALID, "unknown list kernel");
  if (kind != c->list_kernel) c->epoch++;  // the step graphs bake the list kernel in
  c->list_kernel = kind;
  return CVR_OK;
}

int cvr_set_precision(cvr_ctx *c, int precision) {
  if (!c) return CVR_ERR_INVALID;
  if (precision != CVR_PREC_MIXED && precision != CVR_PREC_FP64) return fail(c, CVR_ERR_INVALID, "unknown precision");
  if (c->have_state && precision != c->precision)
    return fail(c, CVR_ERR_STATE, "precision must be chosen before cvr_set_state");
  c->precision = precision;
  return CVR_OK;
}

int cvr_set_state(cvr_ctx *c, int64_t n, const double *pos, const double *vel, const int32_t *type,
                  const int32_t *mol) {
  if (!c) return CVR_ERR_INVALID;
  if (n <= 0 || n > (int64_t)INDEX_MASK || !pos || !type) return fail(c, CVR_ERR_INVALID, "bad atom arrays");
  if (c->all_atom && n > CVR_ALL_ATOM_MAX) return fail(c, CVR_ERR_INVALID, "all_atom_test is for small systems");
  cudaSetDevice(c->device);
  if (n != c->n || !c->x) {
    c->refreshed = false;
    if (int r = alloc_atoms(c, n)) return r;
    if (int r = dalloc(c, &c->stage, 9 * (size_t)n)) return r;
    c->cap = 0;
    c->tpa = choose_tpa(n);
    // list interleave: TPA lanes per atom, or quads of four entries when one lane per atom
    c->log2_tpa = (c->tpa == 32) ? 5 : (c->tpa == 8 ? 3 : 2);
  }
  // The types first, then the atoms per type on the GPU (the range check of
  // every type, and the charge and mass sums at one term per type), read
  // back with the positions behind them: the staged arrays reach the state
  // only after the check.  The velocities follow on the side stream: on a
  // context whose cells, tables and graphs stay, their copy runs beside the
  // run's setup (list build and first forces, which need no velocities),
  // done here, and they reach the atoms' places by id at the end.
  CVR_CUDA(c, cudaMemcpyAsync(c->stage_i, type, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaMemsetAsync(c->d_type_hist, 0, (MAX_TYPES + 1) * sizeof(unsigned long long), c->stream));
  k_type_hist<<<std::min<int64_t>(grid_for(n, 256), 4 * 148), 256, 0, c->stream>>>(c->stage_i, (int)n, c->n_types,
                                                                                  c->d_type_hist);
  c->launches++;
  unsigned long long per_type[MAX_TYPES + 1];
  CVR_CUDA(c, cudaMemcpyAsync(per_type, c->d_type_hist, sizeof(per_type), cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaMemcpyAsync(c->stage, pos, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (mol) CVR_CUDA(c, cudaMemcpyAsync(c->stage_i + n, mol, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  CVR_CUDA(c, cudaEventRecord(c->k_fork, c->stream));  // after the positions: they take the link first
  CVR_CUDA(c, cudaStreamWaitEvent(c->kstream, c->k_fork, 0));
  if (vel)
    CVR_CUDA(c, cudaMemcpyAsync(c->stage + 3 * n, vel, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice,
                                c->kstream));
  CVR_CUDA(c, cudaEventRecord(c->k_join, c->kstream));
  CVR_CUDA(c, cudaStreamSynchronize(c->stream));
  if (per_type[MAX_TYPES] != 0) {
    cudaStreamSynchronize(c->kstream);  // the caller's velocity array is borrowed until the copy ends
    return fail(c, CVR_ERR_INVALID, "atom type out of range");
  }
  c->have_state = true;
  const bool mol_changed = (mol != nullptr) != c->use_mol;
  c->use_mol = mol != nullptr;
  double q2 = 0, mt = 0;
  for (int t = 0; t < c->n_types; ++t) {
    q2 += (double)per_type[t] * (c->charge[t] * c->charge[t]);
    mt += (double)per_type[t] * c->mass[t];
  }
  // the step graphs bake these in (thermo kernel, pair-kernel choice)
  if (mol_changed || mt != c->total_mass || q2 != c->q2_sum) c->epoch++;
  c->total_mass = mt;
  c->q2_sum = q2;
  c->e_self = self_energy(c);
  if (c->precision == CVR_PREC_FP64) {
    DevState<double> s = dev_state<double>(c);
    k_scatter_state<double><<<grid_for(n, 256), 256, 0, c->stream>>>(s, c->stage, nullptr, c->stage_i,
                                                                      mol ? c->stage_i + n : nullptr);
  } else {
    DevState<float> s = dev_state<float>(c);
    k_scatter_state<float><<<grid_for(n, 256), 256, 0, c->stream>>>(s, c->stage, nullptr, c->stage_i,
                                                                    mol ? c->stage_i + n : nullptr);
  }
  c->launches++;
  CVR_CUDA(c, cudaMemsetAsync(c->flags, 0, 4 * sizeof(int), c->stream));
  c->step = 0;
  int rs = CVR_OK;
  if (!c->refreshed || mol_changed) {
    rs = refresh(c);
  } else {
    // same atom count and settings: cells, tables and buffers stay (and so
    // do the step graphs); the list and the forces are redone now, beside
    // the velocity copy (what the next run's setup would do)
    c->list_valid = false;
    c->setup_done = false;
    rs = DISPATCH(c, setup_run, c);
  }
  // the host arrays are borrowed for this call only: the copies from them
  // (asynchronous when they are pinned) end before it returns
  cudaError_t e = cudaStreamWaitEvent(c->stream, c->k_join, 0);
  if (vel && e == cudaSuccess) {
    if (c->precision == CVR_PREC_FP64)
      k_place_velocities<double><<<grid_for(n, 256), 256, 0, c->stream>>>(dev_state<double>(c), c->stage + 3 * n);
    else
      k_place_velocities<float><<<grid_for(n, 256), 256, 0, c->stream>>>(dev_state<float>(c), c->stage + 3 * n);
    c->launches++;
  }
  const cudaError_t e2 = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, CVR_ERR_CUDA, cudaGetErrorString(e));
  return rs;
}

int cvr_build_neighbors(cvr_ctx *c, int force, int *rebuilt) {
  if (!c) return CVR_ERR_INVALID;
  if (int r = ensure_ready(c)) return r;
  cudaSetDevice(c->device);
  int f0[4];
  if (int r = read_flags(c, f0)) return r;
  if (force || !c->list_valid) {
    if (int r = DISPATCH(c, do_build, c, true)) return r;
  } else {
    if (c->precision == CVR_PREC_FP64) {
      k_check<double><<<grid_for(c->n, 256), 256, 0, c->stream>>>(dev_state<double>(c));
    } else {
      k_check<float><<<grid_for(c->n, 256), 256, 0, c->stream>>>(dev_state<float>(c));
    }
    c->launches++;
    if (int r = DISPATCH(c, do_build, c, false)) return r;
  }
  CVR_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(int), c->stream));
  int f[4];
  if (int r = read_flags(c, f)) return r;
  collect_timing(c);
  if (f[1] & ERR_OVERFLOW) {
    if (int r = regrow(c)) return r;
    if (int r = DISPATCH(c, do_build, c, true)) return r;
    CVR_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(int), c->stream));
    if (int r = read_flags(c, f)) return r;
    if (f[1] & ERR_OVERFLOW) return fail(c, CVR_ERR_CAPACITY, "neighbour list overflow");
  }
  c->list_valid = true;
  if (rebuilt) *rebuilt = (f[3] != f0[3]) ? 1 : 0;
  return CVR_OK;
}

int cvr_compute_forces(cvr_ctx *c, double *acc, double *thermo) {
  if (!c) return CVR_ERR_INVALID;
  if (int r = ensure_ready(c)) return r;
  cudaSetDevice(c->device);
  return DISPATCH(c, compute_impl, c, acc, thermo);
}

int cvr_run(cvr_ctx *c, int64_t nsteps, int64_t every, double *thermo) {
  if (!c) return CVR_ERR_INVALID;
  if (nsteps < 0 || every < 0) return fail(c, CVR_ERR_INVALID, "negative step count");
  if (int r = ensure_ready(c)) return r;
  cudaSetDevice(c->device);
  return DISPATCH(c, run_impl, c, nsteps, every, thermo);
}

int cvr_get_state(cvr_ctx *c, double *pos, double *vel, double *acc) {
  if (!c) return CVR_ERR_INVALID;
  if (!c->have_state) return fail(c, CVR_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  const int64_t n = c->n;
  double *dp = c->stage, *dv = c->stage + 3 * n, *da = c->stage + 6 * n;
  if (c->precision == CVR_PREC_FP64)
    k_gather_state<double><<<grid_for(n, 256), 256, 0, c->stream>>>(dev_state<double>(c), dp, dv, da);
  else
    k_gather_state<float><<<grid_for(n, 256), 256, 0, c->stream>>>(dev_state<float>(c), dp, dv, da);
  c->launches++;
  if (pos) CVR_CUDA(c, cudaMemcpyAsync(pos, dp, n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (vel) CVR_CUDA(c, cudaMemcpyAsync(vel, dv, n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (acc) CVR_CUDA(c, cudaMemcpyAsync(acc, da, n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CVR_CUDA(c, cudaStreamSynchronize(c->stream));
  return CVR_OK;
}

int64_t cvr_get_pairs(cvr_ctx *c, int32_t *out) {
  if (!c) return -CVR_ERR_INVALID;
  if (!c->list_valid || c->cap == 0) return -fail(c, CVR_ERR_STATE, "no neighbour list");
  cudaSetDevice(c->device);
  std::vector<std::array<int32_t, 5>> p;
  int r = DISPATCH(c, pairs_impl, c, p);
  if (r) return -r;
  if (out) std::memcpy(out, p.data(), p.size() * sizeof(p[0]));
  return (int64_t)p.size();
}

int64_t cvr_get_sk(cvr_ctx *c, double *out) {
  if (!c) return -CVR_ERR_INVALID;
  if (!c->ewk_on) return 0;
  cudaSetDevice(c->device);
  if (out) {
    cudaError_t e = cudaMemcpyAsync(out, c->d_sk, (size_t)c->nk * sizeof(double2), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return -fail(c, CVR_ERR_CUDA, cudaGetErrorString(e));
  }
  return c->nk;
}

int cvr_get_scalars(cvr_ctx *c, double *thermo) {
  if (!c || !thermo) return CVR_ERR_INVALID;
  std::memcpy(thermo, c->last_thermo, sizeof(c->last_thermo));
  return CVR_OK;
}

int cvr_last_error(const cvr_ctx *c, char *buf, size_t len) {
  if (!c || !buf || len == 0) return CVR_ERR_INVALID;
  std::snprintf(buf, len, "%s", c->err.c_str());
  return CVR_OK;
}

int64_t cvr_launch_count(const cvr_ctx *c) { return c ? c->launches : -1; }

void *cvr_get_stream(const cvr_ctx *c) { return c ? (void *)c->stream : nullptr; }

int cvr_get_info(const cvr_ctx *c, int64_t *out, int len) {
  if (!c || !out) return CVR_ERR_INVALID;
  int flags[4] = {0, 0, 0, 0};
  if (c->flags) {
    cudaMemcpyAsync(flags, c->flags, sizeof(flags), cudaMemcpyDeviceToHost, c->stream);
    cudaStreamSynchronize(c->stream);
  }
  int64_t entries = 0;
  if (len > 12 && c->ncount && c->list_valid) {
    std::vector<int> cnt(c->n);
    cudaMemcpyAsync(cnt.data(), c->ncount, c->n * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    cudaStreamSynchronize(c->stream);
    for (int v : cnt) entries += v;
  }
  const int64_t v[15] = {c->n,     c->nc[0], c->nc[1], c->nc[2], c->cap,   flags[3], c->tpa,
                         c->nk,    c->R,     flags[2], flags[1], c->step, entries,  c->fixed,
                         (c->ewk_on && c->nk > 0 && kforce_tc(c)) ? 1 : 0};
  for (int k = 0; k < len && k < 15; ++k) out[k] = v[k];
  return CVR_OK;
}

int cvr_set_kernel_timing(cvr_ctx *c, int on) {
  if (!c) return CVR_ERR_INVALID;
  collect_timing(c);
  c->timing = on != 0;
  for (auto &k : c->kt) {
    k.ms = 0;
    k.launches = 0;
  }
  return CVR_OK;
}

int cvr_kernel_time(cvr_ctx *c, int kind, double *ms, int64_t *launches) {
  if (!c || kind < 0 || kind >= CVR_N_KT) return CVR_ERR_INVALID;
  collect_timing(c);
  if (ms) *ms = c->kt[kind].ms;
  if (launches) *launches = c->kt[kind].launches;
  return CVR_OK;
}

}  // extern "C"
