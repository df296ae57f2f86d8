// cvr_force.cuh -- force, k-space and integrator kernels (sm_100a).
//
// Replaces, in the reference (CAVIAR; paths relative to its project root):
//   force_field::Lj::calculate_acceleration            src/caviar/objects/force_field/lj.cpp:355-483
//   Electrostatic_ewald_r::calculate_acceleration      src/caviar/objects/force_field/electrostatic_ewald_r.cpp:115-317
//   Electrostatic_ewald_k::calculate_potential_k_coef_cmplx  .../electrostatic_ewald_k/initialize.cpp:117-146
//   Electrostatic_ewald_k::calculate_acceleration      .../electrostatic_ewald_k.cpp:161-294
//   k_space_energy / self_energy                       .../electrostatic_ewald_k/energy.cpp:31-116
//   Md_simulator::integrate_velocity_verlet            src/caviar/objects/md_simulator.cpp:555-668
//   Atom_data::kinetic_energy / finalize_temperature   src/caviar/objects/atom_data/kinetic_energy.cpp:30-202
//
// Structure differs from the reference on purpose: the reference runs a
// half list with Newton's third law (scatter into j), which on a GPU needs
// atomics and gives run-to-run different sums.  Here the list is full
// (every pair in both atoms' rows) and each atom sums its own force in a
// fixed order: no atomics, bit-reproducible.  LJ and Ewald real space share
// one pass over the list.  Energies and virial are FP64 block sums.
#pragma once
#include "cvr_device.cuh"
#include <type_traits>

// List entries each pair-kernel lane has in flight, and the minimum resident
// blocks the pair kernel is compiled for.
#ifndef CVR_PAIR_UNROLL
#define CVR_PAIR_UNROLL 4
#endif
#ifndef CVR_PAIR_MINB
#define CVR_PAIR_MINB 1
#endif
// k-force kernel: minimum resident blocks (FP32) and 16-byte coefficient
// loads in flight per lane while staging.
#ifndef CVR_KF_MINB
#define CVR_KF_MINB 1
#endif
#ifndef CVR_KF_SB
#define CVR_KF_SB 4
#endif

namespace cvr {

template <typename real> struct R2;
template <> struct R2<float> { using t = float2; };
template <> struct R2<double> { using t = double2; };

__device__ __forceinline__ float fast_rcp(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double fast_rcp(double x) { return 1.0 / x; }
__device__ __forceinline__ float fast_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double fast_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float fast_exp(float x) { return __expf(x); }
__device__ __forceinline__ double fast_exp(double x) { return exp(x); }
__device__ __forceinline__ double erfc_r(double x) { return erfc(x); }
__device__ __forceinline__ int type_of(float w) { return __float_as_int(w); }
__device__ __forceinline__ int type_of(double w) { return (int)w; }
__device__ __forceinline__ void sincospi_r(float a, float *s, float *c) { sincospif(a, s, c); }
__device__ __forceinline__ void sincospi_r(double a, double *s, double *c) { sincospi(a, s, c); }

// Stencil offset of a list entry, (dx, dy, dz) * cell width, from its three
// 3-bit fields.  The small integer field is turned into a float exactly by
// placing it in the mantissa of 2^23 and subtracting 2^23 (+ R): no
// int-to-float conversion instruction and no table lookup (the offset table
// in shared memory was the busiest user of the L1 data pipe).
__device__ __forceinline__ float stencil_f(uint32_t e, int shift, float bias) {
  return __uint_as_float(0x4B000000u | ((e >> shift) & 7u)) - bias;
}
__device__ __forceinline__ double stencil_f64(uint32_t e, int shift, double bias) {
  return __longlong_as_double(0x4330000000000000ll | (long long)((e >> shift) & 7u)) - bias;
}
template <typename real> struct Stencil;
template <> struct Stencil<float> {
  float bias, wx, wy, wz;
  __device__ __forceinline__ void get(uint32_t e, float &ox, float &oy, float &oz) const {
    ox = stencil_f(e, CODE_SHIFT, bias) * wx;
    oy = stencil_f(e, CODE_SHIFT + 3, bias) * wy;
    oz = stencil_f(e, CODE_SHIFT + 6, bias) * wz;
  }
};
template <> struct Stencil<double> {
  double bias, wx, wy, wz;
  __device__ __forceinline__ void get(uint32_t e, double &ox, double &oy, double &oz) const {
    ox = stencil_f64(e, CODE_SHIFT, bias) * wx;
    oy = stencil_f64(e, CODE_SHIFT + 3, bias) * wy;
    oz = stencil_f64(e, CODE_SHIFT + 6, bias) * wz;
  }
};

// Block-wide sum of NV doubles into out[blockIdx.x * NV + q] (fixed order).
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double *out) {
  __shared__ double red[NV][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double x = (lane < nw) ? red[q][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) out[(size_t)blockIdx.x * NV + q] = x;
    }
  }
}

template <typename real> struct EwrArgs {
  real alpha, alpha2, two_alpha_spi;  // alpha, alpha^2, 2 alpha / sqrt(pi)
  real cut2;                          // < 0: no cutoff (the reference)
};

// --------------------------------------------------------------- pair force
// TPA lanes per atom stride through the atom's list row; lanes reduce with
// shuffles.  use_mol enables the molecule tests (ignore_intra_molecule,
// Ewald lambda).  ONE_TYPE keeps the single type pair's LJ constants in
// registers (no table lookups).  The LJ cutoff is a select, not a branch.
// EV adds energies + virial (FP64 per thread, FP64 block sums into
// partials[block*3 + {e_lj, e_ewr, virial}]).  Entries are unrolled by
// CVR_PAIR_UNROLL so that several neighbour gathers are in flight per lane.
// Energies and virial: each group of entries (a quad, or one unrolled round)
// is summed in `real`, then added to the FP64 per-atom totals (ev_flush),
// one conversion per group instead of per pair.
template <typename real> struct PairAcc {
  real fx, fy, fz;
  double e_lj, e_ew, vir;
  real g_lj, g_ew, g_vir;
};

template <bool LJ, bool EWR, typename real>
__device__ __forceinline__ void ev_flush(PairAcc<real> &A) {
  if (LJ) A.e_lj += (double)A.g_lj;
  if (EWR) A.e_ew += (double)A.g_ew;
  A.vir += (double)A.g_vir;
  A.g_lj = A.g_ew = A.g_vir = (real)0;
}

// JUMP (the multi-type kernels only): the reference's LJ jump_tol clamp
// (lj.cpp:423-432): after the cutoff test, r^2 below jump_tol is raised to
// it for the LJ coefficient (and the LJ virial and energy); the force keeps
// the true displacement.
template <typename real, bool LJ, bool EWR, bool EV, bool JUMP = false>
__device__ __forceinline__ void pair_term(PairAcc<real> &A, real dx, real dy, real dz, const PairCoef<real> &pc,
                                          bool same_mol, int ignore_intra, const EwrArgs<real> &ew) {
  const real r2 = dx * dx + dy * dy + dz * dz;
  real c = 0, vir_lj = 0;
  if (LJ) {
    // lj.cpp:417-448: skip r^2 > rc^2 (rc2 < 0 when eps = 0).  With Ewald
    // real space the list reaches its cutoff, far beyond the LJ one, and few
    // pairs are inside: the LJ term is then branched around (the same values)
    // instead of computed for every pair and selected.
    const bool in = (r2 <= pc.rc2) && !(same_mol && ignore_intra);
    if (!EWR || in) {
      const real r2l = JUMP ? (r2 < pc.jump2 ? pc.jump2 : r2) : r2;
      const real r2i = fast_rcp(r2l);
      const real s2 = pc.sig2 * r2i;
      const real s6 = s2 * s2 * s2;
      const real cl = r2i * s6 * (pc.eps24 - pc.eps48 * s6) + pc.K;
      c = in ? cl : (real)0;
      if (EV && in) A.g_lj += pc.e4 * (s6 * s6 - s6) + pc.C1 * r2l + pc.C0;
      if (EV && JUMP) vir_lj = c * r2l;
    }
  }
  const real c_lj = c;
  if (EWR) {
    // electrostatic_ewald_r.cpp:179-198: every list pair, coincident skipped
    if (r2 > (real)0 && (ew.cut2 < (real)0 || r2 <= ew.cut2)) {
      const real rinv = fast_rsqrt(r2);
      const real r = r2 * rinv;
      const real ex = fast_exp(-ew.alpha2 * r2);  // exp(-(alpha r)^2)
      real erfcv;
      if constexpr (sizeof(real) == 4)
        erfcv = erfc_as(ew.alpha * r, ex);  // shares ex with the force term
      else
        erfcv = erfc_r(ew.alpha * r);
      const real sv = (ew.two_alpha_spi * ex + erfcv * rinv) * (rinv * rinv);
      const real lam = same_mol ? pc.lam : (real)1;
      c -= lam * pc.qq * sv;
      if (EV) A.g_ew += lam * pc.qq * erfcv * rinv;
    }
  }
  A.fx += c * dx;
  A.fy += c * dy;
  A.fz += c * dz;
  if (EV) {
    if (JUMP)
      A.g_vir -= vir_lj + (c - c_lj) * r2;
    else
      A.g_vir -= c * r2;
  }
}

// Pair displacement r_j - r_i.  Cell-local form: (x4_j - x4_i) + the entry's
// stencil offset.  Fixed-point form (FIXED, mixed precision only): the
// wrapping int32 difference of the 32-bit coordinates, converted to float in
// units of L / 2^32 (the pair kernel's coefficients are scaled to match).
template <typename real, bool FIXED, typename real4>
__device__ __forceinline__ void pair_disp(const real4 &xj, const real4 &xi, uint32_t e, const Stencil<real> &st,
                                          real &dx, real &dy, real &dz) {
  if constexpr (FIXED) {
    (void)e;
    (void)st;
    dx = (real)(int)(__float_as_uint(xj.x) - __float_as_uint(xi.x));
    dy = (real)(int)(__float_as_uint(xj.y) - __float_as_uint(xi.y));
    dz = (real)(int)(__float_as_uint(xj.z) - __float_as_uint(xi.z));
  } else {
    real ox, oy, oz;
    st.get(e, ox, oy, oz);
    dx = (xj.x - xi.x) + ox;
    dy = (xj.y - xi.y) + oy;
    dz = (xj.z - xi.z) + oz;
  }
}

// FIXED: x4 holds fixed-point coordinates; coef_g and ew are in units of
// L / 2^32 and fscale = 2^32 / L turns the summed force back into length
// units (the virial and energies come out unscaled).  Otherwise fscale = 1.
// book != 0 (a step whose second half kick is deferred to the next step's
// k_kick_drift): block 0 takes over k_kick's end-of-step bookkeeping, the
// rebuild flag reset and the step count.
template <typename real, int TPA, bool LJ, bool EWR, bool EV, bool ONE_TYPE, bool FIXED>
__global__ void __launch_bounds__(128, CVR_PAIR_MINB) k_pair(DevState<real> s, const PairCoef<real> *__restrict__ coef_g,
                                              real fscale, EwrArgs<real> ew,
                                              int ignore_intra, int use_mol, double *__restrict__ partials,
                                              int book, long long *__restrict__ counters) {
  if (book && blockIdx.x == 0 && threadIdx.x == 0) {
    *s.flag = 0;
    if (counters) counters[0]++;
  }
  using real4 = typename V4<real>::t;
  __shared__ PairCoef<real> coef[ONE_TYPE ? 1 : MAX_TYPES * MAX_TYPES];
  const int T = s.n_types;
  for (int t = threadIdx.x; t < (ONE_TYPE ? 1 : T * T); t += blockDim.x) coef[t] = coef_g[t];
  Stencil<real> st;
  st.bias = (real)(sizeof(real) == 4 ? 8388608.0 : 4503599627370496.0) + (real)s.cells.R;
  st.wx = (real)s.cells.w[0];
  st.wy = (real)s.cells.w[1];
  st.wz = (real)s.cells.w[2];
  __syncthreads();
  if (*s.err) return;

  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = gid / TPA, lane = gid % TPA;
  const bool valid = i < s.n;
  PairAcc<real> A{0, 0, 0, 0.0, 0.0, 0.0, 0, 0, 0};
  int ti = 0;
  if (valid) {
    const real4 xi = s.x4[i];
    ti = type_of(xi.w);
    const bool um = !ONE_TYPE && use_mol;  // the single-type instantiation runs without molecules
    const int moli = um ? s.mol[i] : 0;
    const int cnt = s.ncount[i];
    const PairCoef<real> *ci = coef + (ONE_TYPE ? 0 : ti * T);
    PairCoef<real> c1;
    if (ONE_TYPE) c1 = coef[0];
    if (TPA == 1) {
      // one lane per atom: entries in quads, one 16-byte load per four; the
      // next quad is loaded before this one's neighbours are gathered, so
      // the list stream's HBM latency overlaps the gathers and the math.
      // Full quads need no per-entry count test; the last, partial one does.
      const uint4 *q4 = reinterpret_cast<const uint4 *>(s.nlist) + i;
      uint4 nxt = make_uint4(0u, 0u, 0u, 0u);
      if (cnt > 0) nxt = __ldcs(q4);
      const int full = cnt & ~3;
      auto quad = [&](const uint4 &e4, int nv, auto check) {
        constexpr bool CHECK = decltype(check)::value;
        const uint32_t e[4] = {e4.x, e4.y, e4.z, e4.w};
        real4 xj[4];
        bool sm[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = (!CHECK || u < nv) ? (int)(e[u] & INDEX_MASK) : i;
          xj[u] = s.x4[j];
          sm[u] = um && (moli == s.mol[j]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (!CHECK || u < nv) {
            real dx, dy, dz;
            pair_disp<real, FIXED>(xj[u], xi, e[u], st, dx, dy, dz);
            pair_term<real, LJ, EWR, EV, !ONE_TYPE>(A, dx, dy, dz, ONE_TYPE ? c1 : ci[type_of(xj[u].w)], sm[u], ignore_intra,
                                         ew);
          }
        }
        if (EV) ev_flush<LJ, EWR>(A);
      };
      for (int k = 0; k < full; k += 4) {
        const uint4 e4 = nxt;
        q4 += s.n_pad;
        if (k + 4 < cnt) nxt = __ldcs(q4);
        quad(e4, 4, std::false_type{});
      }
      if (cnt > full) quad(nxt, cnt - full, std::true_type{});
    } else {
      const size_t stride = (size_t)s.n_pad * TPA;
      const uint32_t *row = s.nlist + (size_t)i * TPA + lane;
      constexpr int U = CVR_PAIR_UNROLL;
      int k = lane;
      for (; k + (U - 1) * TPA < cnt; k += U * TPA) {
        uint32_t e[U];
#pragma unroll
        for (int u = 0; u < U; ++u) e[u] = __ldcs(row + u * stride);
        row += U * stride;
        real4 xj[U];
        bool sm[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = (int)(e[u] & INDEX_MASK);
          xj[u] = s.x4[j];
          sm[u] = um && (moli == s.mol[j]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          real dx, dy, dz;
          pair_disp<real, FIXED>(xj[u], xi, e[u], st, dx, dy, dz);
          pair_term<real, LJ, EWR, EV, !ONE_TYPE>(A, dx, dy, dz, ONE_TYPE ? c1 : ci[type_of(xj[u].w)], sm[u], ignore_intra,
                                       ew);
        }
        if (EV) ev_flush<LJ, EWR>(A);
      }
      for (; k < cnt; k += TPA) {
        const uint32_t e0 = __ldcs(row);
        row += stride;
        const int j0 = (int)(e0 & INDEX_MASK);
        const real4 xj0 = s.x4[j0];
        const bool sm0 = um && (moli == s.mol[j0]);
        real dx, dy, dz;
        pair_disp<real, FIXED>(xj0, xi, e0, st, dx, dy, dz);
        pair_term<real, LJ, EWR, EV, !ONE_TYPE>(A, dx, dy, dz, ONE_TYPE ? c1 : ci[type_of(xj0.w)], sm0, ignore_intra, ew);
      }
      if (EV) ev_flush<LJ, EWR>(A);
    }
  }
#pragma unroll
  for (int o = TPA / 2; o > 0; o >>= 1) {
    A.fx += __shfl_xor_sync(0xffffffffu, A.fx, o);
    A.fy += __shfl_xor_sync(0xffffffffu, A.fy, o);
    A.fz += __shfl_xor_sync(0xffffffffu, A.fz, o);
  }
  if (valid && lane == 0) {
    const real mi = (real)s.mass_inv[ti] * fscale;
    s.ax[i] = A.fx * mi;
    s.ay[i] = A.fy * mi;
    s.az[i] = A.fz * mi;
  }
  if (EV) {
    double v[3] = {0.5 * A.e_lj, 0.5 * A.e_ew, 0.5 * A.vir};  // full list: each pair twice
    block_sum_store<3>(v, partials);
  }
}

// ------------------------------------------------ all-atom test (debug mode)
// The reference's neighbour-list switch all_atom_test (neighborlist.cpp:
// 161-191): the list holds every owned pair once and every owned atom with
// every ghost image, with no distance test, so LJ keeps its own cutoff test
// and the Ewald real-space sum runs over every pair and image.  One thread
// per atom: every other atom at its direct displacement (no minimum image,
// as the reference's owned-owned entries), then every current ghost image
// (atom a at r_a + s L for each non-empty subset of the axes of a's ghost
// zones, s = -zone, exchange_ghost_single_md_domain.cpp:59-215).  Positions
// are the wrapped ones of this step's build (the mode rebuilds every step).
// Energies: each owned pair once, each owned-ghost term with weight 1/2 (the
// reference has no energy of this asymmetric sum); virial as the reference:
// each owned pair once, an owned-ghost term when id_i < id_a (lj.cpp:451-453).
// O(n (n + ghosts)): small systems only.
template <typename real, bool LJ, bool EWR, bool EV>
__global__ void __launch_bounds__(128) k_pair_all(DevState<real> s, const PairCoef<real> *__restrict__ coef_g,
                                                  EwrArgs<real> ew, int ignore_intra, int use_mol,
                                                  double *__restrict__ partials) {
  __shared__ PairCoef<real> coef[MAX_TYPES * MAX_TYPES];
  const int T = s.n_types;
  for (int t = threadIdx.x; t < T * T; t += blockDim.x) coef[t] = coef_g[t];
  __syncthreads();
  if (*s.err) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double fx = 0, fy = 0, fz = 0, e_lj = 0, e_ew = 0, vir = 0;
  int ti = 0;
  if (i < s.n) {
    const double xi = s.x[i], yi = s.y[i], zi = s.z[i];
    ti = s.type[i];
    const int mi = use_mol ? s.mol[i] : 0, idi = s.id[i];
    const PairCoef<real> *ci = coef + ti * T;
    // one pair term in `real` (displacement rounded from FP64), summed in
    // FP64 with energy weight w_e and virial weight w_v
    auto term = [&](double dx, double dy, double dz, int j, double w_e, double w_v) {
      PairAcc<real> A{0, 0, 0, 0.0, 0.0, 0.0, 0, 0, 0};
      const bool sm = use_mol && mi == s.mol[j];
      pair_term<real, LJ, EWR, EV, true>(A, (real)dx, (real)dy, (real)dz, ci[s.type[j]], sm, ignore_intra, ew);
      fx += (double)A.fx;
      fy += (double)A.fy;
      fz += (double)A.fz;
      if (EV) {
        e_lj += w_e * (double)A.g_lj;
        e_ew += w_e * (double)A.g_ew;
        vir += w_v * (double)A.g_vir;
      }
    };
    // owned pairs: each end computes its own term, so energy and virial take half
    for (int j = 0; j < s.n; ++j)
      if (j != i) term(s.x[j] - xi, s.y[j] - yi, s.z[j] - zi, j, 0.5, 0.5);
    for (int a = 0; a < s.n; ++a) {
      const int code = s.gcls[a];
      const int v[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
      if ((v[0] | v[1] | v[2]) == 0) continue;
      for (int m = 1; m < 8; ++m) {
        bool ok = true;
        double sh[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const bool on = (m >> d) & 1;
          if (on && v[d] == 0) ok = false;
          sh[d] = on ? -(double)v[d] * s.box.L[d] : 0.0;
        }
        if (!ok) continue;
        term((s.x[a] + sh[0]) - xi, (s.y[a] + sh[1]) - yi, (s.z[a] + sh[2]) - zi, a, 0.5, idi < s.id[a] ? 1.0 : 0.0);
      }
    }
    const double mi_inv = s.mass_inv[ti];
    s.ax[i] = (real)(fx * mi_inv);
    s.ay[i] = (real)(fy * mi_inv);
    s.az[i] = (real)(fz * mi_inv);
  }
  if (EV) {
    double v3[3] = {e_lj, e_ew, vir};
    block_sum_store<3>(v3, partials);
  }
}

// ------------------------------------------------------------------ k space
// The reference's k-set (initialize.cpp:184-222) is regrouped by (nx, ny)
// column: for column c and m = 0..kmax_z, kpm[m * nxy + c] holds the indices
// of (nx, ny, +m) and (nx, ny, -m) in the k-set (-1 where the set lacks
// it).  e^{i k.r} = X[nx] Y[ny] Z[+-m] with Z[-m] = conj(Z[m]), so one
// complex product P = X Y serves a whole column and each +-m pair costs
// eight FMAs in both the S(k) and the force kernel.
// Tensor-core form of the k-space force (k_kforce_tc, mixed form): per
// block of 128 atoms, D[atom][(column, c)] = sum_k Z[atom][k] B[(column, c)][k]
// with k = (Re z_m, Im z_m) for m < M (zero padded to KTC_K) and c = the
// four sums Cx, Cy, Dx, Dy of k_kforce, as TF32 hi/lo halves (3 products
// per term: hi hi + hi lo + lo hi, FP32-level).  B comes from k_sk_reduce as
// an image of KTC_COLS-column tiles in the MMA's canonical K-major layout
// without swizzle: 8-row x 16-byte core matrices, adjacent in K every 128
// bytes, 8-row groups every KTC_K / 4 * 128 bytes.
constexpr int KTC_ATOMS = 128;                      // atoms per block = TMEM lanes = MMA M
constexpr int KTC_COLS = 64;                        // (nx, ny) columns per N-tile
constexpr int KTC_N = 4 * KTC_COLS;                 // MMA N
constexpr int KTC_K = 24;                           // 2 M <= 24
constexpr int KTC_KPMAX = 12;                       // kmax + 1 per axis held for the epilogue
constexpr int KTC_TILE_FLOATS = KTC_N * KTC_K;      // one operand image (hi or lo) of an N-tile
__host__ __device__ constexpr int ktc_off(int r, int k) {  // byte offset of (row, k) in an operand image
  return (r & 7) * 16 + (k >> 2) * 128 + (r >> 3) * (KTC_K / 4 * 128) + (k & 3) * 4;
}
// TF32 rounding (round to nearest, ties away) of an FP32 value, kept as FP32.
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

template <typename real> struct KArgs {
  int nk, nxy, M, kmax[3], kp;  // M = kmax_z + 1 m-values; kp = max kmax + 1
  const int2 *xy;               // (nx, ny) per column
  // S(k) symmetry: S(-nx, -ny, +-m) = conj(S(nx, ny, -+m)) for real charges,
  // so only ncomp columns (one of each mirror pair present) are summed:
  const int2 *xyc;              // (nx, ny) of the summed columns
  const int *ksrc;              // per column: its summed column, | 1 << 30 if taken from the mirror
  const int *kmir;              // per summed column: the column taken from it (its mirror), or -1
  int ncomp;
  const int2 *kpm;              // [M][nxy] k indices of (nx, ny, +m), (nx, ny, -m)
  const double *fk;             // exp(-k^2/4a^2)/k^2 per used k
  typename R2<real>::t *ptab;   // phase tables [3 * kp][n]
  double2 *partial;             // [nchunks][M][nxy][2]: S(+m), S(-m) of one atom chunk
  double2 *sk;                  // S(k)
  real *kcoef;                  // [nxy][M][8] force coefficients (see k_sk_reduce)
  double *e_partials;           // per block of k_sk_reduce
  double inv_L[3];
  real two_pi_over_L[3];
  double four_pi_over_v;
  double *charge;               // per type
  double k_e;
  int nchunks;
  float *kimg;                  // tensor-core coefficient image (k_kforce_tc), else null
};

// Phase e^{i 2 pi m x / L} from the fractional part of m x / L in FP64 (so
// |x| up to the box size costs no phase accuracy), then sincospi in `real`.
template <typename real>
__device__ __forceinline__ typename R2<real>::t phase(double x_over_L, int m) {
  const double u = (double)m * x_over_L;
  const double f = u - rint(u);
  real sn, cs;
  sincospi_r((real)(2.0 * f), &sn, &cs);
  typename R2<real>::t r;
  r.x = cs;
  r.y = sn;
  return r;
}

template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
  T r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T>
__device__ __forceinline__ T conj_if(T a, bool c) {
  if (c) a.y = -a.y;
  return a;
}

// One atom's phase-table row of one axis: e^{i 2 pi m x / L}, m = 0..kmax,
// into ptab[(row0 + m) * n + i].  Every fourth m is evaluated directly
// (phase), the others as the previous value times the m = 1 phase, so each
// entry is at most three complex products away from a direct value.
template <typename real>
__device__ __forceinline__ void phase_row(typename R2<real>::t *__restrict__ ptab, size_t n, int i, int row0,
                                          double x_over_L, int kmax) {
  using c2 = typename R2<real>::t;
  const c2 e1 = phase<real>(x_over_L, 1);
  c2 z;
  z.x = (real)1;
  z.y = (real)0;
  for (int m = 0; m <= kmax; ++m) {
    if (m > 0) z = (m & 3) ? cmul(z, e1) : phase<real>(x_over_L, m);
    ptab[(size_t)(row0 + m) * n + i] = z;
  }
}

// Phase tables of every atom, once per force evaluation:
// ptab[(d * kp + m) * n + i] = e^{i 2 pi m x_d / L_d}, m = 0..kmax_d
// (row-major by (d, m), so 32 consecutive atoms are 32 consecutive words).
// gate: when set, the launch belongs to a list build and returns unless the
// build's flag is raised (the build reorders atoms: the step's tables, made
// by the position update, are rewritten in the new order).
template <typename real>
__global__ void __launch_bounds__(256) k_phase(DevState<real> s, KArgs<real> a, const int *__restrict__ gate) {
  if (gate && *gate == 0) return;
  if (*s.err) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // one thread per (axis, atom)
  if (t >= 3 * s.n) return;
  const int d = t / s.n, i = t - d * s.n;
  const double x = ((d == 0) ? s.x[i] : ((d == 1) ? s.y[i] : s.z[i])) * a.inv_L[d];
  phase_row<real>(a.ptab, s.n, i, d * a.kp, x, a.kmax[d]);
}

// S(k) partial sums (electrostatic_ewald_k/initialize.cpp:117-146): one thread per
// (column, group of MG m-values), one block row per chunk of CH atoms whose
// phase tables and charges sit in shared memory.  Table rows per atom
// (atom-major, so the lanes' X and Y rows of one atom are distinct words,
// conflict-free): X[0..kp), Y[0..kp), Z[0..MG * groups), zero past kmax and
// past the chunk's last atom, so the inner loops need no guards.
// Consecutive threads take consecutive columns of one m-group: the Z loads
// are warp broadcasts.  Products are summed in `real` over groups of 16
// atoms; groups accumulate in FP64; chunks are summed by k_sk_reduce in a
// fixed order.
template <typename real, int MG, int CH>
__global__ void __launch_bounds__(128) k_sk_partial(DevState<real> s, KArgs<real> a) {
  static_assert(CH % 16 == 0, "atom chunk in whole groups of 16");
  using c2 = typename R2<real>::t;
  extern __shared__ unsigned char smem_raw[];
  const int ngroups = (a.M + MG - 1) / MG;
  const int rw = 2 * a.kp + ngroups * MG;
  c2 *tab = reinterpret_cast<c2 *>(smem_raw);          // [CH][rw]
  real *q = reinterpret_cast<real *>(tab + rw * CH);  // [CH]
  if (*s.err) return;
  const int a0 = blockIdx.y * CH;
  const int na = min(CH, s.n - a0);
  // staging: SB loads in flight per thread before their stores
  constexpr int SB = 8;
  for (int e0 = threadIdx.x; e0 < rw * CH; e0 += SB * blockDim.x) {
    c2 v[SB];
#pragma unroll
    for (int u = 0; u < SB; ++u) {
      const int e = e0 + u * blockDim.x;
      const int row = e / CH, at = e - row * CH;
      const int d = min(row / a.kp, 2), m = row - d * a.kp;
      v[u].x = 0;
      v[u].y = 0;
      if (e < rw * CH && at < na && m <= a.kmax[d]) v[u] = a.ptab[(size_t)(d * a.kp + m) * s.n + a0 + at];
    }
#pragma unroll
    for (int u = 0; u < SB; ++u) {
      const int e = e0 + u * blockDim.x;
      const int row = e / CH, at = e - row * CH;
      if (e < rw * CH) tab[at * rw + row] = v[u];
    }
  }
  for (int t = threadIdx.x; t < CH; t += blockDim.x) q[t] = (t < na) ? (real)a.charge[s.type[a0 + t]] : (real)0;
  __syncthreads();
  const int task = blockIdx.x * blockDim.x + threadIdx.x;
  if (task >= ngroups * a.ncomp) return;
  const int g = task / a.ncomp, col = task - g * a.ncomp;  // a summed column
  const int2 nn = a.xyc[col];
  const int ox = abs(nn.x), oy = a.kp + abs(nn.y), oz = 2 * a.kp + g * MG;
  const bool cx = nn.x < 0, cy = nn.y < 0;
  double tot[MG][4];
#pragma unroll
  for (int u = 0; u < MG; ++u) tot[u][0] = tot[u][1] = tot[u][2] = tot[u][3] = 0.0;
  for (int t0 = 0; t0 < na; t0 += 16) {
    real acc[MG][4];
#pragma unroll
    for (int u = 0; u < MG; ++u) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = (real)0;
    const c2 *ta = tab + t0 * rw;
#pragma unroll 4
    for (int t = 0; t < 16; ++t, ta += rw) {
      c2 w = cmul(conj_if(ta[ox], cx), conj_if(ta[oy], cy));
      const real qt = q[t0 + t];
      w.x *= qt;
      w.y *= qt;
#pragma unroll
      for (int u = 0; u < MG; ++u) {
        const c2 z = ta[oz + u];
        // S(+m) += w z, S(-m) += w conj(z)
        acc[u][0] += w.x * z.x;
        acc[u][0] -= w.y * z.y;
        acc[u][1] += w.x * z.y;
        acc[u][1] += w.y * z.x;
        acc[u][2] += w.x * z.x;
        acc[u][2] += w.y * z.y;
        acc[u][3] += w.y * z.x;
        acc[u][3] -= w.x * z.y;
      }
    }
#pragma unroll
    for (int u = 0; u < MG; ++u)
#pragma unroll
      for (int c = 0; c < 4; ++c) tot[u][c] += (double)acc[u][c];
  }
#pragma unroll
  for (int u = 0; u < MG; ++u) {
    if (g * MG + u < a.M) {
      const size_t idx = ((size_t)blockIdx.y * a.M + g * MG + u) * a.ncomp + col;
      a.partial[2 * idx] = make_double2(tot[u][0], tot[u][1]);
      a.partial[2 * idx + 1] = make_double2(tot[u][2], tot[u][3]);
    }
  }
}

// S(k) = sum of the chunk partials (warps 1 .. RW-1: warp w adds chunks
// w - 1, w - 1 + (RW - 1), ... in order, four loads in flight, while warp 0
// fetches the k indices and f_k; then warp 0 adds the RW - 1 sums in warp
// order: a fixed order, deterministic), one lane per (column, m) pair.
// A column taken from its mirror reads the mirror's sums and conjugates
// them with +m and -m swapped (exact).
// Writes S(k), the FP64 k-space energy partials sum_k f_k |S_k|^2, and the
// force coefficients of the pair: with A_k = (4 pi / V) f_k conj(S_k) =
// a + ib at +m and c + id at -m, kcoef = (a+c, d-b, b+d, a-c) and the same
// times m.
template <typename real, int RW>
__global__ void __launch_bounds__(RW * 32) k_sk_reduce(DevState<real> s, KArgs<real> a) {
  __shared__ double part[RW][4][32];
  if (*s.err) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int np = a.M * a.nxy, npc = a.M * a.ncomp;
  const int p = blockIdx.x * 32 + lane;
  const int pm = p / a.nxy, pcol = p - pm * a.nxy;  // (m, column) of this lane
  const int src = (p < np) ? a.ksrc[pcol] : 0;
  const int pc = pm * a.ncomp + (src & ((1 << 30) - 1));  // its summed (m, column)
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  // warp 0 fetches the lane's k indices, its mirror's and their f_k while
  // warps 1 .. RW-1 sum the chunks (the two latency chains overlap)
  int2 kk = make_int2(-1, -1), mk = make_int2(-1, -1);
  double fe[2] = {0.0, 0.0}, fc[2] = {0.0, 0.0};  // f_k of (+-m); coefficient f_k x weight
  if (w == 0 && p < np) {
    kk = a.kpm[p];
    if (!(src >> 30)) {
      const int mir = a.kmir[src];
      if (mir >= 0) mk = a.kpm[(size_t)pm * a.nxy + mir];
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      // k and its mirror -k (in the column taken from this one) give the same
      // force term: the coefficient of (column, +-m) counts whichever of the two are in the set
      const int k = h ? kk.y : kk.x, km = h ? mk.x : mk.y;
      const int kf = (k >= 0) ? k : km;
      if (kf >= 0) {
        const double f = a.fk[kf];
        if (k >= 0) fe[h] = f;
        fc[h] = f * ((k >= 0 ? 1.0 : 0.0) + (km >= 0 ? 1.0 : 0.0));
      }
    }
  }
  if (p < np && w > 0) {
    for (int c0 = w - 1; c0 < a.nchunks; c0 += 4 * (RW - 1)) {
      double2 u[4][2];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const int c = c0 + h * (RW - 1);
        const size_t idx = (size_t)min(c, a.nchunks - 1) * npc + pc;
        u[h][0] = a.partial[2 * idx];
        u[h][1] = a.partial[2 * idx + 1];
      }
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        if (c0 + h * (RW - 1) < a.nchunks) {
          v[0] += u[h][0].x;
          v[1] += u[h][0].y;
          v[2] += u[h][1].x;
          v[3] += u[h][1].y;
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) part[w][c][lane] = v[c];
  __syncthreads();
  double e = 0;
  if (w == 0 && p < np) {
    double S[4] = {0.0, 0.0, 0.0, 0.0};
    for (int ww = 0; ww < RW; ++ww)
#pragma unroll
      for (int c = 0; c < 4; ++c) S[c] += part[ww][c][lane];
    if (src >> 30) {  // the mirror's sums: S(+m) = conj(S'(-m)), S(-m) = conj(S'(+m))
      const double t0 = S[0], t1 = S[1];
      S[0] = S[2];
      S[1] = -S[3];
      S[2] = t0;
      S[3] = -t1;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = h ? kk.y : kk.x;
      if (k >= 0) {
        const double sr = S[2 * h], si = S[2 * h + 1];
        a.sk[k] = make_double2(sr, si);
        e += fe[h] * (sr * sr + si * si);
      }
    }
    if (!(src >> 30)) {  // force coefficients of a summed column
      const int m = pm, col = src;  // col: the summed column's index
      double A[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const double cf = a.four_pi_over_v * fc[h];
        A[2 * h] = cf * S[2 * h];
        A[2 * h + 1] = -cf * S[2 * h + 1];
      }
      const double c4[4] = {A[0] + A[2], A[3] - A[1], A[1] + A[3], A[0] - A[2]};
      real *o = a.kcoef + ((size_t)col * a.M + m) * 8;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        o[c] = (real)c4[c];
        o[4 + c] = (real)(m * c4[c]);
      }
      if (a.kimg) {
        // B rows of this column for k = 2m, 2m + 1: Cx (q0, q1), Cy (q2, q3),
        // Dx (q7, -q6), Dy (-q5, q4) with q4..q7 = m q0..q3 (see kf_term)
        float *hi = a.kimg + (size_t)(col / KTC_COLS) * 2 * KTC_TILE_FLOATS, *lo = hi + KTC_TILE_FLOATS;
        const int rb = 4 * (col % KTC_COLS);
        const float v[4][2] = {{(float)c4[0], (float)c4[1]},
                               {(float)c4[2], (float)c4[3]},
                               {(float)(m * c4[3]), -(float)(m * c4[2])},
                               {-(float)(m * c4[1]), (float)(m * c4[0])}};
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int o2 = ktc_off(rb + r, 2 * m) / 4;
          const float h0 = to_tf32(v[r][0]), h1 = to_tf32(v[r][1]);
          *reinterpret_cast<float2 *>(hi + o2) = make_float2(h0, h1);
          *reinterpret_cast<float2 *>(lo + o2) = make_float2(to_tf32(v[r][0] - h0), to_tf32(v[r][1] - h1));
        }
      }
    }
  }
  double ev[1] = {e};
  block_sum_store<1>(ev, a.e_partials);
}

// Eight force coefficients of one (column, m) pair: two 16-byte loads (float)
// or four (double), uniform across the warp.
__device__ __forceinline__ void load8(const float *p, float (&r)[8]) {
  const float4 u = __ldg(reinterpret_cast<const float4 *>(p)), v = __ldg(reinterpret_cast<const float4 *>(p) + 1);
  r[0] = u.x; r[1] = u.y; r[2] = u.z; r[3] = u.w; r[4] = v.x; r[5] = v.y; r[6] = v.z; r[7] = v.w;
}
__device__ __forceinline__ void load8(const double *p, double (&r)[8]) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const double2 u = __ldg(q + h);
    r[2 * h] = u.x;
    r[2 * h + 1] = u.y;
  }
}

__device__ __forceinline__ void load8s(const float *p, float (&r)[8]) {
  const float4 u = reinterpret_cast<const float4 *>(p)[0], v = reinterpret_cast<const float4 *>(p)[1];
  r[0] = u.x; r[1] = u.y; r[2] = u.z; r[3] = u.w; r[4] = v.x; r[5] = v.y; r[6] = v.z; r[7] = v.w;
}
__device__ __forceinline__ void load8s(const double *p, double (&r)[8]) {
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const double2 u = reinterpret_cast<const double2 *>(p)[h];
    r[2 * h] = u.x;
    r[2 * h + 1] = u.y;
  }
}

// One (column, m) term of the k-force sums C and D (see k_kforce).
template <typename real>
__device__ __forceinline__ void kf_term(const real (&q)[8], real zx, real zy, real &Cx, real &Cy, real &Dx, real &Dy) {
  Cx += q[0] * zx;
  Cx += q[1] * zy;
  Cy += q[2] * zx;
  Cy += q[3] * zy;
  Dx += q[7] * zx;
  Dx -= q[6] * zy;
  Dy += q[4] * zy;
  Dy -= q[5] * zx;
}

// k-space force (electrostatic_ewald_k.cpp:215-218):
// F_i = k_e q_i sum_k k Im(A_k e^{i k.r_i}).  A block holds 32 atoms (one per
// lane) and W warps; warp w takes the w-th of W equal ranges of (nx, ny)
// columns, so a few thousand atoms still fill the GPU.  Each warp stages its
// columns' coefficients in shared memory, TC columns at a time, with
// 16-byte loads all in flight (one L2 round trip per tile), then reads them
// as broadcasts.  The 32 atoms' phase tables sit in shared memory
// (atom-major).  MZ = M (the number of m-values, exact, so the m-loop
// unrolls without guards) keeps Z[m] in registers; MZ = 0 reads it from
// shared memory for any M.  Per column: C = sum_m (A+ z + A- conj z),
// D = sum_m m (A+ z - A- conj z), then Im(P C) feeds F_x, F_y and Im(P D)
// feeds F_z, P = X[nx] Y[ny].  The W partial forces of an atom are added in
// warp order (deterministic).
// kick_h != 0: the step's second half kick follows in the epilogue (v +=
// kick_h a with the atom's final acceleration, as k_kick<real, false>, whose
// flag reset and step count block 0 also takes over).
template <typename real, int MZ>
__global__ void __launch_bounds__(512, sizeof(real) == 4 ? CVR_KF_MINB : 1) k_kforce(DevState<real> s, KArgs<real> a,
                                                                                  int TC, double kick_h,
                                                                                  long long *__restrict__ counters) {
  if (kick_h != 0.0 && blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    *s.flag = 0;
    if (counters) counters[0]++;
  }
  using c2 = typename R2<real>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x, w = threadIdx.y, W = blockDim.y;
  const int M = a.M, rw = 3 * a.kp;
  const int cw = M * 8;  // reals per column
  real *cfw = reinterpret_cast<real *>(smem_raw) + (size_t)w * TC * cw;                  // [W][TC][M][8]
  int2 *xyw = reinterpret_cast<int2 *>(reinterpret_cast<real *>(smem_raw) + (size_t)W * TC * cw) + w * TC;
  c2 *tab = reinterpret_cast<c2 *>(reinterpret_cast<int2 *>(reinterpret_cast<real *>(smem_raw) + (size_t)W * TC * cw) +
                                   ((W * TC + 1) & ~1));                                  // [32][3 * kp]
  real *red = reinterpret_cast<real *>(tab + 32 * rw);                                     // [W][3][32]
  if (*s.err) return;
  const int i = blockIdx.x * 32 + lane;
  const bool valid = i < s.n;
  for (int row = w; row < rw; row += W) {
    const int d = row / a.kp, m = row - d * a.kp;
    c2 v;
    v.x = 0;
    v.y = 0;
    if (valid && m <= a.kmax[d]) v = a.ptab[(size_t)row * s.n + i];
    tab[lane * rw + row] = v;
  }
  __syncthreads();
  const c2 *ta = tab + lane * rw;
  real zx[MZ > 0 ? MZ : 1], zy[MZ > 0 ? MZ : 1];
  if (MZ > 0) {
#pragma unroll
    for (int m = 0; m < (MZ > 0 ? MZ : 1); ++m) {
      const c2 z = ta[2 * a.kp + m];
      zx[m] = z.x;
      zy[m] = z.y;
    }
  }
  // the summed columns only: a column taken from its mirror adds the same
  // force, which k_sk_reduce has folded into the summed column's coefficients
  const int c0 = (int)(((long)w * a.ncomp) / W), c1 = (int)(((long)(w + 1) * a.ncomp) / W);
  real fx = 0, fy = 0, fz = 0;
  for (int cb = c0; cb < c1; cb += TC) {
    const int nt = min(TC, c1 - cb);
    __syncwarp();
    {
      constexpr int SB = CVR_KF_SB;
      const int nv = nt * cw * (int)sizeof(real) / 16;
      const uint4 *src = reinterpret_cast<const uint4 *>(a.kcoef + (size_t)cb * cw);
      uint4 *dst = reinterpret_cast<uint4 *>(cfw);
      for (int v0 = lane; v0 < nv; v0 += SB * 32) {
        uint4 r[SB];
#pragma unroll
        for (int u = 0; u < SB; ++u)
          if (v0 + u * 32 < nv) r[u] = __ldg(src + v0 + u * 32);
#pragma unroll
        for (int u = 0; u < SB; ++u)
          if (v0 + u * 32 < nv) dst[v0 + u * 32] = r[u];
      }
      for (int c = lane; c < nt; c += 32) xyw[c] = a.xyc[cb + c];
    }
    __syncwarp();
    for (int c = 0; c < nt; ++c) {
      const int2 nn = xyw[c];
      const c2 P = cmul(conj_if(ta[abs(nn.x)], nn.x < 0), conj_if(ta[a.kp + abs(nn.y)], nn.y < 0));
      const real *qc = cfw + (size_t)c * cw;
      real Cx = 0, Cy = 0, Dx = 0, Dy = 0;
      if (MZ > 0) {
#pragma unroll
        for (int m = 0; m < (MZ > 0 ? MZ : 1); ++m) {
          real q[8];
          load8s(qc + m * 8, q);
          kf_term(q, zx[m], zy[m], Cx, Cy, Dx, Dy);
        }
      } else {
#pragma unroll 3
        for (int m = 0; m < M; ++m) {
          real q[8];
          load8s(qc + m * 8, q);
          const c2 z = ta[2 * a.kp + m];
          kf_term(q, z.x, z.y, Cx, Cy, Dx, Dy);
        }
      }
      const real t = P.x * Cy + P.y * Cx;
      fx += (real)nn.x * t;
      fy += (real)nn.y * t;
      fz += P.x * Dy + P.y * Dx;
    }
  }
  real *r = red + w * 3 * 32 + lane;
  r[0] = fx;
  r[32] = fy;
  r[64] = fz;
  __syncthreads();
  if (w != 0 || !valid) return;
  fx = fy = fz = 0;
  for (int ww = 0; ww < W; ++ww) {
    fx += red[ww * 96 + lane];
    fy += red[ww * 96 + 32 + lane];
    fz += red[ww * 96 + 64 + lane];
  }
  const int ti = s.type[i];
  const real qm = (real)(a.k_e * a.charge[ti] * s.mass_inv[ti]);
  s.ax[i] += qm * a.two_pi_over_L[0] * fx;
  s.ay[i] += qm * a.two_pi_over_L[1] * fy;
  s.az[i] += qm * a.two_pi_over_L[2] * fz;
  if (kick_h != 0.0) {
    s.vx[i] = s.vx[i] + kick_h * (double)s.ax[i];
    s.vy[i] = s.vy[i] + kick_h * (double)s.ay[i];
    s.vz[i] = s.vz[i] + kick_h * (double)s.az[i];
  }
}

// ------------------------------------------------------------- integrator
// Velocity Verlet as kick (v += dt/2 a), drift (r += dt v), force, kick:
// algebraically the reference's r += v dt + a dt^2/2, v += dt/2 (a + a_old)
// (md_simulator.cpp:591-616) without storing a_old.  The first half also
// writes the cell-local coordinates for the pair kernel and raises the
// rebuild flag (neighborlist.cpp:91-139 / md_simulator.cpp:487-502).
// After a position update of atom i (cell order) to p: the cell-local
// coordinates for the pair kernel, and whether the list must be rebuilt.
template <typename real>
__device__ __forceinline__ bool update_local(DevState<real> &s, int i, const double (&p)[3]) {
  bool need = false;
  int code = 0, mul = 1;
  if (s.policy == 1) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (s.box.bc[d] == 1 && (p[d] < s.box.lo[d] || p[d] > s.box.hi[d])) need = true;  // owned wrap
      code += (ghost_val(p[d], s.box.gclo[d], s.box.gchi[d], s.box.bc[d]) + 1) * mul;
      mul *= 3;
    }
  }
  typename V4<real>::t q;
  bool fx = false;
  if constexpr (sizeof(real) == 4) {
    if (s.fixed) {  // fixed point: no cell frame, the type from the type array
      q.x = fixed_coord(p[0], s.fx_scale);
      q.y = fixed_coord(p[1], s.fx_scale);
      q.z = fixed_coord(p[2], s.fx_scale);
      q.w = __int_as_float(s.type[i]);
      fx = true;
    }
  }
  if (!fx) {
    int cc[3];
    cell_xyz(s, s.cell[i], cc[0], cc[1], cc[2]);
    q = s.x4[i];
    q.x = (real)(p[0] - (s.box.lo[0] + (cc[0] + 0.5) * s.cells.w[0]));
    q.y = (real)(p[1] - (s.box.lo[1] + (cc[1] + 0.5) * s.cells.w[1]));
    q.z = (real)(p[2] - (s.box.lo[2] + (cc[2] + 0.5) * s.cells.w[2]));
  }
  s.x4[i] = q;
  const float4 b = s.xb[i];
  const float ex = (float)(p[0] - s.box.ctr[0]) - b.x, ey = (float)(p[1] - s.box.ctr[1]) - b.y,
              ez = (float)(p[2] - s.box.ctr[2]) - b.z;
  if (ex * ex + ey * ey + ez * ez > s.thr_sq) need = true;
  if (s.policy == 1 && code != s.gcls[i]) need = true;  // ghost set changed
  if (s.policy == 2) need = true;
  return need;
}

#ifndef KD_PHASE_SUB
#define KD_PHASE_SUB 4
#endif
// PHASE: also the atom's S(k) phase tables at the new position (the values
// k_phase writes), so the step's S(k) chain starts at the chunk partials.
// pre_h != 0: the previous step's second half kick (v += pre_h a, deferred
// from that step, as k_kick computes it) comes first; the two half kicks
// use the same acceleration, so this is the kick + kick-drift sequence
// operation for operation.
template <typename real, bool PHASE>
__global__ void __launch_bounds__(256) k_kick_drift(DevState<real> s, double dt, KArgs<real> ka, double pre_h) {
  // PHASE: KD_PHASE_SUB neighbouring lanes per atom; each computes the
  // atom's update (same loads, merged by the coalescer; same result), the
  // first stores it, and the first three write one axis's phase row each
  constexpr int SUB = PHASE ? KD_PHASE_SUB : 1;
  static_assert(SUB >= 3 || !PHASE, "one lane per axis for the phase rows");
  if (*s.err) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / SUB, sub = t - i * SUB;
  bool need = false;
  if (i < s.n) {
    const double a0 = (double)s.ax[i], a1 = (double)s.ay[i], a2 = (double)s.az[i];
    const double h = 0.5 * dt;
    double u0 = s.vx[i], u1 = s.vy[i], u2 = s.vz[i];
    if (pre_h != 0.0) {
      u0 = u0 + pre_h * a0;
      u1 = u1 + pre_h * a1;
      u2 = u2 + pre_h * a2;
    }
    const double v0 = u0 + h * a0, v1 = u1 + h * a1, v2 = u2 + h * a2;
    const double p[3] = {s.x[i] + dt * v0, s.y[i] + dt * v1, s.z[i] + dt * v2};
    if (sub == 0) {
      if (isnan(a0) || isnan(a1) || isnan(a2)) atomicOr(s.err, ERR_NAN);  // md_simulator.cpp:584-590
      s.vx[i] = v0;
      s.vy[i] = v1;
      s.vz[i] = v2;
      s.x[i] = p[0];
      s.y[i] = p[1];
      s.z[i] = p[2];
      need = update_local(s, i, p);
    }
    if constexpr (PHASE) {
      if (sub < 3) {
        const double pd = (sub == 0) ? p[0] : ((sub == 1) ? p[1] : p[2]);  // static indices: p stays in registers
        phase_row<real>(ka.ptab, s.n, i, sub * ka.kp, pd * ka.inv_L[sub], ka.kmax[sub]);
      }
    }
  }
  if (__any_sync(0xffffffffu, need) && (threadIdx.x & 31) == 0) *s.flag = 1;
}

// ------------------------------------------------------ Langevin (GJF-type)
// The reference's velocity_verlet_langevin (md_simulator.cpp:670-811), per
// step with one Gaussian vector eta per atom:
//   v += dt/2 a + b eta;  r += c v;  forces;  v = a_c v + b eta + dt/2 a
// with a_c = (2 - g dt)/(2 + g dt), b = sqrt(kT g dt/2), c = 2 dt/(2 + g dt)
// (md_simulator.cpp:333-344).  eta is read from (or, with the counter-based
// generator, written to) `eta`, SoA [3][n] in the caller's atom order.

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): ten rounds of two 32x32 -> 64 multiplies with a
// Weyl-sequence key schedule; counter = (atom id, step low, step high, 0),
// key = seed.  Box-Muller turns the four 32-bit words into normals.
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * ctr.x, hi0 = __umulhi(0xD2511F53u, ctr.x);
    const uint32_t lo1 = 0xCD9E8D57u * ctr.z, hi1 = __umulhi(0xCD9E8D57u, ctr.z);
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += 0x9E3779B9u;
    key.y += 0xBB67AE85u;
  }
  return ctr;
}

__device__ __forceinline__ void philox_normals(uint64_t seed, long long step, int id, double g[3]) {
  const uint4 r = philox4x32_10(make_uint4((uint32_t)id, (uint32_t)step, (uint32_t)((unsigned long long)step >> 32), 0u),
                                make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  const double k = 2.3283064365386963e-10;  // 2^-32: uniforms in (0, 1)
  const double u0 = ((double)r.x + 0.5) * k, u1 = ((double)r.y + 0.5) * k;
  const double u2 = ((double)r.z + 0.5) * k, u3 = ((double)r.w + 0.5) * k;
  const double r0 = sqrt(-2.0 * log(u0)), r1 = sqrt(-2.0 * log(u2));
  double s0, c0, s1, c1;
  sincospi(2.0 * u1, &s0, &c0);
  sincospi(2.0 * u3, &s1, &c1);
  g[0] = r0 * c0;
  g[1] = r0 * s0;
  g[2] = r1 * c1;
}

struct LangevinArgs {
  double a, b, c;
  double *eta;             // [3][n], the caller's atom order
  int generate;            // 1: draw eta on the device (counter-based), 0: read the host-made eta
  uint64_t seed;
  const long long *step;   // counters[0]: steps done so far
};

template <typename real>
__global__ void __launch_bounds__(256) k_lgv_kick_drift(DevState<real> s, double dt, LangevinArgs lg) {
  if (*s.err) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool need = false;
  if (i < s.n) {
    const int id = s.id[i];
    double eta[3];
    if (lg.generate) {
      philox_normals(lg.seed, *lg.step, id, eta);
      lg.eta[id] = eta[0];
      lg.eta[s.n + id] = eta[1];
      lg.eta[2 * s.n + id] = eta[2];
    } else {
      eta[0] = lg.eta[id];
      eta[1] = lg.eta[s.n + id];
      eta[2] = lg.eta[2 * s.n + id];
    }
    const double a0 = (double)s.ax[i], a1 = (double)s.ay[i], a2 = (double)s.az[i];
    if (isnan(a0) || isnan(a1) || isnan(a2)) atomicOr(s.err, ERR_NAN);  // md_simulator.cpp:707-713
    // vel += 0.5 * acc * dt + b * eta (md_simulator.cpp:717); pos += vel * c (:764)
    const double v0 = s.vx[i] + (0.5 * a0 * dt + lg.b * eta[0]);
    const double v1 = s.vy[i] + (0.5 * a1 * dt + lg.b * eta[1]);
    const double v2 = s.vz[i] + (0.5 * a2 * dt + lg.b * eta[2]);
    const double p[3] = {s.x[i] + v0 * lg.c, s.y[i] + v1 * lg.c, s.z[i] + v2 * lg.c};
    s.vx[i] = v0;
    s.vy[i] = v1;
    s.vz[i] = v2;
    s.x[i] = p[0];
    s.y[i] = p[1];
    s.z[i] = p[2];
    need = update_local(s, i, p);
  }
  if (__any_sync(0xffffffffu, need) && (threadIdx.x & 31) == 0) *s.flag = 1;
}

// vel = a vel + b eta + 0.5 acc dt (md_simulator.cpp:790); KE partials, flag
// and step counter as k_kick.
template <typename real, bool KE>
__global__ void __launch_bounds__(256) k_lgv_kick(DevState<real> s, double dt, LangevinArgs lg,
                                                  double *__restrict__ partials, long long *__restrict__ counters) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *s.flag = 0;
    if (counters) counters[0]++;
  }
  if (*s.err) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (i < s.n) {
    const int id = s.id[i];
    const double v0 = lg.a * s.vx[i] + lg.b * lg.eta[id] + 0.5 * (double)s.ax[i] * dt;
    const double v1 = lg.a * s.vy[i] + lg.b * lg.eta[s.n + id] + 0.5 * (double)s.ay[i] * dt;
    const double v2 = lg.a * s.vz[i] + lg.b * lg.eta[2 * s.n + id] + 0.5 * (double)s.az[i] * dt;
    s.vx[i] = v0;
    s.vy[i] = v1;
    s.vz[i] = v2;
    if (KE) {
      const double m = s.mass[s.type[i]];
      v[0] = m * (v0 * v0 + v1 * v1 + v2 * v2);
      v[1] = m * v0;
      v[2] = m * v1;
      v[3] = m * v2;
    }
  }
  if (KE) block_sum_store<4>(v, partials);
}

// Second half kick; KE partials (sum m v^2, sum m v) when KE.  Also clears
// the step's rebuild flag (every reader of it has run by now) and counts the
// step in counters[0].
template <typename real, bool KE>
__global__ void __launch_bounds__(256) k_kick(DevState<real> s, double dt, double *__restrict__ partials,
                                              long long *__restrict__ counters) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *s.flag = 0;
    if (counters) counters[0]++;
  }
  if (*s.err) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (i < s.n) {
    const double h = 0.5 * dt;
    const double v0 = s.vx[i] + h * (double)s.ax[i];
    const double v1 = s.vy[i] + h * (double)s.ay[i];
    const double v2 = s.vz[i] + h * (double)s.az[i];
    s.vx[i] = v0;
    s.vy[i] = v1;
    s.vz[i] = v2;
    if (KE) {
      const double m = s.mass[s.type[i]];
      v[0] = m * (v0 * v0 + v1 * v1 + v2 * v2);
      v[1] = m * v0;
      v[2] = m * v1;
      v[3] = m * v2;
    }
  }
  if (KE) block_sum_store<4>(v, partials);
}

// ------------------------------------------------------------ thermostats
// Applied after the velocity update of a velocity-Verlet step, where the
// reference calls Constraint::apply_thermostat (md_simulator.cpp:619-627):
//   Berendsen (constraint/berendsen.cpp:100-131): every `step` steps,
//     v *= clamp(sqrt(1 + (dt/tau)(T0/T - 1)), lambda_min, lambda_max);
//   Nose-Hoover (constraint/nose_hoover.cpp:122-180): zeta += dt zeta_dot with
//     zeta_dot = (-kb n_df T / Q)(T0/T - 1) (type 1, mass Q) or (-1/tau)(T0/T - 1)
//     (type 2), then a -= zeta v (the next step's drift and first kick use it).
// T is the step's instantaneous temperature, 2 KE / (k_b n_df), KE with the
// centre-of-mass motion removed as for the thermo record.
struct ThermostatArgs {
  int kind;  // 1 Berendsen, 2 Nose-Hoover
  double T0, dt, tau, lambda_min, lambda_max;  // Berendsen: tau = coupling
  int every;
  int nh_type;
  double nh_mass, nh_tau, nh_kb;
  double total_mass, dof, k_b;
  int com_removed;
  const double *ke_part;
  int n_ke;
  const long long *counters;  // [0]: steps done, including this one
  double *scal;               // [0] Berendsen factor of this step (1 = none), [1] zeta
};

__global__ void __launch_bounds__(256) k_thermostat_coef(ThermostatArgs a) {
  __shared__ double acc[4][256];
  double v[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < a.n_ke; b += blockDim.x)
    for (int q = 0; q < 4; ++q) v[q] += a.ke_part[(size_t)b * 4 + q];
  for (int q = 0; q < 4; ++q) acc[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int q = 0; q < 4; ++q) acc[q][threadIdx.x] += acc[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double ke = 0.5 * acc[0][0];
  if (a.com_removed && a.total_mass > 0)
    ke -= 0.5 * (acc[1][0] * acc[1][0] + acc[2][0] * acc[2][0] + acc[3][0] * acc[3][0]) / a.total_mass;
  const double T = (a.dof > 0) ? 2.0 * ke / (a.k_b * a.dof) : 0.0;
  const long long timestep = a.counters[0] - 1;  // the reference's current_step of this step
  if (a.kind == 1) {
    double lam = 1.0;
    if (timestep % a.every == 0) {
      lam = sqrt(1.0 + (a.dt / a.tau) * ((a.T0 / T) - 1.0));
      if (lam < a.lambda_min) lam = a.lambda_min;
      if (lam > a.lambda_max) lam = a.lambda_max;
    }
    a.scal[0] = lam;
  } else {
    const double g = a.dof;
    double zd;
    if (a.nh_type == 1)
      zd = (-a.nh_kb * a.dof * T / a.nh_mass) * ((g * a.T0 / (a.dof * T)) - 1.0);
    else
      zd = (-1.0 / a.nh_tau) * ((g * a.T0 / (a.dof * T)) - 1.0);
    a.scal[1] += a.dt * zd;  // Euler step of zeta
  }
}

// Berendsen: v *= lambda (with KE partials of the scaled velocities for the
// thermo record); Nose-Hoover: a -= zeta v.
template <typename real, bool KE>
__global__ void __launch_bounds__(256) k_thermostat_apply(DevState<real> s, int kind, const double *__restrict__ scal,
                                                          double *__restrict__ partials) {
  if (*s.err) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (i < s.n) {
    if (kind == 1) {
      const double lam = scal[0];
      const double v0 = s.vx[i] * lam, v1 = s.vy[i] * lam, v2 = s.vz[i] * lam;
      s.vx[i] = v0;
      s.vy[i] = v1;
      s.vz[i] = v2;
      if (KE) {
        const double m = s.mass[s.type[i]];
        v[0] = m * (v0 * v0 + v1 * v1 + v2 * v2);
        v[1] = m * v0;
        v[2] = m * v1;
        v[3] = m * v2;
      }
    } else {
      const double z = scal[1];
      s.ax[i] = (real)((double)s.ax[i] - z * s.vx[i]);
      s.ay[i] = (real)((double)s.ay[i] - z * s.vy[i]);
      s.az[i] = (real)((double)s.az[i] - z * s.vz[i]);
    }
  }
  if (KE && kind == 1) block_sum_store<4>(v, partials);
}

// ---------------------------------------------------- Ewald dipole term
// The surrounding-medium term of Electrostatic_ewald_k (initialize.cpp:98-115,
// electrostatic_ewald_k.cpp:219-223): M = sum_j q_j r_j over the wrapped
// positions, E = -M k_e 4 pi / (V (1 + 2 eps')), F_i += mult q_i E.  The
// reference adds the term inside its k-vector loop, once per k-vector
// (mult = n_k); mult = 1 gives the textbook term.
template <typename real>
__global__ void __launch_bounds__(256) k_dipole_partial(DevState<real> s, const double *__restrict__ charge,
                                                        double *__restrict__ partials) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[3] = {0, 0, 0};
  if (i < s.n) {
    const double q = charge[s.type[i]];
    const double p[3] = {s.x[i], s.y[i], s.z[i]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double x = p[d];
      if (s.box.bc[d] == 1) x -= s.box.L[d] * floor((x - s.box.lo[d]) / s.box.L[d]);
      v[d] = q * x;
    }
  }
  block_sum_store<3>(v, partials);
}

// One block: M from the partials, E = -coef M into dip[0..2], M into dip[3..5].
__global__ void __launch_bounds__(256) k_dipole_field(const double *__restrict__ partials, int nparts, double coef,
                                                      double *__restrict__ dip) {
  __shared__ double acc[3][256];
  double v[3] = {0, 0, 0};
  for (int b = threadIdx.x; b < nparts; b += blockDim.x)
    for (int q = 0; q < 3; ++q) v[q] += partials[(size_t)b * 3 + q];
  for (int q = 0; q < 3; ++q) acc[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int q = 0; q < 3; ++q) acc[q][threadIdx.x] += acc[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 3) {
    dip[3 + threadIdx.x] = acc[threadIdx.x][0];
    dip[threadIdx.x] = -acc[threadIdx.x][0] * coef;
  }
}

template <typename real>
__global__ void __launch_bounds__(256) k_dipole_apply(DevState<real> s, const double *__restrict__ charge,
                                                      const double *__restrict__ dip, double mult) {
  if (*s.err) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const int t = s.type[i];
  const double f = mult * charge[t] * s.mass_inv[t];
  s.ax[i] = (real)((double)s.ax[i] + f * dip[0]);
  s.ay[i] = (real)((double)s.ay[i] + f * dip[1]);
  s.az[i] = (real)((double)s.az[i] + f * dip[2]);
}

// ------------------------------------------- Ewald slab correction (ELC)
// force_field electrostatic_ewald_slab_correction (electrostatic_ewald_slab_
// correction/initialize.cpp:33-255, field.cpp:27-144, energy.cpp:33-111), FP64.
// Slab-local coordinates (x, y in the periodic plane, z along the normal
// axis); wave numbers kx_i = 2 pi (i+1)/lx, ky_j = 2 pi (j+1)/ly,
// kp_ij = |(kx_i, ky_j)| with weights 1/(k (exp(k lz) - 1)); per k the charge
// sums chi of sinh/cosh(k z) times sin/cos of the in-plane phases; the field
// on atom i is their derivative combination, times 2 (-4 pi/(lx ly)) k_e,
// plus the dipole term -M k_e 4 pi/(lx ly lz) along the normal axis, where M
// is the normal dipole moment of the PREVIOUS force call (the reference
// computes the field before it updates its stored moment).
constexpr int SLAB_KMAX = 8;
constexpr int SLAB_CH = 32;  // atoms per chunk of the chi sums

struct SlabArgs {
  int axis, kx, ky, nv, nch;
  double lx, ly, lz, ke, sum_e_coef, dipole_coef;
  double kxv[SLAB_KMAX], kyv[SLAB_KMAX], kxc[SLAB_KMAX], kyc[SLAB_KMAX];
  double kpv[SLAB_KMAX * SLAB_KMAX], kpc[SLAB_KMAX * SLAB_KMAX];
  const double *charge;
  double *partial;  // [chunk][nv]
  double *chi;      // [nv]: x-terms 4 kx, y-terms 4 ky, p-terms 8 kx ky, then M
  double *state;    // [0] M of the previous call, [1] this call's slab energy
};

template <typename real>
__device__ __forceinline__ void slab_local(const DevState<real> &s, int axis, int i, double p[3]) {
  const double g[3] = {s.x[i], s.y[i], s.z[i]};
  // give_slab_local_coordinates (electrostatic_ewald_slab_correction.h)
  const int lx = axis == 0 ? 1 : (axis == 1 ? 2 : 0), ly = axis == 0 ? 2 : (axis == 1 ? 0 : 1);
  p[0] = g[lx];
  p[1] = g[ly];
  p[2] = g[axis];
}

// chi partial sums of one chunk: block = chunk, threads over the nv values.
template <typename real>
__global__ void __launch_bounds__(128) k_slab_chi_partial(DevState<real> s, SlabArgs a) {
  const int a0 = blockIdx.x * SLAB_CH, a1 = min(s.n, a0 + SLAB_CH);
  const int KX = a.kx, KY = a.ky;
  for (int v = threadIdx.x; v < a.nv; v += blockDim.x) {
    double acc = 0.0;
    for (int i = a0; i < a1; ++i) {
      const double q = a.charge[s.type[i]];
      double p[3];
      slab_local(s, a.axis, i, p);
      double t;
      if (v < 4 * KX) {
        const int ix = v >> 2, c = v & 3;
        const double kx = a.kxv[ix];
        const double h = (c >> 1) ? cosh(kx * p[2]) : sinh(kx * p[2]);
        const double f = (c & 1) ? cos(kx * p[0]) : sin(kx * p[0]);
        t = q * h * f;
      } else if (v < 4 * KX + 4 * KY) {
        const int iy = (v - 4 * KX) >> 2, c = (v - 4 * KX) & 3;
        const double ky = a.kyv[iy];
        const double h = (c >> 1) ? cosh(ky * p[2]) : sinh(ky * p[2]);
        const double f = (c & 1) ? cos(ky * p[1]) : sin(ky * p[1]);
        t = q * h * f;
      } else if (v < 4 * KX + 4 * KY + 8 * KX * KY) {
        const int w = v - 4 * KX - 4 * KY, ip = w >> 3, c = w & 7;  // c = 4 h + 2 a + b
        const int ix = ip / KY, iy = ip % KY;
        const double kp = a.kpv[ip];
        const double h = (c >> 2) ? cosh(kp * p[2]) : sinh(kp * p[2]);
        const double fx = ((c >> 1) & 1) ? cos(a.kxv[ix] * p[0]) : sin(a.kxv[ix] * p[0]);
        const double fy = (c & 1) ? cos(a.kyv[iy] * p[1]) : sin(a.kyv[iy] * p[1]);
        t = q * h * fx * fy;
      } else {
        t = q * p[2];  // normal dipole moment
      }
      acc += t;
    }
    a.partial[(size_t)blockIdx.x * a.nv + v] = acc;
  }
}

// chi = sum of the chunk partials (fixed order); slab energy (energy.cpp:33-111).
__global__ void __launch_bounds__(256) k_slab_chi_reduce(SlabArgs a) {
  __shared__ double red[256];
  double e = 0.0;
  const int KX = a.kx, KY = a.ky;
  for (int v = threadIdx.x; v < a.nv; v += blockDim.x) {
    double c = 0.0;
    for (int ch = 0; ch < a.nch; ++ch) c += a.partial[(size_t)ch * a.nv + v];
    a.chi[v] = c;
    // sign of c^2 in the energy: + for the cosh terms, - for the sinh terms
    if (v < 4 * KX) {
      e += ((v & 3) >> 1 ? 1.0 : -1.0) * c * c * a.kxc[v >> 2];
    } else if (v < 4 * KX + 4 * KY) {
      const int w = v - 4 * KX;
      e += ((w & 3) >> 1 ? 1.0 : -1.0) * c * c * a.kyc[w >> 2];
    } else if (v < 4 * KX + 4 * KY + 8 * KX * KY) {
      const int w = v - 4 * KX - 4 * KY;
      e += ((w & 7) >> 2 ? 1.0 : -1.0) * c * c * 2.0 * a.kpc[w >> 3];
    }
  }
  red[threadIdx.x] = e;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double M = a.chi[a.nv - 1];
    a.state[1] = red[0] * a.ke * a.sum_e_coef + 0.5 * a.dipole_coef * M * M;
  }
}

// Field on each atom and its acceleration (field.cpp:27-144).
template <typename real>
__global__ void __launch_bounds__(128) k_slab_field(DevState<real> s, SlabArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n || *s.err) return;
  const int KX = a.kx, KY = a.ky;
  const double *cx_ = a.chi, *cy_ = a.chi + 4 * KX, *cp_ = a.chi + 4 * KX + 4 * KY;
  double p[3];
  slab_local(s, a.axis, i, p);
  double f[3] = {0, 0, 0};
  for (int ix = 0; ix < KX; ++ix) {
    const double kx = a.kxv[ix];
    const double sh = sinh(kx * p[2]), chh = cosh(kx * p[2]);
    double sxx, cxx;
    sincos(kx * p[0], &sxx, &cxx);
    const double *c = cx_ + 4 * ix;  // [h][f]: sinh-sin, sinh-cos, cosh-sin, cosh-cos
    f[0] += a.kxc[ix] * -kx * (-c[0] * cxx * sh + c[1] * sxx * sh + c[2] * cxx * chh - c[3] * sxx * chh);
    f[2] += a.kxc[ix] * -kx * (-c[0] * chh * sxx - c[1] * chh * cxx + c[2] * sh * sxx + c[3] * sh * cxx);
    for (int iy = 0; iy < KY; ++iy) {
      const int ip = ix * KY + iy;
      const double kp = a.kpv[ip], ky = a.kyv[iy];
      const double sp = sinh(kp * p[2]), cp = cosh(kp * p[2]);
      double syy, cyy;
      sincos(ky * p[1], &syy, &cyy);
      const double *q = cp_ + 8 * ip;  // [h][a][b]: h sinh/cosh, a sin/cos x, b sin/cos y
      const double gx = -kx * (-q[0] * cxx * sp * syy - q[1] * cxx * sp * cyy + q[2] * sxx * sp * syy +
                               q[4] * cxx * cp * syy + q[3] * sxx * sp * cyy + q[5] * cxx * cp * cyy -
                               q[6] * sxx * cp * syy - q[7] * sxx * cp * cyy);
      const double gy = -ky * (-q[0] * cyy * sp * sxx + q[1] * syy * sp * sxx - q[2] * cyy * sp * cxx +
                               q[4] * cyy * cp * sxx + q[3] * syy * sp * cxx - q[5] * syy * cp * sxx +
                               q[6] * cyy * cp * cxx - q[7] * syy * cp * cxx);
      const double gz = -kp * (-q[0] * cp * sxx * syy - q[1] * cp * sxx * cyy - q[2] * cp * cxx * syy +
                               q[4] * sp * sxx * syy - q[3] * cp * cxx * cyy + q[5] * sp * sxx * cyy +
                               q[6] * sp * cxx * syy + q[7] * sp * cxx * cyy);
      f[0] += 2.0 * a.kpc[ip] * gx;
      f[1] += 2.0 * a.kpc[ip] * gy;
      f[2] += 2.0 * a.kpc[ip] * gz;
      if (ix == 0) {
        const double shy = sinh(ky * p[2]), chy = cosh(ky * p[2]);
        const double *y = cy_ + 4 * iy;
        f[1] += a.kyc[iy] * -ky * (-y[0] * cyy * shy + y[1] * syy * shy + y[2] * cyy * chy - y[3] * syy * chy);
        f[2] += a.kyc[iy] * -ky * (-y[0] * syy * chy - y[1] * cyy * chy + y[2] * syy * shy + y[3] * cyy * shy);
      }
    }
  }
  const double sc = 2.0 * a.sum_e_coef * a.ke;
  // back to global axes as give_slab_global_coordinates does (for normal axes x
  // and y its rotation is not the inverse of the local one; kept for parity),
  // plus the lagged dipole field along the normal axis
  double g[3];
  if (a.axis == 0) {
    g[0] = sc * f[1];
    g[1] = sc * f[2];
    g[2] = sc * f[0];
  } else if (a.axis == 1) {
    g[0] = sc * f[2];
    g[1] = sc * f[0];
    g[2] = sc * f[1];
  } else {
    g[0] = sc * f[0];
    g[1] = sc * f[1];
    g[2] = sc * f[2];
  }
  g[a.axis] -= a.state[0] * a.dipole_coef;
  const int t = s.type[i];
  const double qm = a.charge[t] * s.mass_inv[t];
  s.ax[i] = (real)((double)s.ax[i] + qm * g[0]);
  s.ay[i] = (real)((double)s.ay[i] + qm * g[1]);
  s.az[i] = (real)((double)s.az[i] + qm * g[2]);
}

__global__ void k_slab_store_moment(SlabArgs a) { a.state[0] = a.chi[a.nv - 1]; }

// Sets the step graph's IF condition from the device rebuild flag: the list
// build nodes run only on steps that need them.
__global__ void k_set_rebuild_condition(const int *__restrict__ flag, cudaGraphConditionalHandle h) {
  cudaGraphSetConditional(h, (*flag != 0) ? 1u : 0u);
}

// KE partials without moving anything (thermo outside the step loop).
template <typename real>
__global__ void __launch_bounds__(256) k_ke(DevState<real> s, double *__restrict__ partials) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (i < s.n) {
    const double m = s.mass[s.type[i]];
    const double v0 = s.vx[i], v1 = s.vy[i], v2 = s.vz[i];
    v[0] = m * (v0 * v0 + v1 * v1 + v2 * v2);
    v[1] = m * v0;
    v[2] = m * v1;
    v[3] = m * v2;
  }
  block_sum_store<4>(v, partials);
}

// Rebuild check outside the step loop (cvr_build_neighbors with force = 0).
template <typename real>
__global__ void __launch_bounds__(256) k_check(DevState<real> s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool need = false;
  if (i < s.n) {
    int cc[3];
    cell_xyz(s, s.cell[i], cc[0], cc[1], cc[2]);
    const double p[3] = {s.x[i], s.y[i], s.z[i]};
    float e[3];
    int code = 0, mul = 1;
    const float4 b = s.xb[i];
    const float bb[3] = {b.x, b.y, b.z};
    for (int d = 0; d < 3; ++d) {
      e[d] = (float)(p[d] - s.box.ctr[d]) - bb[d];
      if (s.policy == 1) {
        if (s.box.bc[d] == 1 && (p[d] < s.box.lo[d] || p[d] > s.box.hi[d])) need = true;
        code += (ghost_val(p[d], s.box.gclo[d], s.box.gchi[d], s.box.bc[d]) + 1) * mul;
        mul *= 3;
      }
    }
    if (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] > s.thr_sq) need = true;
    if (s.policy == 1 && code != s.gcls[i]) need = true;
    if (s.policy == 2) need = true;
  }
  if (__any_sync(0xffffffffu, need) && (threadIdx.x & 31) == 0) *s.flag = 1;
}

// ------------------------------------------------------------------ thermo
struct ThermoArgs {
  const double *ke_part;
  int n_ke;
  const double *ev_part;
  int n_ev;
  const double *ek_part;
  int n_ek;
  double total_mass, dof, volume, k_b, n_atoms, ek_coef, e_self;
  const double *dipole;  // E, M of the dipole term (nullable)
  const double *slab_e;  // slab-correction energy of the last force call (nullable)
  double dipole_coef;    // k_e 4 pi / (V (1 + 2 eps')): energy 0.5 coef |M|^2 (energy.cpp:52-56)
  int com_removed;
  const int *n_builds;
  long long *counters;  // [0] steps done, [1] next thermo record
  double *out;          // base of the records, CVR_N_THERMO doubles each
};

// One block of THERMO_THREADS: each thread sums its strided share of the
// block partials (loops unrolled so that several loads are in flight), then
// warp shuffles and one warp finish the sums (a fixed order).
constexpr int THERMO_THREADS = 1024;
__global__ void __launch_bounds__(THERMO_THREADS) k_thermo(ThermoArgs a) {
  __shared__ double red[8][32];
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
  for (int b = threadIdx.x; b < a.n_ke; b += blockDim.x) {
    const double4 k = *reinterpret_cast<const double4 *>(a.ke_part + (size_t)b * 4);
    v[0] += k.x;
    v[1] += k.y;
    v[2] += k.z;
    v[3] += k.w;
  }
#pragma unroll 4
  for (int b = threadIdx.x; b < a.n_ev; b += blockDim.x)
    for (int q = 0; q < 3; ++q) v[4 + q] += a.ev_part[(size_t)b * 3 + q];
#pragma unroll 4
  for (int b = threadIdx.x; b < a.n_ek; b += blockDim.x) v[7] += a.ek_part[b];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (warp != 0) return;
  double acc[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    double x = (lane < nw) ? red[q][lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    acc[q] = x;
  }
  if (lane == 0) {
    const long long rec = a.counters[1]++;
    double *out = a.out + rec * 10;
    const double mv2 = acc[0];
    double ke = 0.5 * mv2;
    if (a.com_removed && a.total_mass > 0) {
      const double px = acc[1], py = acc[2], pz = acc[3];
      ke -= 0.5 * (px * px + py * py + pz * pz) / a.total_mass;
    }
    const double temp = (a.dof > 0) ? 2.0 * ke / (a.k_b * a.dof) : 0.0;
    const double vir = acc[6];
    out[0] = (double)a.counters[0];
    out[1] = ke;
    out[2] = temp;
    out[3] = acc[4];
    out[4] = acc[5];
    out[5] = a.ek_coef * acc[7];
    if (a.dipole) {
      const double *M = a.dipole + 3;
      out[5] += 0.5 * a.dipole_coef * (M[0] * M[0] + M[1] * M[1] + M[2] * M[2]);
    }
    if (a.slab_e) out[5] += *a.slab_e;
    out[6] = a.e_self;
    out[7] = vir;
    out[8] = a.n_atoms * a.k_b * temp / a.volume + vir / (3.0 * a.volume);
    out[9] = (double)(*a.n_builds);
  }
}

// Gather the cell-ordered state back to id order (AoS, host layout), with
// positions wrapped once per axis like Domain::fix_position.
template <typename real>
__global__ void k_gather_state(DevState<real> s, double *__restrict__ pos, double *__restrict__ vel,
                               double *__restrict__ acc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= s.n) return;
  const int o = s.id[k];
  double p[3] = {s.x[k], s.y[k], s.z[k]};
  for (int d = 0; d < 3; ++d)
    if (s.box.bc[d] == 1) {
      if (p[d] < s.box.lo[d])
        p[d] = __dadd_rn(p[d], s.box.L[d]);
      else if (p[d] > s.box.hi[d])
        p[d] = __dsub_rn(p[d], s.box.L[d]);
    }
  if (pos) {
    pos[3 * (size_t)o] = p[0];
    pos[3 * (size_t)o + 1] = p[1];
    pos[3 * (size_t)o + 2] = p[2];
  }
  if (vel) {
    vel[3 * (size_t)o] = s.vx[k];
    vel[3 * (size_t)o + 1] = s.vy[k];
    vel[3 * (size_t)o + 2] = s.vz[k];
  }
  if (acc) {
    acc[3 * (size_t)o] = (double)s.ax[k];
    acc[3 * (size_t)o + 1] = (double)s.ay[k];
    acc[3 * (size_t)o + 2] = (double)s.az[k];
  }
}

// Scatter the caller's AoS state (id order) into the SoA arrays.
// Atoms per type (and, in hist[MAX_TYPES], atoms whose type is out of
// [0, nt)) of the caller's type array: shared-memory counters per block,
// one global add per counter and block (integer sums: order-free).
__global__ void __launch_bounds__(256) k_type_hist(const int *__restrict__ type, int n, int nt,
                                                   unsigned long long *__restrict__ hist) {
  __shared__ unsigned int h[MAX_TYPES + 1];
  for (int t = threadIdx.x; t <= MAX_TYPES; t += blockDim.x) h[t] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned t = (unsigned)type[i];
    atomicAdd(&h[t < (unsigned)nt ? t : MAX_TYPES], 1u);
  }
  __syncthreads();
  for (int t = threadIdx.x; t <= MAX_TYPES; t += blockDim.x)
    if (h[t]) atomicAdd(&hist[t], (unsigned long long)h[t]);
}

template <typename real>
__global__ void k_scatter_state(DevState<real> s, const double *__restrict__ pos, const double *__restrict__ vel,
                                const int *__restrict__ typ, const int *__restrict__ mol) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  s.x[i] = pos[3 * (size_t)i];
  s.y[i] = pos[3 * (size_t)i + 1];
  s.z[i] = pos[3 * (size_t)i + 2];
  s.vx[i] = vel ? vel[3 * (size_t)i] : 0.0;
  s.vy[i] = vel ? vel[3 * (size_t)i + 1] : 0.0;
  s.vz[i] = vel ? vel[3 * (size_t)i + 2] : 0.0;
  s.type[i] = typ[i];
  s.mol[i] = mol ? mol[i] : -1;
  s.id[i] = i;
  s.ax[i] = 0;
  s.ay[i] = 0;
  s.az[i] = 0;
}

// Velocities in the caller's order (AoS) to the atoms' current places, by
// id: the state may have been reordered since the positions were placed.
template <typename real>
__global__ void k_place_velocities(DevState<real> s, const double *__restrict__ vel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const size_t k = 3 * (size_t)s.id[i];
  s.vx[i] = vel[k];
  s.vy[i] = vel[k + 1];
  s.vz[i] = vel[k + 2];
}

}  // namespace cvr
