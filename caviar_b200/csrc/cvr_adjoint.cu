// cvr_adjoint.cu -- gradient of a trajectory loss through velocity Verlet on
// the GPU: forces, their vector-Jacobian product (VJP) w.r.t. positions and
// force-field parameters, and a checkpointed reverse sweep.
//
// No reference counterpart: the reference has no gradients.  The forward
// follows the reference's force definitions (LJ with the linear force shift,
// lj.cpp:439-448; Ewald real space, electrostatic_ewald_r.cpp:196-198, here
// with an explicit cutoff; Ewald k space over the reference's k-set,
// initialize.cpp:184-222 and electrostatic_ewald_k.cpp:197-234; velocity
// Verlet, md_simulator.cpp:555-668) on one periodic cube under the minimum
// image (every cutoff <= L/2).
//
// Every force evaluation of a trajectory uses the same kernel (the energy
// form, with a zero weight where the energy is not wanted), so the segments
// the reverse sweep re-runs are bit-identical to the forward pass.
//
// Loss J = (1/M) sum_{t=1..M} U(r_t).  Reverse sweep over the state (r, v, a)
// with cotangents (Gr, Gv, Ga); for step t (r' = r_{t+1}):
//   Gr -= F(r')/M;  Ga += dt/2 Gv;  Gr += (dF/dr)^T (Ga/m);  theta_bar += (dF/dtheta)^T (Ga/m)
//   (Gr, Gv, Ga) <- (Gr, Gv + dt Gr, dt/2 Gv + dt^2/2 Gr)
// and finally the VJP at r_0 for a_0 = F(r_0)/m.  Positions and velocities
// are checkpointed every K steps; the reverse sweep re-runs each segment
// forward, keeping its K positions and forces.
//
// Kernels (real = float for the mixed form, double for FP64):
//   k_adj_tables   per atom and axis, e^{i 2 pi m x / L} for m = 0..k_max
//   k_adj_sk       species-resolved S_a(k) = sum_{i in a} e^{ik.r_i} and, for
//                  the VJP, T_a(k) = sum_{i in a} (k.u_i) e^{ik.r_i}, per atom
//                  chunk (FP32 sub-sums of 16 atoms, FP64 chunk sums)
//   k_adj_kreduce  chunks -> S, T; per-k energy and charge-gradient terms
//   k_adj_atom     one warp per atom: all pairs (minimum image) and all
//                  k-vectors -> F_i or w_i = sum_j K_ij (u_j - u_i) + k-space,
//                  and the FP64 parameter sums
//   k_adj_accum    deterministic FP64 sums of per-block partials
//   k_adj_drift / k_adj_kick / k_adj_rev_pre / k_adj_rev_post   FP64 state updates
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/caviar_b200.h"
#include "cvr_device.cuh"

namespace {

constexpr int NT = 2;         // types
constexpr int NTT = NT * NT;  // ordered type pairs
constexpr int KMAX_ADJ = 10;
constexpr int ATOM_WARPS = 8;  // warps (atoms) per block of k_adj_atom
constexpr int SK_CHUNK = 256;  // atoms per S(k) chunk
constexpr int SK_THREADS = 128;

// accumulator slots (FP64, device)
enum : int {
  A_ELJ = 0, A_EEW = 1, A_EK = 2,
  A_DE = 3,               // dU/deps raw, NTT ordered pairs
  A_DS = A_DE + NTT,      // dU/dsigma raw
  A_DQ = A_DS + NTT,      // dU/dq, NT
  A_VE = A_DQ + NT,       // VJP eps raw
  A_VS = A_VE + NTT,      // VJP sigma raw
  A_VQ = A_VS + NTT,      // VJP q
  A_N = A_VQ + NT
};

template <typename real> struct R2;
template <> struct R2<float> { using t = float2; };
template <> struct R2<double> { using t = double2; };

struct Params {
  int n, nt, kmax, kp, nk;
  double L, invL, V, rc_lj2, rc_r2, alpha, k_e, dt;
  double mass_inv[NT], charge[NT];
  double eps[NTT], sig[NTT];
  const int *type;
  const int4 *kn;
  const double *fk;
};

struct Map {
  int idx[16];
};

__device__ __forceinline__ void sincospi_a(float a, float *s, float *c) { sincospif(a, s, c); }
__device__ __forceinline__ void sincospi_a(double a, double *s, double *c) { sincospi(a, s, c); }

template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T2> __device__ __forceinline__ T2 conj_if(T2 a, bool c) {
  if (c) a.y = -a.y;
  return a;
}

// e^{i 2 pi m x / L}, m = 0..k_max, per atom and axis: tab[(i*3 + axis)*kp + m]
template <typename real>
__global__ void k_adj_tables(Params p, const double *__restrict__ X, typename R2<real>::t *__restrict__ tab) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.n * 3 * p.kp) return;
  const int m = t % p.kp, ax = (t / p.kp) % 3, i = t / (3 * p.kp);
  const double u = (double)m * (X[ax * p.n + i] * p.invL);
  real sn, cs;
  sincospi_a((real)(2.0 * (u - rint(u))), &sn, &cs);
  typename R2<real>::t v;
  v.x = cs;
  v.y = sn;
  tab[t] = v;
}

template <typename real>
__device__ __forceinline__ typename R2<real>::t atom_phase(const typename R2<real>::t *__restrict__ tb, int kp, int4 kn) {
  const auto cx = conj_if(tb[abs(kn.x)], kn.x < 0);
  const auto cy = conj_if(tb[kp + abs(kn.y)], kn.y < 0);
  const auto cz = conj_if(tb[2 * kp + abs(kn.z)], kn.z < 0);
  return cmul(cmul(cx, cy), cz);
}

// Species-resolved structure factors of one atom chunk (blockIdx.y):
// part[(chunk*nk + k)*NS + s], s = {S_0, S_1} or {S_0, S_1, T_0, T_1}.
template <typename real, bool VJP>
__global__ void __launch_bounds__(SK_THREADS) k_adj_sk(Params p, const typename R2<real>::t *__restrict__ tab,
                                                       const double *__restrict__ U, double2 *__restrict__ part) {
  constexpr int NS = VJP ? 2 * NT : NT;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= p.nk) return;
  const int a0 = blockIdx.y * SK_CHUNK, a1 = min(p.n, a0 + SK_CHUNK);
  const int4 kn = p.kn[k];
  const real kf = (real)(6.28318530717958647692 * p.invL);
  double2 acc[NS];
  typename R2<real>::t sub[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    acc[s] = make_double2(0, 0);
    sub[s].x = sub[s].y = (real)0;
  }
  for (int i = a0; i < a1; ++i) {
    const auto e = atom_phase<real>(tab + (size_t)i * 3 * p.kp, p.kp, kn);
    const int t = p.type[i];
    const bool t0 = (t == 0);
    if (t0) {
      sub[0].x += e.x;
      sub[0].y += e.y;
    } else {
      sub[1].x += e.x;
      sub[1].y += e.y;
    }
    if (VJP) {
      const real ku = kf * ((real)kn.x * (real)U[3 * i] + (real)kn.y * (real)U[3 * i + 1] + (real)kn.z * (real)U[3 * i + 2]);
      if (t0) {
        sub[NT].x += ku * e.x;
        sub[NT].y += ku * e.y;
      } else {
        sub[NT + 1].x += ku * e.x;
        sub[NT + 1].y += ku * e.y;
      }
    }
    if (((i - a0) & 15) == 15 || i == a1 - 1) {
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        acc[s].x += (double)sub[s].x;
        acc[s].y += (double)sub[s].y;
        sub[s].x = sub[s].y = (real)0;
      }
    }
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) part[((size_t)blockIdx.y * p.nk + k) * NS + s] = acc[s];
}

template <int NV>
__device__ __forceinline__ void block_sum_part(double (&v)[NV], double *red, double *part_out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[q * 32 + warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0;
    for (int w = 0; w < nw; ++w) s += red[threadIdx.x * 32 + w];
    part_out[(size_t)blockIdx.x * NV + threadIdx.x] = s;
  }
}

// Chunk sums -> A_k = C f_k conj(S_k), B_k = C f_k T_k (C = 4 pi k_e / V), and
// per-k terms: MODE 1 (energy): {E_k, dE_k/dq_0, dE_k/dq_1};
// MODE 2 (VJP): {u . dF_k/dq_0, u . dF_k/dq_1}.
template <typename real, int MODE>
__global__ void __launch_bounds__(256) k_adj_kreduce(Params p, const double2 *__restrict__ part, int nchunks,
                                                     typename R2<real>::t *__restrict__ Ak,
                                                     typename R2<real>::t *__restrict__ Bk,
                                                     double *__restrict__ kpart) {
  constexpr bool VJP = MODE == 2;
  constexpr int NS = VJP ? 2 * NT : NT;
  constexpr int NV = MODE == 1 ? 1 + NT : NT;
  __shared__ double red[NV * 32];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double v[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = 0;
  if (k < p.nk) {
    double2 s[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) s[q] = make_double2(0, 0);
    for (int c = 0; c < nchunks; ++c)
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        const double2 x = part[((size_t)c * p.nk + k) * NS + q];
        s[q].x += x.x;
        s[q].y += x.y;
      }
    const double Cf = 12.56637061435917295384 * p.k_e / p.V * p.fk[k];
    const double Sx = p.charge[0] * s[0].x + p.charge[1] * s[1].x;
    const double Sy = p.charge[0] * s[0].y + p.charge[1] * s[1].y;
    typename R2<real>::t a;
    a.x = (real)(Cf * Sx);
    a.y = (real)(-Cf * Sy);
    Ak[k] = a;
    if (MODE == 1) {
      v[0] = 0.5 * Cf * (Sx * Sx + Sy * Sy);
#pragma unroll
      for (int t = 0; t < NT; ++t) v[1 + t] = Cf * (s[t].x * Sx + s[t].y * Sy);  // Re(S_t conj S)
    }
    if (VJP) {
      const double Tx = p.charge[0] * s[NT].x + p.charge[1] * s[NT + 1].x;
      const double Ty = p.charge[0] * s[NT].y + p.charge[1] * s[NT + 1].y;
      typename R2<real>::t b;
      b.x = (real)(Cf * Tx);
      b.y = (real)(Cf * Ty);
      Bk[k] = b;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        // Im(T_t conj S + T conj S_t)
        const double im1 = s[NT + t].y * Sx - s[NT + t].x * Sy;
        const double im2 = Ty * s[t].x - Tx * s[t].y;
        v[t] = Cf * (im1 + im2);
      }
    }
  }
  if (MODE != 0) block_sum_part<NV>(v, red, kpart);
}

// Pair terms of one ordered pair (type pair tp, charges qi qj, r2):
// c (F_i += c d), c1 = (1/r) dc/dr, and the parameter derivatives.
template <typename real> struct PairOut {
  real c, c1;
  real U_lj, Uq;           // LJ energy, Ewald real energy per unit q_i q_j
  real dc_e, dc_s, dU_e, dU_s, cq;
};

// FP32 (mixed) pair terms use the hardware reciprocal / reciprocal square
// root / exponential and erfc from Abramowitz & Stegun 7.1.26 sharing the
// Gaussian (erfc_as); the FP64 form keeps the correctly rounded functions.
__device__ __forceinline__ float adj_rcp(float x) { return __fdividef(1.f, x); }
__device__ __forceinline__ double adj_rcp(double x) { return 1.0 / x; }

template <typename real>
__device__ __forceinline__ PairOut<real> pair_terms(const Params &p, int tp, real qq, real r2, bool need_d2,
                                                    bool need_param, bool need_energy) {
  PairOut<real> o;
  o.c = o.c1 = o.U_lj = o.Uq = o.dc_e = o.dc_s = o.dU_e = o.dU_s = o.cq = (real)0;
  const real e = (real)p.eps[tp];
  if (r2 <= (real)p.rc_lj2 && e != (real)0) {
    const real sg = (real)p.sig[tp], rc2 = (real)p.rc_lj2;
    const real r2i = adj_rcp(r2), s2 = sg * sg * r2i, s6 = s2 * s2 * s2, s12 = s6 * s6;
    const real c2 = sg * sg / rc2, c6 = c2 * c2 * c2, c12 = c6 * c6;
    const real ce = (real)4 * ((-(real)12 * s12 + (real)6 * s6) * r2i + ((real)12 * c12 - (real)6 * c6) / rc2);
    o.c = e * ce;
    if (need_d2) o.c1 = e * (real)4 * ((real)168 * s12 - (real)48 * s6) * r2i * r2i;
    if (need_param || need_energy) {
      const real Ue = (real)4 * (s12 - s6) - (real)4 * (c12 - c6) +
                      (real)4 * ((real)12 * c12 - (real)6 * c6) * (r2 - rc2) / ((real)2 * rc2);
      o.U_lj = e * Ue;
      o.dc_e = ce;
      o.dU_e = Ue;
      const real isg = (real)1 / sg;
      o.dc_s = e * (real)4 * ((-(real)144 * s12 + (real)36 * s6) * r2i + ((real)144 * c12 - (real)36 * c6) / rc2) * isg;
      o.dU_s = e *
               ((real)4 * ((real)12 * s12 - (real)6 * s6) - (real)4 * ((real)12 * c12 - (real)6 * c6) +
                (r2 - rc2) / ((real)2 * rc2) * (real)4 * ((real)144 * c12 - (real)36 * c6)) *
               isg;
    }
  }
  if (r2 <= (real)p.rc_r2 && p.k_e != 0.0) {
    const real al = (real)p.alpha, beta = (real)(2.0 * p.alpha * 0.56418958354775628695);
    real r, ri, G, ec;
    if constexpr (sizeof(real) == 4) {
      ri = rsqrtf(r2);
      r = r2 * ri;
      G = __expf(-al * al * r2);
      ec = cvr::erfc_as(al * r, G);
    } else {
      r = sqrt(r2);
      ri = (real)1 / r;
      G = exp(-al * al * r2);
      ec = erfc(al * r);
    }
    const real E1 = -beta * G * ri - ec * ri * ri;
    const real cq = (real)p.k_e * E1 * ri;
    o.cq = cq;
    o.c += qq * cq;
    if (need_d2) {
      const real E2 = beta * G * ((real)2 * al * al + (real)2 * ri * ri) + (real)2 * ec * ri * ri * ri;
      o.c1 += qq * (real)p.k_e * (E2 - E1 * ri) * ri * ri;
    }
    if (need_energy || need_param) o.Uq = (real)p.k_e * ec * ri;
  }
  return o;
}

// One warp per atom i: MODE 0 forces; 1 forces + energies + dU/dtheta;
// 2 VJP w_i = sum_j K_ij (u_j - u_i) + k-space, and u . dF/dtheta.
template <typename real, int MODE>
__global__ void __launch_bounds__(ATOM_WARPS * 32) k_adj_atom(Params p, const double *__restrict__ X,
                                                              const double *__restrict__ U,
                                                              const typename R2<real>::t *__restrict__ tab,
                                                              const typename R2<real>::t *__restrict__ Ak,
                                                              const typename R2<real>::t *__restrict__ Bk,
                                                              double *__restrict__ out, double *__restrict__ part) {
  constexpr int NV = MODE == 1 ? 2 + 2 * NTT + NT : (MODE == 2 ? 2 * NTT + NT : 1);
  __shared__ double red[NV * 32];
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * ATOM_WARPS + (threadIdx.x >> 5);
  const int n = p.n;
  double v[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = 0;
  if (i < n) {
    const double xi = X[i], yi = X[n + i], zi = X[2 * n + i];
    const int ti = p.type[i];
    const real qi = (real)p.charge[ti];
    real ui[3] = {0, 0, 0};
    if (MODE == 2) {
      ui[0] = (real)U[3 * i];
      ui[1] = (real)U[3 * i + 1];
      ui[2] = (real)U[3 * i + 2];
    }
    real acc[3] = {0, 0, 0};
    const double L = p.L, iL = p.invL;
    for (int j = lane; j < n; j += 32) {
      if (j == i) continue;
      double dd[3] = {X[j] - xi, X[n + j] - yi, X[2 * n + j] - zi};
      real d[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) d[a] = (real)(dd[a] - L * rint(dd[a] * iL));
      const real r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 > (real)p.rc_r2 && r2 > (real)p.rc_lj2) continue;
      const int tj = p.type[j];
      const int tp = ti * NT + tj;
      const real qj = (real)p.charge[tj];
      const PairOut<real> o = pair_terms<real>(p, tp, qi * qj, r2, MODE == 2, MODE != 0, MODE == 1);
      if (MODE != 2) {
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] += o.c * d[a];
        if (MODE == 1) {
          v[0] += 0.5 * (double)o.U_lj;
          v[1] += 0.5 * (double)(qi * qj * o.Uq);
          const double he = 0.5 * (double)o.dU_e, hs = 0.5 * (double)o.dU_s;
          const double hqi = 0.5 * (double)(qj * o.Uq), hqj = 0.5 * (double)(qi * o.Uq);
#pragma unroll
          for (int q = 0; q < NTT; ++q)  // static indices keep v in registers
            if (q == tp) {
              v[2 + q] += he;
              v[2 + NTT + q] += hs;
            }
#pragma unroll
          for (int q = 0; q < NT; ++q) v[2 + 2 * NTT + q] += (q == ti ? hqi : 0.0) + (q == tj ? hqj : 0.0);
        }
      } else {
        const real du[3] = {(real)U[3 * j] - ui[0], (real)U[3 * j + 1] - ui[1], (real)U[3 * j + 2] - ui[2]};
        const real ddu = d[0] * du[0] + d[1] * du[1] + d[2] * du[2];
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] += o.c * du[a] + o.c1 * ddu * d[a];
        const real ud = ui[0] * d[0] + ui[1] * d[1] + ui[2] * d[2];
        const double ge = (double)(o.dc_e * ud), gs = (double)(o.dc_s * ud);
        const double gqi = (double)(qj * o.cq * ud), gqj = (double)(qi * o.cq * ud);
#pragma unroll
        for (int q = 0; q < NTT; ++q)
          if (q == tp) {
            v[q] += ge;
            v[NTT + q] += gs;
          }
#pragma unroll
        for (int q = 0; q < NT; ++q) v[2 * NTT + q] += (q == ti ? gqi : 0.0) + (q == tj ? gqj : 0.0);
      }
    }
    // k space: lanes over k-vectors
    const typename R2<real>::t *tb = tab + (size_t)i * 3 * p.kp;
    const real kf = (real)(6.28318530717958647692 * p.invL);
    for (int k = lane; k < p.nk; k += 32) {
      const int4 kn = p.kn[k];
      const auto e = atom_phase<real>(tb, p.kp, kn);
      const auto A = Ak[k];
      real coef;
      if (MODE != 2) {
        coef = qi * (e.x * A.y + e.y * A.x);  // q_i C f_k Im(e conj S)
      } else {
        const auto B = Bk[k];
        const real re1 = e.x * A.x - e.y * A.y;  // C f_k Re(e conj S)
        const real re2 = B.x * e.x + B.y * e.y;  // C f_k Re(T conj e)
        const real ku = kf * ((real)kn.x * ui[0] + (real)kn.y * ui[1] + (real)kn.z * ui[2]);
        coef = qi * (ku * re1 - re2);
      }
      acc[0] += coef * kf * (real)kn.x;
      acc[1] += coef * kf * (real)kn.y;
      acc[2] += coef * kf * (real)kn.z;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      real x = acc[a];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) out[a * n + i] = (double)x;
    }
  }
  if (MODE != 0) block_sum_part<NV>(v, red, part);
}

// dst[map[v]] += scale * sum_p part[p*nv + v], one warp per value, fixed order.
__global__ void k_adj_accum(const double *__restrict__ part, int nparts, int nv, Map m, double scale,
                            double *__restrict__ dst) {
  const int v = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (v >= nv) return;
  double s = 0;
  for (int q = lane; q < nparts; q += 32) s += part[(size_t)q * nv + v];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) dst[m.idx[v]] += scale * s;
}

// Xout = Xin + dt V + dt^2/2 F/m (md_simulator.cpp:591-593), SoA [3][n]
__global__ void k_adj_drift(Params p, const double *__restrict__ Xin, const double *__restrict__ V,
                            const double *__restrict__ F, double *__restrict__ Xout) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * p.n) return;
  const double mi = p.mass_inv[p.type[t % p.n]];
  Xout[t] = Xin[t] + V[t] * p.dt + F[t] * mi * 0.5 * p.dt * p.dt;
}

// V += dt/2 (Fold + Fnew)/m (md_simulator.cpp:616)
__global__ void k_adj_kick(Params p, double *__restrict__ V, const double *__restrict__ Fo,
                           const double *__restrict__ Fn) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * p.n) return;
  V[t] += 0.5 * p.dt * (Fo[t] + Fn[t]) * p.mass_inv[p.type[t % p.n]];
}

// Gr -= F/M; Ga += dt/2 Gv; u = Ga/m.  G*, F SoA [3][n]; u AoS [n][3].
__global__ void k_adj_rev_pre(Params p, double *__restrict__ Gr, const double *__restrict__ Gv,
                              double *__restrict__ Ga, const double *__restrict__ F, double *__restrict__ u,
                              double invM) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * p.n) return;
  const int i = t % p.n, a = t / p.n;
  Gr[t] -= invM * F[t];
  const double ga = Ga[t] + 0.5 * p.dt * Gv[t];
  Ga[t] = ga;
  u[3 * i + a] = ga * p.mass_inv[p.type[i]];
}

// Gr += w; (Gv, Ga) <- (Gv + dt Gr, dt/2 Gv + dt^2/2 Gr)
__global__ void k_adj_rev_post(Params p, double *__restrict__ Gr, double *__restrict__ Gv,
                               double *__restrict__ Ga, const double *__restrict__ W) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * p.n) return;
  const double gr = Gr[t] + W[t];
  const double gv = Gv[t];
  Gr[t] = gr;
  Gv[t] = gv + p.dt * gr;
  Ga[t] = 0.5 * p.dt * gv + 0.5 * p.dt * p.dt * gr;
}

__global__ void k_adj_u_from_ga(Params p, const double *__restrict__ Ga, double *__restrict__ u) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * p.n) return;
  const int i = t % p.n, a = t / p.n;
  u[3 * i + a] = Ga[t] * p.mass_inv[p.type[i]];
}

}  // namespace

struct cvr_adj {
  int device = 0, precision = CVR_PREC_MIXED;
  cudaStream_t stream = nullptr;
  Params p{};
  bool params_set = false, state_set = false;
  std::vector<int> type_h;
  std::vector<double> mass_h, charge_h, eps_h, sig_h;
  int n_types = 0;
  // device
  int *type = nullptr;
  int4 *kn = nullptr;
  double *fk = nullptr;
  double *x0 = nullptr, *v0 = nullptr;  // the state the loss starts from, SoA [3][n]
  double *X = nullptr, *Xb = nullptr, *V = nullptr, *F = nullptr, *Fb = nullptr;
  double *Gr = nullptr, *Gv = nullptr, *Ga = nullptr, *W = nullptr, *u = nullptr;
  void *tab = nullptr, *Ak = nullptr, *Bk = nullptr;
  double2 *skpart = nullptr;
  double *apart = nullptr, *kpart = nullptr, *accum = nullptr;
  double *ck = nullptr, *seg = nullptr;  // checkpoints, segment positions + forces
  size_t ck_cap = 0, seg_cap = 0;
  int nchunks = 0;
  std::string err;
};

namespace {

int afail(cvr_adj *a, int code, const std::string &m) {
  if (a) a->err = m;
  return code;
}

int cuda_ok(cvr_adj *a, const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return afail(a, CVR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return CVR_OK;
}

template <typename T>
int dalloc(cvr_adj *a, T **ptr, size_t count) {
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  if (cudaMalloc((void **)ptr, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess)
    return afail(a, CVR_ERR_NOMEM, "cudaMalloc");
  return CVR_OK;
}

inline int blocks(int n, int t) { return (n + t - 1) / t; }

Map seq_map(int off, int nv) {
  Map m{};
  for (int v = 0; v < nv && v < 16; ++v) m.idx[v] = off + v;
  return m;
}

// One force evaluation (MODE 0/1) or VJP (MODE 2) at positions X.
// MODE 0/1 write F (SoA); MODE 1 adds scale * {energies, dU/dtheta} into accum;
// MODE 2 reads u (AoS), writes W and adds scale * u . dF/dtheta into accum.
template <typename real, int MODE>
int eval(cvr_adj *a, const double *X, double *out, double scale) {
  using T2 = typename R2<real>::t;
  Params &p = a->p;
  cudaStream_t st = a->stream;
  T2 *tab = static_cast<T2 *>(a->tab), *Ak = static_cast<T2 *>(a->Ak), *Bk = static_cast<T2 *>(a->Bk);
  const int nt3 = p.n * 3 * p.kp;
  k_adj_tables<real><<<blocks(nt3, 256), 256, 0, st>>>(p, X, tab);
  if (p.nk > 0) {
    dim3 g(blocks(p.nk, SK_THREADS), a->nchunks);
    k_adj_sk<real, MODE == 2><<<g, SK_THREADS, 0, st>>>(p, tab, a->u, a->skpart);
    const int kb = blocks(p.nk, 256);
    k_adj_kreduce<real, MODE><<<kb, 256, 0, st>>>(p, a->skpart, a->nchunks, Ak, Bk, a->kpart);
    if (MODE == 1) {
      Map m{};
      m.idx[0] = A_EK;
      for (int t = 0; t < NT; ++t) m.idx[1 + t] = A_DQ + t;
      k_adj_accum<<<1, 32 * (1 + NT), 0, st>>>(a->kpart, kb, 1 + NT, m, scale, a->accum);
    } else if (MODE == 2) {
      k_adj_accum<<<1, 32 * NT, 0, st>>>(a->kpart, kb, NT, seq_map(A_VQ, NT), scale, a->accum);
    }
  }
  const int ab = blocks(p.n, ATOM_WARPS);
  k_adj_atom<real, MODE><<<ab, ATOM_WARPS * 32, 0, st>>>(p, X, a->u, tab, Ak, Bk, out, a->apart);
  if (MODE == 1) {
    const int nv = 2 + 2 * NTT + NT;
    Map m{};
    m.idx[0] = A_ELJ;
    m.idx[1] = A_EEW;
    for (int t = 0; t < NTT; ++t) {
      m.idx[2 + t] = A_DE + t;
      m.idx[2 + NTT + t] = A_DS + t;
    }
    for (int t = 0; t < NT; ++t) m.idx[2 + 2 * NTT + t] = A_DQ + t;
    k_adj_accum<<<1, 32 * nv, 0, st>>>(a->apart, ab, nv, m, scale, a->accum);
  } else if (MODE == 2) {
    const int nv = 2 * NTT + NT;
    Map m{};
    for (int t = 0; t < NTT; ++t) {
      m.idx[t] = A_VE + t;
      m.idx[NTT + t] = A_VS + t;
    }
    for (int t = 0; t < NT; ++t) m.idx[2 * NTT + t] = A_VQ + t;
    k_adj_accum<<<1, 32 * nv, 0, st>>>(a->apart, ab, nv, m, scale, a->accum);
  }
  return cuda_ok(a, "adjoint evaluation launch");
}

template <int MODE>
int evalp(cvr_adj *a, const double *X, double *out, double scale) {
  return a->precision == CVR_PREC_FP64 ? eval<double, MODE>(a, X, out, scale) : eval<float, MODE>(a, X, out, scale);
}

int ready(cvr_adj *a) {
  if (!a) return CVR_ERR_INVALID;
  if (!a->params_set) return afail(a, CVR_ERR_STATE, "cvr_adj_set_params has not been called");
  if (!a->state_set) return afail(a, CVR_ERR_STATE, "cvr_adj_set_state has not been called");
  cudaSetDevice(a->device);
  return CVR_OK;
}

// host-side terms: self energy -(alpha/sqrt(pi)) k_e sum q^2 and its q-gradient
double self_energy(const cvr_adj *a, double *dq) {
  double e = 0;
  for (int t = 0; t < NT; ++t) dq[t] = 0;
  if (a->p.nk == 0) return 0;
  for (int i = 0; i < a->p.n; ++i) {
    const double q = a->charge_h[a->type_h[i]];
    e += q * q;
    dq[a->type_h[i]] += 2 * q;
  }
  const double c = -0.56418958354775628695 * a->p.alpha * a->p.k_e;
  for (int t = 0; t < NT; ++t) dq[t] *= c;
  return c * e;
}

// fold raw ordered-type-pair sums into gradients of the shared symmetric parameters
void fold(const cvr_adj *a, const double *raw_e, const double *raw_s, const double *raw_q, const double *extra_q,
          double *g) {
  const int nt = a->n_types;
  for (int x = 0; x < nt; ++x)
    for (int y = 0; y < nt; ++y) {
      const int xy = x * NT + y, yx = y * NT + x;
      g[x * nt + y] = x == y ? raw_e[xy] : raw_e[xy] + raw_e[yx];
      g[nt * nt + x * nt + y] = x == y ? raw_s[xy] : raw_s[xy] + raw_s[yx];
    }
  for (int t = 0; t < nt; ++t) g[2 * nt * nt + t] = raw_q[t] + (extra_q ? extra_q[t] : 0.0);
}

int download_soa(cvr_adj *a, const double *src, double *dst_aos) {
  const int n = a->p.n;
  std::vector<double> h(3 * (size_t)n);
  cudaMemcpyAsync(h.data(), src, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, a->stream);
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return afail(a, CVR_ERR_CUDA, "download");
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) dst_aos[3 * i + d] = h[(size_t)d * n + i];
  return CVR_OK;
}

}  // namespace

extern "C" {

int cvr_adj_create(cvr_adj **out, int64_t n, double box_len, int n_types, const double *mass, int precision,
                   int device) {
  if (!out) return CVR_ERR_INVALID;
  *out = nullptr;
  if (n < 2 || n > (1 << 24) || !(box_len > 0) || n_types < 1 || n_types > NT || !mass) return CVR_ERR_INVALID;
  if (precision != CVR_PREC_MIXED && precision != CVR_PREC_FP64) return CVR_ERR_INVALID;
  for (int t = 0; t < n_types; ++t)
    if (!(mass[t] > 0)) return CVR_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return CVR_ERR_CUDA;
  cvr_adj *a = new cvr_adj();
  a->device = device;
  a->precision = precision;
  a->n_types = n_types;
  a->mass_h.assign(mass, mass + n_types);
  Params &p = a->p;
  p.n = (int)n;
  p.nt = n_types;
  p.L = box_len;
  p.invL = 1.0 / box_len;
  p.V = box_len * box_len * box_len;
  for (int t = 0; t < NT; ++t) p.mass_inv[t] = t < n_types ? 1.0 / mass[t] : 0.0;
  cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking);
  const size_t N3 = 3 * (size_t)n;
  int rc = 0;
  if ((rc = dalloc(a, &a->type, n)) || (rc = dalloc(a, &a->x0, N3)) || (rc = dalloc(a, &a->v0, N3)) ||
      (rc = dalloc(a, &a->X, N3)) || (rc = dalloc(a, &a->Xb, N3)) || (rc = dalloc(a, &a->V, N3)) ||
      (rc = dalloc(a, &a->F, N3)) || (rc = dalloc(a, &a->Fb, N3)) || (rc = dalloc(a, &a->Gr, N3)) ||
      (rc = dalloc(a, &a->Gv, N3)) || (rc = dalloc(a, &a->Ga, N3)) || (rc = dalloc(a, &a->W, N3)) ||
      (rc = dalloc(a, &a->u, N3)) || (rc = dalloc(a, &a->accum, A_N)) ||
      (rc = dalloc(a, &a->apart, (size_t)blocks((int)n, ATOM_WARPS) * 16))) {
    cvr_adj_destroy(a);
    return rc;
  }
  cudaMemset(a->u, 0, N3 * sizeof(double));
  *out = a;
  return CVR_OK;
}

void cvr_adj_destroy(cvr_adj *a) {
  if (!a) return;
  cudaSetDevice(a->device);
  if (a->stream) cudaStreamSynchronize(a->stream);
  void *ptrs[] = {a->type, a->kn, a->fk, a->x0, a->v0, a->X, a->Xb, a->V, a->F, a->Fb, a->Gr, a->Gv, a->Ga,
                  a->W, a->u, a->tab, a->Ak, a->Bk, a->skpart, a->apart, a->kpart, a->accum, a->ck, a->seg};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (a->stream) cudaStreamDestroy(a->stream);
  delete a;
}

int cvr_adj_set_params(cvr_adj *a, const double *charge, const double *eps, const double *sigma, double rc_lj,
                       double alpha, double rc_r, int kmax, double k_e, double dt) {
  if (!a || !charge || !eps || !sigma) return CVR_ERR_INVALID;
  if (kmax < 0 || kmax > KMAX_ADJ) return afail(a, CVR_ERR_INVALID, "k_max must be in [0, 10]");
  if (!(alpha > 0) || !(dt >= 0) || !(rc_lj > 0) || !(rc_r >= 0))
    return afail(a, CVR_ERR_INVALID, "alpha > 0, rc_lj > 0, rc_r >= 0, dt >= 0");
  Params &p = a->p;
  if (rc_lj > 0.5 * p.L * (1 + 1e-12) || rc_r > 0.5 * p.L * (1 + 1e-12))
    return afail(a, CVR_ERR_GEOMETRY, "cutoffs must be at most half the box (minimum image)");
  const int nt = a->n_types;
  for (int x = 0; x < nt; ++x)
    for (int y = 0; y < nt; ++y)
      if (eps[x * nt + y] != eps[y * nt + x] || sigma[x * nt + y] != sigma[y * nt + x] || !(sigma[x * nt + y] > 0))
        return afail(a, CVR_ERR_INVALID, "eps and sigma must be symmetric, sigma > 0");
  cudaSetDevice(a->device);
  a->charge_h.assign(charge, charge + nt);
  a->eps_h.assign(eps, eps + nt * nt);
  a->sig_h.assign(sigma, sigma + nt * nt);
  for (int t = 0; t < NT; ++t) p.charge[t] = t < nt ? charge[t] : 0.0;
  for (int x = 0; x < NT; ++x)
    for (int y = 0; y < NT; ++y) {
      const bool ok = x < nt && y < nt;
      p.eps[x * NT + y] = ok ? eps[x * nt + y] : 0.0;
      p.sig[x * NT + y] = ok ? sigma[x * nt + y] : 1.0;
    }
  p.rc_lj2 = rc_lj * rc_lj;
  p.rc_r2 = rc_r * rc_r;
  p.alpha = alpha;
  p.k_e = k_e;
  p.dt = dt;
  const bool kchanged = !a->params_set || kmax != p.kmax;
  p.kmax = kmax;
  p.kp = kmax + 1;
  // the reference's k-set (initialize.cpp:184-222): first (2k)^3 of the nesting, 0 skipped
  std::vector<int4> kn;
  std::vector<double> fk;
  const long long used = (long long)(2 * kmax) * (2 * kmax) * (2 * kmax);
  for (int x = -kmax; x <= kmax; ++x)
    for (int y = -kmax; y <= kmax; ++y)
      for (int z = -kmax; z <= kmax; ++z) {
        if ((long long)kn.size() >= used) break;
        if (!x && !y && !z) continue;
        kn.push_back(make_int4(x, y, z, 0));
        const double ksq = (6.28318530717958647692 * p.invL) * (6.28318530717958647692 * p.invL) * (x * x + y * y + z * z);
        fk.push_back(std::exp(-ksq / (4 * alpha * alpha)) / ksq);
      }
  p.nk = (int)kn.size();
  a->nchunks = blocks(p.n, SK_CHUNK);
  int rc = 0;
  const size_t r2 = a->precision == CVR_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  if (kchanged) {
    if ((rc = dalloc(a, &a->kn, kn.size())) || (rc = dalloc(a, &a->fk, fk.size())) ||
        (rc = dalloc(a, &a->skpart, (size_t)a->nchunks * std::max(p.nk, 1) * 2 * NT)) ||
        (rc = dalloc(a, &a->kpart, (size_t)blocks(std::max(p.nk, 1), 256) * 4)))
      return rc;
    if (a->tab) cudaFree(a->tab);
    if (a->Ak) cudaFree(a->Ak);
    if (a->Bk) cudaFree(a->Bk);
    a->tab = a->Ak = a->Bk = nullptr;
    if (cudaMalloc(&a->tab, (size_t)p.n * 3 * p.kp * r2) != cudaSuccess ||
        cudaMalloc(&a->Ak, std::max(p.nk, 1) * r2) != cudaSuccess ||
        cudaMalloc(&a->Bk, std::max(p.nk, 1) * r2) != cudaSuccess)
      return afail(a, CVR_ERR_NOMEM, "cudaMalloc");
  }
  if (!kn.empty()) {
    cudaMemcpy(a->kn, kn.data(), kn.size() * sizeof(int4), cudaMemcpyHostToDevice);
    cudaMemcpy(a->fk, fk.data(), fk.size() * sizeof(double), cudaMemcpyHostToDevice);
  }
  p.kn = a->kn;
  p.fk = a->fk;
  p.type = a->type;
  a->params_set = true;
  return CVR_OK;
}

int cvr_adj_set_state(cvr_adj *a, const double *pos, const double *vel, const int32_t *type) {
  if (!a || !pos || !type) return CVR_ERR_INVALID;
  cudaSetDevice(a->device);
  const int n = a->p.n;
  for (int i = 0; i < n; ++i)
    if (type[i] < 0 || type[i] >= a->n_types) return afail(a, CVR_ERR_INVALID, "atom type out of range");
  a->type_h.assign(type, type + n);
  std::vector<double> soa(6 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      soa[(size_t)d * n + i] = pos[3 * i + d];
      soa[(size_t)(3 + d) * n + i] = vel ? vel[3 * i + d] : 0.0;
    }
  cudaMemcpyAsync(a->x0, soa.data(), 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, a->stream);
  cudaMemcpyAsync(a->v0, soa.data() + 3 * (size_t)n, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice,
                  a->stream);
  cudaMemcpyAsync(a->type, type, n * sizeof(int32_t), cudaMemcpyHostToDevice, a->stream);
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return afail(a, CVR_ERR_CUDA, "upload");
  a->p.type = a->type;
  a->state_set = true;
  return CVR_OK;
}

int cvr_adj_forces(cvr_adj *a, double *force, double *energy, double *dU) {
  if (int rc = ready(a)) return rc;
  cudaMemsetAsync(a->accum, 0, A_N * sizeof(double), a->stream);
  if (int rc = evalp<1>(a, a->x0, a->F, 1.0)) return rc;
  std::vector<double> acc(A_N);
  cudaMemcpyAsync(acc.data(), a->accum, A_N * sizeof(double), cudaMemcpyDeviceToHost, a->stream);
  if (force) {
    if (int rc = download_soa(a, a->F, force)) return rc;
  } else if (cudaStreamSynchronize(a->stream) != cudaSuccess) {
    return afail(a, CVR_ERR_CUDA, "force evaluation failed");
  }
  double dq_self[NT];
  const double es = self_energy(a, dq_self);
  if (energy) {
    energy[0] = acc[A_ELJ];
    energy[1] = acc[A_EEW];
    energy[2] = acc[A_EK];
    energy[3] = es;
  }
  if (dU) fold(a, &acc[A_DE], &acc[A_DS], &acc[A_DQ], dq_self, dU);
  return CVR_OK;
}

int cvr_adj_force_vjp(cvr_adj *a, const double *u, double *w, double *g) {
  if (int rc = ready(a)) return rc;
  if (!u) return afail(a, CVR_ERR_INVALID, "u is required");
  cudaMemcpyAsync(a->u, u, 3 * (size_t)a->p.n * sizeof(double), cudaMemcpyHostToDevice, a->stream);
  cudaMemsetAsync(a->accum, 0, A_N * sizeof(double), a->stream);
  if (int rc = evalp<2>(a, a->x0, a->W, 1.0)) return rc;
  std::vector<double> acc(A_N);
  cudaMemcpyAsync(acc.data(), a->accum, A_N * sizeof(double), cudaMemcpyDeviceToHost, a->stream);
  if (w) {
    if (int rc = download_soa(a, a->W, w)) return rc;
  } else if (cudaStreamSynchronize(a->stream) != cudaSuccess) {
    return afail(a, CVR_ERR_CUDA, "VJP failed");
  }
  if (g) fold(a, &acc[A_VE], &acc[A_VS], &acc[A_VQ], nullptr, g);
  return CVR_OK;
}

static int forward_step(cvr_adj *a, const double *Xin, double *Xout, double *Fin, double *Fout, double scale,
                        bool energy) {
  const int n3 = 3 * a->p.n, tb = 256;
  k_adj_drift<<<blocks(n3, tb), tb, 0, a->stream>>>(a->p, Xin, a->V, Fin, Xout);
  if (int rc = energy ? evalp<1>(a, Xout, Fout, scale) : evalp<0>(a, Xout, Fout, scale)) return rc;
  k_adj_kick<<<blocks(n3, tb), tb, 0, a->stream>>>(a->p, a->V, Fin, Fout);
  return cuda_ok(a, "forward step");
}

int cvr_adj_loss(cvr_adj *a, int64_t nsteps, double *loss, double *pos_out, double *vel_out) {
  if (int rc = ready(a)) return rc;
  if (nsteps < 0) return afail(a, CVR_ERR_INVALID, "nsteps < 0");
  const size_t N3 = 3 * (size_t)a->p.n;
  cudaMemsetAsync(a->accum, 0, A_N * sizeof(double), a->stream);
  cudaMemcpyAsync(a->X, a->x0, N3 * sizeof(double), cudaMemcpyDeviceToDevice, a->stream);
  cudaMemcpyAsync(a->V, a->v0, N3 * sizeof(double), cudaMemcpyDeviceToDevice, a->stream);
  if (int rc = evalp<1>(a, a->X, a->F, 0.0)) return rc;
  double *x = a->X, *xb = a->Xb, *f = a->F, *fb = a->Fb;
  const double scale = nsteps ? 1.0 / (double)nsteps : 0.0;
  for (int64_t t = 0; t < nsteps; ++t) {
    if (int rc = forward_step(a, x, xb, f, fb, scale, true)) return rc;
    std::swap(x, xb);
    std::swap(f, fb);
  }
  std::vector<double> acc(A_N);
  cudaMemcpyAsync(acc.data(), a->accum, A_N * sizeof(double), cudaMemcpyDeviceToHost, a->stream);
  if (pos_out) {
    if (int rc = download_soa(a, x, pos_out)) return rc;
  }
  if (vel_out) {
    if (int rc = download_soa(a, a->V, vel_out)) return rc;
  }
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return afail(a, CVR_ERR_CUDA, "loss run failed");
  double dq[NT];
  const double es = self_energy(a, dq);
  if (loss) *loss = nsteps ? acc[A_ELJ] + acc[A_EEW] + acc[A_EK] + es : 0.0;
  return CVR_OK;
}

int cvr_adj_loss_grad(cvr_adj *a, int64_t nsteps, int64_t checkpoint_every, double *loss, double *g_pos,
                      double *g_vel, double *g_theta) {
  if (int rc = ready(a)) return rc;
  if (nsteps < 1 || checkpoint_every < 1) return afail(a, CVR_ERR_INVALID, "nsteps >= 1, checkpoint_every >= 1");
  const int n3 = 3 * a->p.n, tb = 256;
  const size_t N3 = (size_t)n3;
  const int64_t M = nsteps, K = std::min<int64_t>(checkpoint_every, nsteps);
  const int64_t nseg = (M + K - 1) / K;
  if ((size_t)nseg * 2 * N3 > a->ck_cap) {
    if (int rc = dalloc(a, &a->ck, (size_t)nseg * 2 * N3)) return rc;
    a->ck_cap = (size_t)nseg * 2 * N3;
  }
  if ((size_t)(K + 1) * 2 * N3 > a->seg_cap) {
    if (int rc = dalloc(a, &a->seg, (size_t)(K + 1) * 2 * N3)) return rc;
    a->seg_cap = (size_t)(K + 1) * 2 * N3;
  }
  cudaStream_t st = a->stream;
  const double invM = 1.0 / (double)M;
  cudaMemsetAsync(a->accum, 0, A_N * sizeof(double), st);
  // forward: loss, dU/dtheta, checkpoints
  cudaMemcpyAsync(a->X, a->x0, N3 * sizeof(double), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(a->V, a->v0, N3 * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (int rc = evalp<1>(a, a->X, a->F, 0.0)) return rc;
  double *x = a->X, *xb = a->Xb, *f = a->F, *fb = a->Fb;
  for (int64_t t = 0; t < M; ++t) {
    if (t % K == 0) {
      double *c = a->ck + (size_t)(t / K) * 2 * N3;
      cudaMemcpyAsync(c, x, N3 * sizeof(double), cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(c + N3, a->V, N3 * sizeof(double), cudaMemcpyDeviceToDevice, st);
    }
    if (int rc = forward_step(a, x, xb, f, fb, invM, true)) return rc;
    std::swap(x, xb);
    std::swap(f, fb);
  }
  // reverse
  cudaMemsetAsync(a->Gr, 0, N3 * sizeof(double), st);
  cudaMemsetAsync(a->Gv, 0, N3 * sizeof(double), st);
  cudaMemsetAsync(a->Ga, 0, N3 * sizeof(double), st);
  for (int64_t s = nseg - 1; s >= 0; --s) {
    const int64_t t0 = s * K, t1 = std::min(M, t0 + K);
    const double *c = a->ck + (size_t)s * 2 * N3;
    double *segX = a->seg, *segF = a->seg + (size_t)(K + 1) * N3;
    cudaMemcpyAsync(segX, c, N3 * sizeof(double), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(a->V, c + N3, N3 * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (int rc = evalp<1>(a, segX, segF, 0.0)) return rc;
    for (int64_t t = t0; t < t1; ++t) {
      const int64_t q = t - t0;
      if (int rc = forward_step(a, segX + q * N3, segX + (q + 1) * N3, segF + q * N3, segF + (q + 1) * N3, 0.0, true))
        return rc;
    }
    for (int64_t t = t1 - 1; t >= t0; --t) {
      const int64_t q = t - t0 + 1;
      k_adj_rev_pre<<<blocks(n3, tb), tb, 0, st>>>(a->p, a->Gr, a->Gv, a->Ga, segF + q * N3, a->u, invM);
      if (int rc = evalp<2>(a, segX + q * N3, a->W, 1.0)) return rc;
      k_adj_rev_post<<<blocks(n3, tb), tb, 0, st>>>(a->p, a->Gr, a->Gv, a->Ga, a->W);
    }
  }
  // a_0 = F(r_0)/m
  k_adj_u_from_ga<<<blocks(n3, tb), tb, 0, st>>>(a->p, a->Ga, a->u);
  if (int rc = evalp<2>(a, a->x0, a->W, 1.0)) return rc;
  {
    // Gr += W: rev_post with dt = 0 would also touch Gv/Ga; a plain add is enough here
    Params p0 = a->p;
    p0.dt = 0;
    k_adj_rev_post<<<blocks(n3, tb), tb, 0, st>>>(p0, a->Gr, a->Gv, a->Ga, a->W);
  }
  if (int rc = cuda_ok(a, "reverse sweep")) return rc;
  std::vector<double> acc(A_N);
  cudaMemcpyAsync(acc.data(), a->accum, A_N * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (g_pos)
    if (int rc = download_soa(a, a->Gr, g_pos)) return rc;
  if (g_vel) {
    // the final rev_post with dt = 0 set Gv unchanged; Gv is the velocity cotangent
    if (int rc = download_soa(a, a->Gv, g_vel)) return rc;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return afail(a, CVR_ERR_CUDA, "adjoint run failed");
  double dq_self[NT];
  const double es = self_energy(a, dq_self);
  if (loss) *loss = acc[A_ELJ] + acc[A_EEW] + acc[A_EK] + es;
  if (g_theta) {
    double re[NTT], rs[NTT], rq[NT];
    for (int t = 0; t < NTT; ++t) {
      re[t] = acc[A_DE + t] + acc[A_VE + t];
      rs[t] = acc[A_DS + t] + acc[A_VS + t];
    }
    for (int t = 0; t < NT; ++t) rq[t] = acc[A_DQ + t] + acc[A_VQ + t];
    fold(a, re, rs, rq, dq_self, g_theta);
  }
  return CVR_OK;
}

int cvr_adj_last_error(const cvr_adj *a, char *buf, size_t len) {
  if (!a || !buf || !len) return CVR_ERR_INVALID;
  std::snprintf(buf, len, "%s", a->err.c_str());
  return CVR_OK;
}

void *cvr_adj_stream(const cvr_adj *a) { return a ? (void *)a->stream : nullptr; }

}  // extern "C"
