// cvr_batch.cu -- many small independent periodic systems (replicas) advanced
// together: one persistent CTA per replica for all steps, all replicas in one
// CUDA graph launch.
//
// No reference counterpart for the batching: the reference runs one system
// per process (each replica as its own system needs its list radius and ghost
// cutoff at L/2, the largest its one-ghost-image scheme allows,
// exchange_ghost_single_md_domain.cpp:59-99).  Physics per replica: LJ with
// the reference's linear force shift (lj.cpp:439-448) up to rc_lj, Ewald real
// space (electrostatic_ewald_r.cpp:196-198) up to rc_r <= L/2 under the
// minimum image (all pairs: at rc = L/2 half of all pairs are inside, so a
// cell list would save at most 2x), Ewald k space over the reference's k-set
// (initialize.cpp:184-222) and force (electrostatic_ewald_k.cpp:197-234).
//
// Layout: FP64 positions/velocities in global memory (concatenated, SoA);
// each CTA keeps its replica's positions in shared memory as 32-bit
// fixed-point coordinates u = round(x 2^32 / L) mod 2^32, so the minimum-image
// displacement of a pair is the wrapping int32 difference (one integer
// subtraction and one conversion per axis; resolution L / 2^32), the pair
// constants are scaled to those units (h = L / 2^32) and the summed pair
// forces are multiplied by 1/h once per atom; the k-space phases take their
// argument m u mod 2^32 exactly in integer arithmetic.  The k-space
// accumulation S(k) is FP64; energies and virial are FP64 block sums.
//
// Launch shape (threads per CTA) per replica size class is chosen by timing
// candidates on the state itself (the autotuner below), replicas start in
// decreasing size order (longest first), and the per-class launches are one
// CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/caviar_b200.h"
#include "cvr_device.cuh"

namespace {

constexpr int NMAX = 2048;  // atoms per replica
constexpr int KMAXB = 6;    // k_max per axis
constexpr int KP = KMAXB + 1;
constexpr int RUNMAX = 2 * KMAXB + 1;  // longest nz run of the k-set
constexpr int TMAX = 4;
constexpr int CH = 64;   // atoms per phase-table stage of S(k)
constexpr int GMAX = 4;  // atom groups per k-run in S(k)
constexpr int NTH = 8;   // per-replica results: ke, e_lj, e_ewr, e_k, e_self, virial, temperature, steps

// skip: every k of the run has its mirror -k at a smaller index (in a run
// that is summed); S(k) = conj(S(-k)) is then filled from it and the mirror's
// force term, equal to this run's, counts twice.
struct KRunB {
  int nx, ny, nz0, len, k0, skip;
};

constexpr int KFILL_MASK = (1 << 30) - 1;
constexpr int KTWICE = 1 << 30;

struct BatchDev {
  const int *order;
  const long long *off;
  const int *n, *nq;  // atoms, charged atoms (stored first) per replica
  const double *L, *rc_lj, *rc_r;
  double *x, *y, *z, *vx, *vy, *vz;
  float *fx, *fy, *fz;  // FP32 forces of the current positions (carried between launches)
  const int *type;
  const int4 *kint;
  const KRunB *runs;
  // per k: bits 0-29 = 1 + the mirror's index when k's run is skipped (S(k)
  // filled from it), bit 30 = k's force term counts twice (its mirror is skipped)
  const int *kinfo;
  double *out;  // [replica][NTH]
  int nk, nruns, kmax, n_types;
  float eps[TMAX * TMAX], sig[TMAX * TMAX], charge[TMAX];
  double mass[TMAX], mass_inv[TMAX], chargeD[TMAX];
  double alpha, k_e, dt;
};

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf_if(float2 a, bool c) {
  if (c) a.y = -a.y;
  return a;
}

using cvr::erfc_as;  // Abramowitz & Stegun 7.1.26 (cvr_device.cuh)

// e^{i 2 pi m x / L} for the fixed-point coordinate u of x: m x / L = m u / 2^32,
// reduced mod 1 exactly by the wrapping product, then sincospi of the signed
// residue over 2^31 (in [-1, 1)).
__device__ __forceinline__ float2 fixed_phase(uint32_t u, int m) {
  float sn, cs;
  sincospif((float)(int)((uint32_t)m * u) * 4.656612873077393e-10f, &sn, &cs);
  return make_float2(cs, sn);
}

template <int TPB, int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *red, double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[q * 32 + warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int q = 0; q < NV; ++q) {
      double s = 0;
      for (int w = 0; w < TPB / 32; ++w) s += red[q * 32 + w];
      out[q] = s;  // thread 0's totals
    }
  __syncthreads();
}

// Shared-memory state of one replica (np = atoms rounded up to 32).
struct Smem {
  float4 *ljc;      // per type pair: sig2, eps24, eps48, K (this replica's LJ cutoff)
  float4 *lje;      // per type pair: e4, C0, C1, k_e q_i q_j
  float4 *xh, *xl;  // xh: fixed-point coordinates (uint32 bits) and type; xl.w: charge
  double2 *skd;     // FP64 S(k) accumulators
  double *red;
  float2 *ak;   // (4 pi / V) f_k conj(S_k) for the k-force
  float2 *skp;  // FP32 S(k) partials of one stage, per atom group
  float2 *tab;  // phase tables of a stage of CH atoms
  float *fsx, *fsy, *fsz;  // force accumulators
  float *fk;
};

__host__ __device__ inline int groups_for(int tpb, int nruns) {
  const int g = nruns > 0 ? tpb / nruns : 1;
  return g < 1 ? 1 : (g > GMAX ? GMAX : g);
}

__host__ __device__ inline size_t smem_bytes(int nk, int np, int G) {
  return (size_t)2 * TMAX * TMAX * 16 + (size_t)2 * np * 16 + (size_t)nk * 16 + 9 * 32 * 8 + (size_t)nk * 8 +
         (size_t)G * nk * 8 + (size_t)CH * 3 * KP * 8 + (size_t)3 * np * 4 + (size_t)((nk + 3) & ~3) * 4;
}

__device__ inline Smem carve(unsigned char *raw, int nk, int np, int G) {
  Smem S;
  S.ljc = reinterpret_cast<float4 *>(raw);
  S.lje = S.ljc + TMAX * TMAX;
  S.xh = S.lje + TMAX * TMAX;
  S.xl = S.xh + np;
  S.skd = reinterpret_cast<double2 *>(S.xl + np);
  S.red = reinterpret_cast<double *>(S.skd + nk);
  S.ak = reinterpret_cast<float2 *>(S.red + 9 * 32);
  S.skp = S.ak + nk;
  S.tab = S.skp + (size_t)G * nk;
  S.fsx = reinterpret_cast<float *>(S.tab + CH * 3 * KP);
  S.fsy = S.fsx + np;
  S.fsz = S.fsy + np;
  S.fk = S.fsz + np;
  return S;
}

// Per-replica pair constants and cutoffs, in units of h = L / 2^32 (lengths
// / h: rc2, rr2 / h^2, alpha * h, 2 alpha / sqrt(pi) * h, k_e / h; the LJ
// tables likewise), so that a pair term takes the fixed-point displacement.
struct PairK {
  float rc2, rr2, alpha2, alpha, tas, ke;
  float4 lc, le;  // uniform LJ constants (UNI)
};

// One ordered pair (i, j): c with F_i += c d, d = r_j - r_i (minimum image).
// EWR: this pair may carry charge on both ends.  Energies into e[0..2] (lj, ewr, virial) scaled by w.
template <bool UNI, bool EWR, bool EV>
__device__ __forceinline__ float pair_c(const Smem &S, const PairK &K, const float4 &ih, const float4 &il,
                                        const float4 &jh, const float4 &jl, float (&d)[3], double (&e)[3], double w) {
  // minimum image: the wrapping difference of the fixed-point coordinates
  d[0] = (float)(int)(__float_as_uint(jh.x) - __float_as_uint(ih.x));
  d[1] = (float)(int)(__float_as_uint(jh.y) - __float_as_uint(ih.y));
  d[2] = (float)(int)(__float_as_uint(jh.z) - __float_as_uint(ih.z));
  const float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  float4 lc, le;
  if (UNI) {
    lc = K.lc;
    le = K.le;
  } else {
    const int tp = __float_as_int(ih.w) * TMAX + __float_as_int(jh.w);
    lc = S.ljc[tp];
    le = S.lje[tp];
  }
  float c = 0.f;
  if (r2 <= K.rc2 && lc.y != 0.f) {
    const float r2i = __fdividef(1.f, r2), s2 = lc.x * r2i, s6 = s2 * s2 * s2;
    c = r2i * s6 * (lc.y - lc.z * s6) + lc.w;
    if (EV) e[0] += w * (double)(le.x * (s6 * s6 - s6) + le.z * r2 + le.y);
  }
  if (EWR) {
    const float qq = UNI ? K.ke * il.w * jl.w : le.w;
    if (qq != 0.f && r2 <= K.rr2) {
      const float rinv = rsqrtf(r2), rr = r2 * rinv;
      const float ex = __expf(-K.alpha2 * r2);
      const float er = erfc_as(K.alpha * rr, ex);
      c -= qq * (K.tas * ex + er * rinv) * (rinv * rinv);
      if (EV) e[1] += w * (double)(qq * er * rinv);
    }
  }
  if (EV) e[2] -= w * (double)(c * r2);
  return c;
}

// Off-diagonal tile: atoms of block I (one per lane) with atoms of block J,
// each unordered pair once (Newton's third law).  Lane l meets atom
// J*32 + (l + s) % 32 at step s; the reaction force on that atom travels with
// it (shuffled one lane down per step) and is home after 32 steps.
template <bool UNI, bool EWR, bool EV>
__device__ __forceinline__ void tile(const Smem &S, const PairK &K, int I, int J, int n, double (&e)[3]) {
  const int lane = threadIdx.x & 31;
  const int i = I * 32 + lane;
  const bool vi = i < n;
  const float4 ih = S.xh[i], il = S.xl[i];
  float fi[3] = {0.f, 0.f, 0.f}, fj[3] = {0.f, 0.f, 0.f};
#pragma unroll 4
  for (int s = 0; s < 32; ++s) {
    const int j = J * 32 + ((lane + s) & 31);
    if (vi && j < n) {
      const float4 jh = S.xh[j], jl = S.xl[j];
      float d[3];
      const float c = pair_c<UNI, EWR, EV>(S, K, ih, il, jh, jl, d, e, 1.0);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        fi[a] = fmaf(c, d[a], fi[a]);
        fj[a] = fmaf(-c, d[a], fj[a]);
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) fj[a] = __shfl_sync(0xffffffffu, fj[a], (lane + 1) & 31);
  }
  S.fsx[i] += fi[0];
  S.fsy[i] += fi[1];
  S.fsz[i] += fi[2];
  const int jj = J * 32 + lane;
  S.fsx[jj] += fj[0];
  S.fsy[jj] += fj[1];
  S.fsz[jj] += fj[2];
}

// Diagonal tile: ordered pairs inside block I (each pair from both ends).
template <bool UNI, bool EWR, bool EV>
__device__ __forceinline__ void tile_diag(const Smem &S, const PairK &K, int I, int n, double (&e)[3]) {
  const int lane = threadIdx.x & 31;
  const int i = I * 32 + lane;
  const bool vi = i < n;
  const float4 ih = S.xh[i], il = S.xl[i];
  float fi[3] = {0.f, 0.f, 0.f};
  for (int s = 1; s < 32; ++s) {
    const int j = I * 32 + ((lane + s) & 31);
    if (vi && j < n) {
      const float4 jh = S.xh[j], jl = S.xl[j];
      float d[3];
      const float c = pair_c<UNI, EWR, EV>(S, K, ih, il, jh, jl, d, e, 0.5);
#pragma unroll
      for (int a = 0; a < 3; ++a) fi[a] = fmaf(c, d[a], fi[a]);
    }
  }
  S.fsx[i] += fi[0];
  S.fsy[i] += fi[1];
  S.fsz[i] += fi[2];
}

// Forces of the replica's current positions into S.fs* (all pairs under the
// minimum image, then k space).  EV: energies and virial into ev[0..4]
// (this thread's share: lj, ewald_r, ewald_k, -, virial).
template <int TPB, bool UNI, bool EV>
__device__ void batch_forces(const BatchDev &p, const Smem &S, int r, int n, int nq, double L, int G,
                             double (&ev)[5]) {
  constexpr int W = TPB / 32;
  const int warp = threadIdx.x >> 5;
  const double h = L * 2.3283064365386963e-10;  // L / 2^32
  PairK K;
  K.rc2 = (float)(p.rc_lj[r] * p.rc_lj[r] / (h * h));
  K.rr2 = (float)(p.rc_r[r] * p.rc_r[r] / (h * h));
  K.alpha = (float)(p.alpha * h);
  K.alpha2 = K.alpha * K.alpha;
  K.tas = (float)(2.0 * p.alpha * 0.56418958354775628695 * h);
  K.ke = (float)(p.k_e / h);
  K.lc = S.ljc[0];
  K.le = S.lje[0];
  const int nb = (n + 31) >> 5;
  for (int i = threadIdx.x; i < nb * 32; i += TPB) S.fsx[i] = S.fsy[i] = S.fsz[i] = 0.f;
  __syncthreads();
  double e[3] = {0, 0, 0};
  // ---- pairs: round-robin schedule of block pairs (circle method), every
  // block in at most one tile per round, a barrier between rounds
  const int nbe = nb + (nb & 1), m = nbe - 1, half = nbe >> 1;
  for (int round = 0; round < m; ++round) {
    for (int q = warp; q < half; q += W) {
      int I, J;
      if (q == 0) {
        I = m;
        J = round;
      } else {
        I = (round + q) % m;
        J = (round - q + m) % m;
      }
      if (I >= nb || J >= nb) continue;
      const bool ewr = (I * 32 < nq) && (J * 32 < nq);  // warp-uniform: charged atoms come first
      if (ewr)
        tile<UNI, true, EV>(S, K, I, J, n, e);
      else
        tile<UNI, false, EV>(S, K, I, J, n, e);
    }
    __syncthreads();
  }
  for (int I = warp; I < nb; I += W) {
    if (I * 32 < nq)
      tile_diag<UNI, true, EV>(S, K, I, n, e);
    else
      tile_diag<UNI, false, EV>(S, K, I, n, e);
  }
  __syncthreads();
  // pair forces from units of h back to length units
  {
    const float inv_h = (float)(4294967296.0 / L);
    for (int i = threadIdx.x; i < nb * 32; i += TPB) {
      S.fsx[i] *= inv_h;
      S.fsy[i] *= inv_h;
      S.fsz[i] *= inv_h;
    }
  }
  if (EV) {
    ev[0] += e[0];
    ev[1] += e[1];
    ev[4] += e[2];
  }
  // ---- k space: S(k) along the k-set's nz runs, G atom groups per run, per
  // stage of CH atoms: FP32 sums of at most CH/G atoms, then FP64 per k
  const int nk = p.nk, kmax = p.kmax;
  for (int k = threadIdx.x; k < nk; k += TPB) S.skd[k] = make_double2(0.0, 0.0);
  const int items = p.nruns * G;
  for (int a0 = 0; a0 < nq; a0 += CH) {  // neutral atoms (stored after the charged ones) add nothing
    const int na = min(CH, nq - a0);
    __syncthreads();
    for (int t = threadIdx.x; t < na * 3 * KP; t += TPB) {
      const int at = t / (3 * KP), rem = t % (3 * KP), dd = rem / KP, mm = rem % KP;
      float2 v = make_float2(0.f, 0.f);
      if (mm <= kmax) {
        const float4 h = S.xh[a0 + at];
        const uint32_t u = __float_as_uint(dd == 0 ? h.x : (dd == 1 ? h.y : h.z));
        v = fixed_phase(u, mm);
      }
      S.tab[t] = v;
    }
    __syncthreads();
    for (int it = threadIdx.x; it < items; it += TPB) {
      const int ri = it % p.nruns, g = it / p.nruns;
      const KRunB run = p.runs[ri];
      if (run.skip) continue;
      float2 acc[RUNMAX];
#pragma unroll
      for (int u = 0; u < RUNMAX; ++u) acc[u] = make_float2(0.f, 0.f);
      const int mx = abs(run.nx), my = abs(run.ny), mz = abs(run.nz0);
      for (int at = g; at < na; at += G) {
        const float2 *tb = S.tab + at * 3 * KP;
        const float q = S.xl[a0 + at].w;
        float2 ph = cmulf(cmulf(conjf_if(tb[mx], run.nx < 0), conjf_if(tb[KP + my], run.ny < 0)),
                          conjf_if(tb[2 * KP + mz], run.nz0 < 0));
        ph.x *= q;
        ph.y *= q;
        const float2 ez = tb[2 * KP + 1];
#pragma unroll
        for (int u = 0; u < RUNMAX; ++u)
          if (u < run.len) {
            acc[u].x += ph.x;
            acc[u].y += ph.y;
            ph = cmulf(ph, ez);
          }
      }
#pragma unroll
      for (int u = 0; u < RUNMAX; ++u)
        if (u < run.len) S.skp[(size_t)g * nk + run.k0 + u] = acc[u];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nk; k += TPB) {
      if (p.kinfo[k] & KFILL_MASK) continue;  // filled from its mirror below
      double2 a = S.skd[k];
      for (int g = 0; g < G; ++g) {
        const float2 v = S.skp[(size_t)g * nk + k];
        a.x += (double)v.x;
        a.y += (double)v.y;
      }
      S.skd[k] = a;
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nk; k += TPB) {  // S(k) = conj(S(-k)) of the skipped runs
    const int f = p.kinfo[k] & KFILL_MASK;
    if (f) {
      const double2 v = S.skd[f - 1];
      S.skd[k] = make_double2(v.x, -v.y);
    }
  }
  __syncthreads();
  const double Vd = L * L * L;
  for (int k = threadIdx.x; k < nk; k += TPB) {
    const double2 sk = S.skd[k];
    const double fkk = (double)S.fk[k];
    const double cf = 12.56637061435917295384 / Vd * fkk * ((p.kinfo[k] & KTWICE) ? 2.0 : 1.0);
    S.ak[k] = make_float2((float)(cf * sk.x), (float)(-cf * sk.y));
    if (EV) ev[2] += 6.28318530717958647692 / Vd * p.k_e * fkk * (sk.x * sk.x + sk.y * sk.y);
  }
  __syncthreads();
  // ---- k-force of each charged atom, phases along the nz runs
  const float tpl = (float)(6.28318530717958647692 / L);
  for (int i = threadIdx.x; i < nq; i += TPB) {
    float2 tx[KP], ty[KP], tz[KP];
    const float4 h = S.xh[i], lo = S.xl[i];
    const uint32_t uc[3] = {__float_as_uint(h.x), __float_as_uint(h.y), __float_as_uint(h.z)};
#pragma unroll
    for (int mm = 0; mm < KP; ++mm) {
      tx[mm] = fixed_phase(uc[0], mm);
      ty[mm] = fixed_phase(uc[1], mm);
      tz[mm] = fixed_phase(uc[2], mm);
    }
    float fx = 0, fy = 0, fz = 0;
    for (int rr = 0; rr < p.nruns; ++rr) {
      const KRunB run = p.runs[rr];
      if (run.skip) continue;  // counted twice in its mirror's coefficients
      float2 px = tx[0], py = ty[0], pz = tz[0];
#pragma unroll
      for (int mm = 0; mm < KP; ++mm) {
        if (mm == abs(run.nx)) px = tx[mm];
        if (mm == abs(run.ny)) py = ty[mm];
        if (mm == abs(run.nz0)) pz = tz[mm];
      }
      // e^{i k.r} along the run: start at nz0, then one step of e^{i 2 pi z / L} per k
      float2 ph = cmulf(cmulf(conjf_if(px, run.nx < 0), conjf_if(py, run.ny < 0)), conjf_if(pz, run.nz0 < 0));
      const float2 ez = tz[1];
      float tsum = 0.f;
      for (int u = 0; u < run.len; ++u) {
        const float2 A = S.ak[run.k0 + u];
        const float t = A.x * ph.y + A.y * ph.x;
        tsum += t;
        fz += (float)(run.nz0 + u) * t;
        ph = cmulf(ph, ez);
      }
      fx += (float)run.nx * tsum;
      fy += (float)run.ny * tsum;
    }
    const float qk = (float)p.k_e * lo.w * tpl;
    S.fsx[i] += qk * fx;
    S.fsy[i] += qk * fy;
    S.fsz[i] += qk * fz;
  }
}

// Fixed-point copy u = round(x 2^32 / L) mod 2^32 of one atom's FP64
// position (the bits of u in xh.x-z, the type in xh.w, the charge in xl.w).
__device__ __forceinline__ void to_smem(const BatchDev &p, const Smem &S, int i, long long gi, double L) {
  const double sc = 4294967296.0 / L;
  const double c[3] = {p.x[gi], p.y[gi], p.z[gi]};
  uint32_t u[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) u[a] = (uint32_t)(unsigned long long)llrint(c[a] * sc);  // 2^32 wraps to 0
  const int t = p.type[gi];
  S.xh[i] = make_float4(__uint_as_float(u[0]), __uint_as_float(u[1]), __uint_as_float(u[2]), __int_as_float(t));
  S.xl[i] = make_float4(0.f, 0.f, 0.f, p.charge[t]);
}

// One launch: nsteps velocity-Verlet steps of replica order[first + blockIdx.x].
// compute_first = 0 takes the forces of the current positions from fx/fy/fz
// (written by the previous launch), so runs split over several launches are
// bit-identical to one run.  Energies and virial come from a separate
// evaluation at the final positions (the stepping forces never depend on
// whether energies are wanted).  Each thread owns atoms tid, tid + TPB, ...
// for the integrator and the k-space force; the pair tiles write forces of
// any atom, ordered by barriers.
template <int TPB, bool UNI>
__global__ void __launch_bounds__(TPB, 1) k_batch(BatchDev p, int first, int nsteps, int np, int G,
                                                   int compute_first) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int r = p.order[first + blockIdx.x];
  const int n = p.n[r], nq = p.nq[r];
  const long long o = p.off[r];
  const double L = p.L[r];
  const Smem S = carve(smraw, p.nk, np, G);
  // LJ constants for this replica's cutoff (lj.cpp:439-448) and k_e q_i q_j
  if (threadIdx.x < TMAX * TMAX) {
    const int a = threadIdx.x / TMAX, b = threadIdx.x % TMAX, T = p.n_types;
    const bool ok = a < T && b < T;
    // in units of h = L / 2^32 (see PairK): sigma^2 / h^2, K h^2, C1 h^2, k_e q q / h
    const double hh = L * 2.3283064365386963e-10, h2 = hh * hh;
    const double rc2 = p.rc_lj[r] * p.rc_lj[r];
    const double e = ok ? p.eps[a * T + b] : 0.0, sg = ok ? p.sig[a * T + b] : 0.0;
    const double rcinv = 1.0 / rc2, c2 = sg * sg * rcinv, c6 = c2 * c2 * c2, c12 = c6 * c6;
    const double g = 4.0 * e * (12.0 * c12 - 6.0 * c6);
    S.ljc[threadIdx.x] = make_float4((float)(sg * sg / h2), (float)(24.0 * e), (float)(48.0 * e),
                                     (float)(4.0 * e * (12.0 * c12 * rcinv - 6.0 * c6 * rcinv) * h2));
    S.lje[threadIdx.x] = make_float4((float)(4.0 * e), (float)(-4.0 * e * (c12 - c6) - 0.5 * g),
                                     (float)(g / (2.0 * rc2) * h2),
                                     ok ? (float)(p.k_e * p.chargeD[a] * p.chargeD[b] / hh) : 0.f);
  }
  // f_k = exp(-k^2 / 4 alpha^2) / k^2 for this box (initialize.cpp:201-221)
  const double tpl = 6.28318530717958647692 / L, fa = 1.0 / (4.0 * p.alpha * p.alpha);
  for (int k = threadIdx.x; k < p.nk; k += TPB) {
    const int4 kn = p.kint[k];
    const double ksq = tpl * tpl * (double)(kn.x * kn.x + kn.y * kn.y + kn.z * kn.z);
    S.fk[k] = (float)(exp(-ksq * fa) / ksq);
  }
  for (int i = threadIdx.x; i < np; i += TPB) {
    if (i < n) {
      to_smem(p, S, i, o + i, L);
    } else {
      S.xh[i] = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
      S.xl[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  __syncthreads();
  double ev[5] = {0, 0, 0, 0, 0};
  if (compute_first) {
    batch_forces<TPB, UNI, false>(p, S, r, n, nq, L, G, ev);
  } else {
    for (int i = threadIdx.x; i < n; i += TPB) {
      S.fsx[i] = p.fx[o + i];
      S.fsy[i] = p.fy[o + i];
      S.fsz[i] = p.fz[o + i];
    }
  }
  const double dt = p.dt, h = 0.5 * dt;
  for (int step = 0; step < nsteps; ++step) {
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += TPB) {
      const long long gi = o + i;
      const double mi = p.mass_inv[p.type[gi]];
      double *X[3] = {p.x, p.y, p.z}, *V[3] = {p.vx, p.vy, p.vz};
      const float fv[3] = {S.fsx[i], S.fsy[i], S.fsz[i]};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double v = V[a][gi] + h * (double)fv[a] * mi;
        double x = X[a][gi] + dt * v;
        x -= L * floor(x / L);
        V[a][gi] = v;
        X[a][gi] = x;
      }
      to_smem(p, S, i, gi, L);
    }
    __syncthreads();
    batch_forces<TPB, UNI, false>(p, S, r, n, nq, L, G, ev);
    for (int i = threadIdx.x; i < n; i += TPB) {
      const long long gi = o + i;
      const double mi = p.mass_inv[p.type[gi]];
      p.vx[gi] += h * (double)S.fsx[i] * mi;
      p.vy[gi] += h * (double)S.fsy[i] * mi;
      p.vz[gi] += h * (double)S.fsz[i] * mi;
    }
  }
  // forces of the final positions, carried to the next launch
  for (int i = threadIdx.x; i < n; i += TPB) {
    p.fx[o + i] = S.fsx[i];
    p.fy[o + i] = S.fsy[i];
    p.fz[o + i] = S.fsz[i];
  }
  __syncthreads();
  batch_forces<TPB, UNI, true>(p, S, r, n, nq, L, G, ev);  // energies only; S.fs* is scratch here
  __syncthreads();
  // kinetic energy (COM removed), energies
  double kv[9] = {0, 0, 0, 0, 0, ev[0], ev[1], ev[4], ev[2]};
  for (int i = threadIdx.x; i < n; i += TPB) {
    const long long gi = o + i;
    const double ms = p.mass[p.type[gi]];
    const double v0 = p.vx[gi], v1 = p.vy[gi], v2 = p.vz[gi];
    kv[0] += ms * (v0 * v0 + v1 * v1 + v2 * v2);
    kv[1] += ms * v0;
    kv[2] += ms * v1;
    kv[3] += ms * v2;
    kv[4] += ms;
  }
  double tot[9];
  block_sum<TPB, 9>(kv, S.red, tot);
  if (threadIdx.x == 0) {
    double q2 = 0;
    for (int i = 0; i < n; ++i) {
      const double q = p.chargeD[p.type[o + i]];
      q2 += q * q;
    }
    double *out = p.out + (size_t)r * NTH;
    const double ke = 0.5 * tot[0] - 0.5 * (tot[1] * tot[1] + tot[2] * tot[2] + tot[3] * tot[3]) / tot[4];
    out[0] = ke;
    out[1] = tot[5];
    out[2] = tot[6];
    out[3] = tot[8];
    out[4] = -0.56418958354775628695 * p.alpha * q2 * p.k_e;
    out[5] = tot[7];
    out[6] = (n > 1) ? 2.0 * ke / (3.0 * n - 3.0) : 0.0;
    out[7] = (double)nsteps;
  }
}

using KernelFn = void (*)(BatchDev, int, int, int, int, int);

struct Shape {
  int tpb;
  KernelFn fn, fn_uni;
};

// Launch shapes (threads per CTA); the uniform-LJ form when every type pair has the same eps and sigma
const Shape kShapes[] = {
    {128, k_batch<128, false>, k_batch<128, true>},
    {256, k_batch<256, false>, k_batch<256, true>},
    {512, k_batch<512, false>, k_batch<512, true>},
};

}  // namespace

struct cvr_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n_rep = 0, n_types = 0;
  long long n_total = 0;
  std::vector<int> n, nq;
  std::vector<long long> off;
  std::vector<double> L, rc_lj, rc_r;
  std::vector<int> slot_of;  // caller's atom index -> stored slot (charged atoms first within a replica)
  std::vector<double> charge_h;
  bool uniform = false;      // every type pair has the same eps and sigma
  BatchDev dev{};
  std::vector<void *> allocs;
  // size classes: [first, count) in the order array, chosen shape
  struct Class {
    int first, count, nmax, shape;
  };
  std::vector<Class> classes;
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};  // one per size class: the graph's parallel branches
  cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
  cudaGraphExec_t graph = nullptr;
  int graph_steps = -1;
  std::string err;
  bool tuned = false;
  bool forces_valid = false;  // fx/fy/fz hold the forces of the current positions
  std::vector<double> tune_ms;
};

namespace {

int bfail(cvr_batch *b, int code, const std::string &m) {
  if (b) b->err = m;
  return code;
}

template <typename T>
int balloc(cvr_batch *b, T **p, size_t count) {
  void *q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return bfail(b, CVR_ERR_NOMEM, "cudaMalloc");
  b->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return CVR_OK;
}

int launch_class(cvr_batch *b, const cvr_batch::Class &c, int shape, int nsteps, int compute_first,
                 cudaStream_t st) {
  const Shape &s = kShapes[shape];
  const int np = (c.nmax + 31) & ~31;
  const int G = groups_for(s.tpb, b->dev.nruns);
  (b->uniform ? s.fn_uni : s.fn)<<<c.count, s.tpb, smem_bytes(b->dev.nk, np, G), st>>>(b->dev, c.first, nsteps, np,
                                                                                         G, compute_first);
  return cudaGetLastError() == cudaSuccess ? CVR_OK : CVR_ERR_CUDA;
}

}  // namespace

extern "C" {

int cvr_batch_create(cvr_batch **out, int n_rep, const int64_t *n_atoms, const double *box_len, int n_types,
                     const double *mass, const double *charge, int device) {
  if (!out) return CVR_ERR_INVALID;
  *out = nullptr;
  if (n_rep <= 0 || !n_atoms || !box_len || !mass || !charge || n_types <= 0 || n_types > TMAX) return CVR_ERR_INVALID;
  for (int r = 0; r < n_rep; ++r)
    if (n_atoms[r] < 1 || n_atoms[r] > NMAX || !(box_len[r] > 0)) return CVR_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return CVR_ERR_CUDA;
  cvr_batch *b = new cvr_batch();
  b->device = device;
  b->n_rep = n_rep;
  b->n_types = n_types;
  b->n.assign(n_atoms, n_atoms + n_rep);
  b->nq.assign(n_rep, 0);
  b->L.assign(box_len, box_len + n_rep);
  b->charge_h.assign(charge, charge + n_types);
  b->off.resize(n_rep);
  long long o = 0;
  for (int r = 0; r < n_rep; ++r) {
    b->off[r] = o;
    o += n_atoms[r];
  }
  b->n_total = o;
  cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int c = 0; c < 3; ++c) {
    cudaStreamCreateWithFlags(&b->side[c], cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&b->join[c], cudaEventDisableTiming);
  }
  BatchDev &d = b->dev;
  d.n_types = n_types;
  for (int t = 0; t < n_types; ++t) {
    d.mass[t] = mass[t];
    d.mass_inv[t] = mass[t] == 0 ? 0 : 1.0 / mass[t];
    d.chargeD[t] = charge[t];
    d.charge[t] = (float)charge[t];
  }
  int rc = 0;
  int *dn;
  long long *doff;
  int *dorder;
  double *dL;
  if ((rc = balloc(b, &dn, 2 * n_rep)) || (rc = balloc(b, &doff, n_rep)) || (rc = balloc(b, &dorder, n_rep)) ||
      (rc = balloc(b, &dL, 3 * n_rep)))
    return rc;
  const size_t N = (size_t)o;
  double *arr;
  float *farr;
  int *dtype;
  double *dout;
  if ((rc = balloc(b, &arr, 6 * N)) || (rc = balloc(b, &farr, 3 * N)) || (rc = balloc(b, &dtype, N)) ||
      (rc = balloc(b, &dout, (size_t)n_rep * NTH)))
    return rc;
  d.x = arr;
  d.y = arr + N;
  d.z = arr + 2 * N;
  d.vx = arr + 3 * N;
  d.vy = arr + 4 * N;
  d.vz = arr + 5 * N;
  cudaMemset(farr, 0, 3 * N * sizeof(float));
  d.fx = farr;
  d.fy = farr + N;
  d.fz = farr + 2 * N;
  d.type = dtype;
  d.out = dout;
  d.n = dn;
  d.nq = dn + n_rep;
  d.off = doff;
  d.order = dorder;
  d.L = dL;
  d.rc_lj = dL + n_rep;
  d.rc_r = dL + 2 * n_rep;
  // replicas in decreasing size; size classes by the atoms-per-thread a shape needs
  std::vector<int> order(n_rep);
  for (int r = 0; r < n_rep; ++r) order[r] = r;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->n[a] > b->n[c]; });
  const int bounds[3] = {2048, 1024, 512};
  int k = 0;
  for (int ci = 0; ci < 3; ++ci) {
    const int hi = bounds[ci], lo = (ci < 2) ? bounds[ci + 1] : 0;
    const int first = k;
    while (k < n_rep && b->n[order[k]] > lo && b->n[order[k]] <= hi) ++k;
    if (k > first) b->classes.push_back({first, k - first, b->n[order[first]], -1});
  }
  cudaMemcpy(dn, b->n.data(), n_rep * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemset(dn + n_rep, 0, n_rep * sizeof(int));
  cudaMemcpy(doff, b->off.data(), n_rep * sizeof(long long), cudaMemcpyHostToDevice);
  cudaMemcpy(dorder, order.data(), n_rep * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(dL, b->L.data(), n_rep * sizeof(double), cudaMemcpyHostToDevice);
  *out = b;
  return CVR_OK;
}

void cvr_batch_destroy(cvr_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (void *p : b->allocs) cudaFree(p);
  for (int c = 0; c < 3; ++c) {
    cudaStreamDestroy(b->side[c]);
    cudaEventDestroy(b->join[c]);
  }
  cudaEventDestroy(b->fork);
  cudaStreamDestroy(b->stream);
  delete b;
}

int cvr_batch_set_forces(cvr_batch *b, const double *eps, const double *sigma, const double *rc_lj,
                         const double *rc_r, double alpha, int kmax, double k_e, double dt) {
  if (!b || !eps || !sigma || !rc_lj || !rc_r) return CVR_ERR_INVALID;
  if (kmax < 0 || kmax > KMAXB) return bfail(b, CVR_ERR_INVALID, "k_max above 6 is not supported by the batch path");
  if (!(alpha > 0) || !(dt >= 0)) return bfail(b, CVR_ERR_INVALID, "alpha > 0, dt >= 0");
  cudaSetDevice(b->device);
  const int T = b->n_types;
  b->uniform = true;
  for (int t = 0; t < T * T; ++t) {
    b->dev.eps[t] = (float)eps[t];
    b->dev.sig[t] = (float)sigma[t];
    if (eps[t] != eps[0] || sigma[t] != sigma[0]) b->uniform = false;
  }
  for (int r = 0; r < b->n_rep; ++r)
    if (!(rc_r[r] <= 0.5 * b->L[r] * (1 + 1e-12)) || !(rc_lj[r] <= 0.5 * b->L[r] * (1 + 1e-12)))
      return bfail(b, CVR_ERR_GEOMETRY, "cutoffs must be at most half the box (minimum image)");
  b->rc_lj.assign(rc_lj, rc_lj + b->n_rep);
  b->rc_r.assign(rc_r, rc_r + b->n_rep);
  cudaMemcpy((void *)b->dev.rc_lj, rc_lj, b->n_rep * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy((void *)b->dev.rc_r, rc_r, b->n_rep * sizeof(double), cudaMemcpyHostToDevice);
  b->dev.alpha = alpha;
  b->dev.k_e = k_e;
  b->dev.dt = dt;
  b->dev.kmax = kmax;
  // the reference's k-set (initialize.cpp:184-222) in runs of nz at fixed (nx, ny)
  std::vector<int4> kint;
  std::vector<KRunB> runs;
  const long long used = (long long)(2 * kmax) * (2 * kmax) * (2 * kmax);
  for (int a = -kmax; a <= kmax; ++a)
    for (int c = -kmax; c <= kmax; ++c)
      for (int z = -kmax; z <= kmax; ++z) {
        if ((long long)kint.size() >= used) break;
        if (a == 0 && c == 0 && z == 0) continue;
        const int k = (int)kint.size();
        kint.push_back(make_int4(a, c, z, 0));
        if (!runs.empty() && runs.back().nx == a && runs.back().ny == c && runs.back().nz0 + runs.back().len == z)
          runs.back().len++;
        else
          runs.push_back({a, c, z, 1, k, 0});
      }
  b->dev.nk = (int)kint.size();
  b->dev.nruns = (int)runs.size();
  // For real charges S(-k) = conj(S(k)) and k, -k give the same force term:
  // a run whose every k has its mirror at a smaller index is skipped (that
  // mirror's run is always summed), its S(k) filled by conjugation and its
  // force counted twice through the mirror's coefficient.
  std::vector<int> kinfo(kint.size(), 0);
  {
    std::map<std::tuple<int, int, int>, int> kidx;
    for (int k = 0; k < (int)kint.size(); ++k) kidx[std::make_tuple(kint[k].x, kint[k].y, kint[k].z)] = k;
    std::vector<int> mir(kint.size(), -1);
    for (int k = 0; k < (int)kint.size(); ++k) {
      const auto it = kidx.find(std::make_tuple(-kint[k].x, -kint[k].y, -kint[k].z));
      if (it != kidx.end()) mir[k] = it->second;
    }
    for (KRunB &r : runs) {
      r.skip = 1;
      for (int u = 0; u < r.len; ++u) r.skip = r.skip && mir[r.k0 + u] >= 0 && mir[r.k0 + u] < r.k0 + u;
      if (r.skip)
        for (int u = 0; u < r.len; ++u) {
          kinfo[r.k0 + u] = mir[r.k0 + u] + 1;
          kinfo[mir[r.k0 + u]] |= KTWICE;
        }
    }
  }
  int4 *dk;
  KRunB *dr;
  int *dki;
  if (int rc = balloc(b, &dk, kint.size())) return rc;
  if (int rc = balloc(b, &dr, runs.size())) return rc;
  if (int rc = balloc(b, &dki, kinfo.size())) return rc;
  cudaMemcpy(dk, kint.data(), kint.size() * sizeof(int4), cudaMemcpyHostToDevice);
  cudaMemcpy(dr, runs.data(), runs.size() * sizeof(KRunB), cudaMemcpyHostToDevice);
  cudaMemcpy(dki, kinfo.data(), kinfo.size() * sizeof(int), cudaMemcpyHostToDevice);
  b->dev.kint = dk;
  b->dev.runs = dr;
  b->dev.kinfo = dki;
  for (const Shape &s : kShapes) {
    const int sm = (int)smem_bytes(b->dev.nk, NMAX, groups_for(s.tpb, b->dev.nruns));
    if (cudaFuncSetAttribute(s.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess ||
        cudaFuncSetAttribute(s.fn_uni, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess)
      return bfail(b, CVR_ERR_CUDA, "shared memory attribute");
  }
  b->tuned = false;
  b->forces_valid = false;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return CVR_OK;
}

int cvr_batch_set_state(cvr_batch *b, const double *pos, const double *vel, const int32_t *type) {
  if (!b || !pos || !type) return CVR_ERR_INVALID;
  cudaSetDevice(b->device);
  const size_t N = (size_t)b->n_total;
  for (size_t i = 0; i < N; ++i)
    if (type[i] < 0 || type[i] >= b->n_types) return bfail(b, CVR_ERR_INVALID, "atom type out of range");
  // within each replica, charged atoms first (stable): the pair tiles then
  // know from the block index alone whether Ewald terms can occur
  b->slot_of.assign(N, 0);
  for (int r = 0; r < b->n_rep; ++r) {
    const long long o = b->off[r];
    int k = 0;
    for (int pass = 0; pass < 2; ++pass)
      for (int i = 0; i < b->n[r]; ++i) {
        const bool charged = b->charge_h[type[o + i]] != 0.0;
        if (charged == (pass == 0)) b->slot_of[o + i] = (int)(o + k++);
      }
    int q = 0;
    for (int i = 0; i < b->n[r]; ++i) q += b->charge_h[type[o + i]] != 0.0;
    b->nq[r] = q;
  }
  std::vector<double> soa(6 * N, 0.0);
  std::vector<int32_t> ts(N);
  for (size_t i = 0; i < N; ++i) {
    const size_t sl = (size_t)b->slot_of[i];
    ts[sl] = type[i];
    for (int a = 0; a < 3; ++a) {
      soa[a * N + sl] = pos[3 * i + a];
      soa[(3 + a) * N + sl] = vel ? vel[3 * i + a] : 0.0;
    }
  }
  cudaMemcpyAsync(b->dev.x, soa.data(), 6 * N * sizeof(double), cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync((void *)b->dev.type, ts.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync((void *)b->dev.nq, b->nq.data(), b->n_rep * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  b->forces_valid = false;
  return cudaStreamSynchronize(b->stream) == cudaSuccess ? CVR_OK : bfail(b, CVR_ERR_CUDA, "upload");
}

// Autotuner: for each size class, time every launch shape (threads per CTA,
// which also sets the atom groups per k-run of S(k)) that fits the shared
// memory on 2 steps of the real state (restored afterwards); keep the fastest.
static int batch_tune(cvr_batch *b) {
  const size_t N = (size_t)b->n_total;
  double *save = nullptr;
  if (cudaMalloc(&save, 6 * N * sizeof(double)) != cudaSuccess) return bfail(b, CVR_ERR_NOMEM, "tune buffer");
  cudaMemcpyAsync(save, b->dev.x, 6 * N * sizeof(double), cudaMemcpyDeviceToDevice, b->stream);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  b->tune_ms.clear();
  for (auto &c : b->classes) {
    float best = 1e30f;
    int best_s = -1;
    for (int si = 0; si < (int)(sizeof(kShapes) / sizeof(kShapes[0])); ++si) {
      const Shape &s = kShapes[si];
      const int np = (c.nmax + 31) & ~31;
      if (smem_bytes(b->dev.nk, np, groups_for(s.tpb, b->dev.nruns)) > 227 * 1024) continue;
      if (s.tpb > 2 * np) continue;  // more threads than pair-tile warps and atoms can use
      cudaEventRecord(e0, b->stream);
      if (launch_class(b, c, si, 2, 1, b->stream)) {
        cudaFree(save);
        return bfail(b, CVR_ERR_CUDA, "tuning launch failed");
      }
      cudaEventRecord(e1, b->stream);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      b->tune_ms.push_back(ms);
      if (ms < best) {
        best = ms;
        best_s = si;
      }
    }
    if (best_s < 0) {
      cudaFree(save);
      return bfail(b, CVR_ERR_GEOMETRY, "no launch shape fits the replica size");
    }
    c.shape = best_s;
  }
  cudaMemcpyAsync(b->dev.x, save, 6 * N * sizeof(double), cudaMemcpyDeviceToDevice, b->stream);
  cudaStreamSynchronize(b->stream);
  cudaFree(save);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tuned = true;
  b->forces_valid = false;
  return CVR_OK;
}

int cvr_batch_run(cvr_batch *b, int64_t nsteps, double *out) {
  if (!b) return CVR_ERR_INVALID;
  if (nsteps < 0 || nsteps > (1 << 30)) return bfail(b, CVR_ERR_INVALID, "bad step count");
  if (!b->dev.kint) return bfail(b, CVR_ERR_STATE, "cvr_batch_set_forces has not been called");
  if (b->slot_of.empty()) return bfail(b, CVR_ERR_STATE, "cvr_batch_set_state has not been called");
  cudaSetDevice(b->device);
  if (!b->tuned)
    if (int rc = batch_tune(b)) return rc;
  if (!b->forces_valid) {
    for (auto &c : b->classes)
      if (launch_class(b, c, c.shape, 0, 1, b->stream)) return bfail(b, CVR_ERR_CUDA, "force launch failed");
    b->forces_valid = true;
  }
  if (!b->graph || b->graph_steps != (int)nsteps) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    cudaGraph_t g;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return bfail(b, CVR_ERR_CUDA, "capture");
    // size classes as parallel branches: the small-replica class fills the
    // SMs the large-replica class leaves idle
    int lrc = CVR_OK;
    cudaEventRecord(b->fork, b->stream);
    for (size_t ci = 0; ci < b->classes.size(); ++ci) {
      cudaStreamWaitEvent(b->side[ci], b->fork, 0);
      lrc |= launch_class(b, b->classes[ci], b->classes[ci].shape, (int)nsteps, 0, b->side[ci]);
      cudaEventRecord(b->join[ci], b->side[ci]);
      cudaStreamWaitEvent(b->stream, b->join[ci], 0);
    }
    const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (ce != cudaSuccess || lrc != CVR_OK) return bfail(b, CVR_ERR_CUDA, "capture of the replica launches failed");
    if (cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) return bfail(b, CVR_ERR_CUDA, "instantiate");
    cudaGraphDestroy(g);
    b->graph_steps = (int)nsteps;
  }
  if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) return bfail(b, CVR_ERR_CUDA, "graph launch");
  if (out)
    cudaMemcpyAsync(out, b->dev.out, (size_t)b->n_rep * NTH * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
  const cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return bfail(b, CVR_ERR_CUDA, cudaGetErrorString(e));
  return CVR_OK;
}

int cvr_batch_get_state(cvr_batch *b, double *pos, double *vel, double *acc) {
  if (!b) return CVR_ERR_INVALID;
  cudaSetDevice(b->device);
  const size_t N = (size_t)b->n_total;
  std::vector<double> soa(6 * N);
  std::vector<float> a(3 * N);
  std::vector<int32_t> t(N);
  cudaMemcpyAsync(soa.data(), b->dev.x, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
  cudaMemcpyAsync(a.data(), b->dev.fx, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, b->stream);
  cudaMemcpyAsync(t.data(), b->dev.type, N * sizeof(int32_t), cudaMemcpyDeviceToHost, b->stream);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bfail(b, CVR_ERR_CUDA, "download");
  for (size_t i = 0; i < N; ++i) {
    const size_t sl = b->slot_of.empty() ? i : (size_t)b->slot_of[i];
    for (int d = 0; d < 3; ++d) {
      if (pos) pos[3 * i + d] = soa[d * N + sl];
      if (vel) vel[3 * i + d] = soa[(3 + d) * N + sl];
      if (acc) acc[3 * i + d] = (double)a[d * N + sl] * b->dev.mass_inv[t[sl]];
    }
  }
  return CVR_OK;
}

int cvr_batch_info(const cvr_batch *b, int64_t *out, int len) {
  if (!b || !out) return CVR_ERR_INVALID;
  std::vector<int64_t> v = {b->n_rep, b->n_total, (int64_t)b->classes.size()};
  for (auto &c : b->classes) {
    v.push_back(c.count);
    v.push_back(c.nmax);
    v.push_back(c.shape >= 0 ? kShapes[c.shape].tpb : 0);
    v.push_back(c.shape >= 0 ? groups_for(kShapes[c.shape].tpb, b->dev.nruns) : 0);
  }
  for (int k = 0; k < len && k < (int)v.size(); ++k) out[k] = v[k];
  return CVR_OK;
}

int cvr_batch_last_error(const cvr_batch *b, char *buf, size_t len) {
  if (!b || !buf || !len) return CVR_ERR_INVALID;
  std::snprintf(buf, len, "%s", b->err.c_str());
  return CVR_OK;
}

void *cvr_batch_stream(const cvr_batch *b) { return b ? (void *)b->stream : nullptr; }

}  // extern "C"
