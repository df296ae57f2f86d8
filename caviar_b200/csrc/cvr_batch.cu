// cvr_batch.cu -- many small independent periodic systems (replicas) advanced
// together: one persistent CTA per replica for all steps, all replicas in one
// CUDA graph launch.
//
// No reference counterpart: the reference runs one system per process, and
// its one-ghost-image scheme cannot hold boxes smaller than twice the list
// radius (exchange_ghost_single_md_domain.cpp:59-99), which is where most of
// these replicas sit (L = 4.3 .. 13.7 sigma).  Physics per replica: LJ with
// the reference's linear force shift (lj.cpp:439-448) up to rc_lj, Ewald real
// space (electrostatic_ewald_r.cpp:196-198) up to rc_r <= L/2 under the
// minimum image (all pairs: at rc = L/2 half of all pairs are inside, so a
// cell list would save at most 2x), Ewald k space over the reference's k-set
// (initialize.cpp:184-222) and force (electrostatic_ewald_k.cpp:197-234).
//
// Layout: FP64 positions/velocities in global memory (concatenated, SoA);
// each CTA keeps its replica's positions in shared memory as box-centred
// FP32 hi/lo pairs (x = hi + lo), so the minimum-image displacement is
// formed to ~1e-7 absolute from FP32 arithmetic; the k-space accumulation
// S(k) is FP64; energies and virial are FP64 block sums.
//
// Launch shape (threads per CTA) per replica size class is chosen by timing
// candidates on the state itself (the autotuner below), replicas start in
// decreasing size order (longest first), and the per-class launches are one
// CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/caviar_b200.h"

namespace {

constexpr int NMAX = 2048;  // atoms per replica
constexpr int KMAXB = 6;    // k_max per axis
constexpr int KP = KMAXB + 1;
constexpr int TMAX = 4;
constexpr int CH = 64;  // atoms per phase-table stage of S(k)
constexpr int NTH = 8;  // per-replica results: ke, e_lj, e_ewr, e_k, e_self, virial, temperature, steps

struct KRunB {
  int nx, ny, nz0, len, k0;
};

struct BatchDev {
  const int *order;
  const long long *off;
  const int *n;
  const double *L, *rc_lj, *rc_r;
  double *x, *y, *z, *vx, *vy, *vz;
  float *fx, *fy, *fz;  // FP32 forces of the current positions (carried between launches)
  const int *type;
  const int4 *kint;
  const KRunB *runs;
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

// erfc(x) for x >= 0 from its rational-exponential approximation
// erfc(x) = t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2), t = 1 / (1 + p x),
// absolute error below 1.5e-7 (Abramowitz & Stegun, Handbook of Mathematical
// Functions, 1964, eq. 7.1.26).  ex = exp(-x^2), which the force needs anyway.
__device__ __forceinline__ float erfc_as(float x, float ex) {
  const float t = __fdividef(1.f, fmaf(0.3275911f, x, 1.f));
  return t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f),
                  0.254829592f) * ex;
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

// Shared-memory state of one replica.
struct Smem {
  float4 *ljc;      // per type pair: sig2, eps24, eps48, K (this replica's LJ cutoff)
  float4 *lje;      // per type pair: e4, C0, C1, k_e q_i q_j
  float4 *xh, *xl;  // hi, lo of the box-centred position; type in xh.w, charge in xl.w
  float2 *ak;       // (4 pi / V) f_k conj(S_k) for the k-force
  float *fk;
  float2 *tab;      // phase tables of a stage of CH atoms
  double *red;
};

// Forces on this thread's MPT atoms (all pairs, minimum image, then k space).
// EV: energies and virial into ev[0..4] (this thread's share).
template <int TPB, int MPT, bool EV>
__device__ void batch_forces(const BatchDev &p, const Smem &S, int r, int n, double L, float3 (&f)[MPT],
                             double (&ev)[5]) {
  const float Lh = (float)L, Ll = (float)(L - (double)Lh), iL = (float)(1.0 / L);
  const float rc2 = (float)(p.rc_lj[r] * p.rc_lj[r]), rr2 = (float)(p.rc_r[r] * p.rc_r[r]);
  const float alpha = (float)p.alpha, alpha2 = alpha * alpha, tas = (float)(2.0 * p.alpha * 0.56418958354775628695);
  float4 ih[MPT], il[MPT];
#pragma unroll
  for (int m = 0; m < MPT; ++m) {
    const int i = threadIdx.x + m * TPB;
    ih[m] = (i < n) ? S.xh[i] : make_float4(0, 0, 0, 0);
    il[m] = (i < n) ? S.xl[i] : make_float4(0, 0, 0, 0);
    f[m] = make_float3(0, 0, 0);
  }
  for (int j = 0; j < n; ++j) {
    const float4 jh = S.xh[j], jl = S.xl[j];
#pragma unroll
    for (int m = 0; m < MPT; ++m) {
      const int i = threadIdx.x + m * TPB;
      if (i >= n || i == j) continue;
      float d[3];
      const float hh[3] = {jh.x - ih[m].x, jh.y - ih[m].y, jh.z - ih[m].z};
      const float ll[3] = {jl.x - il[m].x, jl.y - il[m].y, jl.z - il[m].z};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float k = rintf(hh[a] * iL);
        d[a] = fmaf(-k, Lh, hh[a]) + fmaf(-k, Ll, ll[a]);
      }
      const float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const int tp = __float_as_int(ih[m].w) * TMAX + __float_as_int(jh.w);
      const float4 lc = S.ljc[tp], le = S.lje[tp];
      float c = 0.f;
      if (r2 <= rc2 && lc.y != 0.f) {
        const float r2i = __fdividef(1.f, r2), s2 = lc.x * r2i, s6 = s2 * s2 * s2;
        c = r2i * s6 * (lc.y - lc.z * s6) + lc.w;
        if (EV) ev[0] += 0.5 * (double)(le.x * (s6 * s6 - s6) + le.z * r2 + le.y);
      }
      if (le.w != 0.f && r2 <= rr2) {
        const float rinv = rsqrtf(r2), rr = r2 * rinv;
        const float ex = __expf(-alpha2 * r2);
        const float er = erfc_as(alpha * rr, ex);
        c -= le.w * (tas * ex + er * rinv) * (rinv * rinv);
        if (EV) ev[1] += 0.5 * (double)(le.w * er * rinv);
      }
      f[m].x += c * d[0];
      f[m].y += c * d[1];
      f[m].z += c * d[2];
      if (EV) ev[4] -= 0.5 * (double)(c * r2);
    }
  }
  // ---- k space: S(k) in passes of TPB k-vectors over stages of CH atoms
  const int kmax = p.kmax;
  const double Vd = L * L * L;
  for (int k0 = 0; k0 < p.nk; k0 += TPB) {
    const int k = k0 + threadIdx.x;
    int4 kn = make_int4(0, 0, 0, 0);
    if (k < p.nk) kn = p.kint[k];
    double sr = 0, si = 0;
    for (int a0 = 0; a0 < n; a0 += CH) {
      const int na = min(CH, n - a0);
      __syncthreads();
      for (int t = threadIdx.x; t < na * 3 * KP; t += TPB) {
        const int at = t / (3 * KP), rem = t % (3 * KP), dd = rem / KP, m = rem % KP;
        float2 v = make_float2(0.f, 0.f);
        if (m <= kmax) {
          const float4 h = S.xh[a0 + at], lo = S.xl[a0 + at];
          const float hx = dd == 0 ? h.x : (dd == 1 ? h.y : h.z);
          const float lx = dd == 0 ? lo.x : (dd == 1 ? lo.y : lo.z);
          // phase of the box-centred coordinate; e^{ik.(x - L/2)} = e^{ik.x} (-1)^n
          const double u = (double)m * (((double)hx + (double)lx) / L);
          float sn, cs;
          sincospif((float)(2.0 * (u - rint(u))), &sn, &cs);
          if (m & 1) {
            sn = -sn;
            cs = -cs;
          }
          v = make_float2(cs, sn);
        }
        S.tab[t] = v;
      }
      __syncthreads();
      if (k < p.nk) {
        const int mx = abs(kn.x), my = abs(kn.y), mz = abs(kn.z);
        float pr = 0.f, pim = 0.f;
        for (int at = 0; at < na; ++at) {
          const float2 *tb = S.tab + at * 3 * KP;
          const float2 ph = cmulf(cmulf(conjf_if(tb[mx], kn.x < 0), conjf_if(tb[KP + my], kn.y < 0)),
                                  conjf_if(tb[2 * KP + mz], kn.z < 0));
          const float q = S.xl[a0 + at].w;
          pr += q * ph.x;
          pim += q * ph.y;
        }
        sr += (double)pr;
        si += (double)pim;
      }
    }
    if (k < p.nk) {
      const double fkk = (double)S.fk[k];
      const double cf = 12.56637061435917295384 / Vd * fkk;
      S.ak[k] = make_float2((float)(cf * sr), (float)(-cf * si));
      if (EV) ev[2] += 6.28318530717958647692 / Vd * p.k_e * fkk * (sr * sr + si * si);
    }
  }
  __syncthreads();
  // ---- k-force: each of this thread's atoms with its own phase table in registers
  const float tpl = (float)(6.28318530717958647692 / L);
#pragma unroll 1
  for (int m = 0; m < MPT; ++m) {
    const int i = threadIdx.x + m * TPB;
    if (i >= n) continue;
    float2 tx[KP], ty[KP], tz[KP];
    const float4 h = S.xh[i], lo = S.xl[i];
    const double pc[3] = {(double)h.x + lo.x, (double)h.y + lo.y, (double)h.z + lo.z};
#pragma unroll
    for (int mm = 0; mm < KP; ++mm) {
      float2 e[3];
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) {
        const double u = (double)mm * (pc[dd] / L);
        float sn, cs;
        sincospif((float)(2.0 * (u - rint(u))), &sn, &cs);
        if (mm & 1) {
          sn = -sn;
          cs = -cs;
        }
        e[dd] = make_float2(cs, sn);
      }
      tx[mm] = e[0];
      ty[mm] = e[1];
      tz[mm] = e[2];
    }
    float fx = 0, fy = 0, fz = 0;
    for (int rr = 0; rr < p.nruns; ++rr) {
      const KRunB run = p.runs[rr];
      float2 px = tx[0], py = ty[0];
#pragma unroll
      for (int mm = 0; mm < KP; ++mm) {
        if (mm == abs(run.nx)) px = tx[mm];
        if (mm == abs(run.ny)) py = ty[mm];
      }
      float2 pz = tz[0];
#pragma unroll
      for (int mm = 0; mm < KP; ++mm)
        if (mm == abs(run.nz0)) pz = tz[mm];
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
#pragma unroll
    for (int mm = 0; mm < MPT; ++mm)  // static indices keep f in registers
      if (mm == m) {
        f[mm].x += qk * fx;
        f[mm].y += qk * fy;
        f[mm].z += qk * fz;
      }
  }
}

// Box-centred hi/lo FP32 copy of one atom's FP64 position (wrapped into [0, L)).
__device__ __forceinline__ void to_smem(const BatchDev &p, const Smem &S, int i, long long gi, double L) {
  double c[3] = {p.x[gi], p.y[gi], p.z[gi]};
  float hv[3], lv[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double v = c[a] - 0.5 * L;
    hv[a] = (float)v;
    lv[a] = (float)(v - (double)hv[a]);
  }
  const int t = p.type[gi];
  S.xh[i] = make_float4(hv[0], hv[1], hv[2], __int_as_float(t));
  S.xl[i] = make_float4(lv[0], lv[1], lv[2], p.charge[t]);
}

// One launch: nsteps velocity-Verlet steps of replica order[first + blockIdx.x].
// compute_first = 0 takes the forces of the current positions from fx/fy/fz
// (written by the previous launch), so runs split over several launches are
// bit-identical to one run.  Energies and virial come from a separate
// evaluation at the final positions (the stepping forces never depend on
// whether energies are wanted).
template <int TPB, int MPT>
__global__ void __launch_bounds__(TPB, 1) k_batch(BatchDev p, int first, int nsteps, int nmax, int compute_first) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int r = p.order[first + blockIdx.x];
  const int n = p.n[r];
  const long long o = p.off[r];
  const double L = p.L[r];
  Smem S;
  S.ljc = reinterpret_cast<float4 *>(smraw);
  S.lje = S.ljc + TMAX * TMAX;
  S.xh = S.lje + TMAX * TMAX;
  S.xl = S.xh + nmax;
  S.ak = reinterpret_cast<float2 *>(S.xl + nmax);
  S.fk = reinterpret_cast<float *>(S.ak + p.nk);
  S.tab = reinterpret_cast<float2 *>(S.fk + ((p.nk + 3) & ~3));
  S.red = reinterpret_cast<double *>(S.tab + CH * 3 * KP);
  // LJ constants for this replica's cutoff (lj.cpp:439-448) and k_e q_i q_j
  if (threadIdx.x < TMAX * TMAX) {
    const int a = threadIdx.x / TMAX, b = threadIdx.x % TMAX, T = p.n_types;
    const bool ok = a < T && b < T;
    const float rc2 = (float)(p.rc_lj[r] * p.rc_lj[r]);
    const float e = ok ? p.eps[a * T + b] : 0.f, sg = ok ? p.sig[a * T + b] : 0.f;
    const float rcinv = 1.f / rc2, c2 = sg * sg * rcinv, c6 = c2 * c2 * c2, c12 = c6 * c6;
    const float g = 4.f * e * (12.f * c12 - 6.f * c6);
    S.ljc[threadIdx.x] = make_float4(sg * sg, 24.f * e, 48.f * e, 4.f * e * (12.f * c12 * rcinv - 6.f * c6 * rcinv));
    S.lje[threadIdx.x] = make_float4(4.f * e, -4.f * e * (c12 - c6) - 0.5f * g, g / (2.f * rc2),
                                     ok ? (float)(p.k_e * p.chargeD[a] * p.chargeD[b]) : 0.f);
  }
  // f_k = exp(-k^2 / 4 alpha^2) / k^2 for this box (initialize.cpp:201-221)
  const double tpl = 6.28318530717958647692 / L, fa = 1.0 / (4.0 * p.alpha * p.alpha);
  for (int k = threadIdx.x; k < p.nk; k += TPB) {
    const int4 kn = p.kint[k];
    const double ksq = tpl * tpl * (double)(kn.x * kn.x + kn.y * kn.y + kn.z * kn.z);
    S.fk[k] = (float)(exp(-ksq * fa) / ksq);
  }
  for (int i = threadIdx.x; i < n; i += TPB) to_smem(p, S, i, o + i, L);
  __syncthreads();
  float3 f[MPT];
  double ev[5] = {0, 0, 0, 0, 0};
  if (compute_first) {
    batch_forces<TPB, MPT, false>(p, S, r, n, L, f, ev);
  } else {
#pragma unroll
    for (int m = 0; m < MPT; ++m) {
      const int i = threadIdx.x + m * TPB;
      f[m] = (i < n) ? make_float3(p.fx[o + i], p.fy[o + i], p.fz[o + i]) : make_float3(0.f, 0.f, 0.f);
    }
  }
  const double dt = p.dt, h = 0.5 * dt;
  for (int step = 0; step < nsteps; ++step) {
    __syncthreads();
#pragma unroll
    for (int m = 0; m < MPT; ++m) {
      const int i = threadIdx.x + m * TPB;
      if (i >= n) continue;
      const long long gi = o + i;
      const double mi = p.mass_inv[p.type[gi]];
      double *X[3] = {p.x, p.y, p.z}, *V[3] = {p.vx, p.vy, p.vz};
      const float fv[3] = {f[m].x, f[m].y, f[m].z};
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
    batch_forces<TPB, MPT, false>(p, S, r, n, L, f, ev);
#pragma unroll
    for (int m = 0; m < MPT; ++m) {
      const int i = threadIdx.x + m * TPB;
      if (i >= n) continue;
      const long long gi = o + i;
      const double mi = p.mass_inv[p.type[gi]];
      p.vx[gi] += h * (double)f[m].x * mi;
      p.vy[gi] += h * (double)f[m].y * mi;
      p.vz[gi] += h * (double)f[m].z * mi;
    }
  }
  {
    __syncthreads();
    float3 fe[MPT];
    batch_forces<TPB, MPT, true>(p, S, r, n, L, fe, ev);
  }
  __syncthreads();
  // forces, kinetic energy (COM removed), energies
  double kv[9] = {0, 0, 0, 0, 0, ev[0], ev[1], ev[4], 0};
#pragma unroll
  for (int m = 0; m < MPT; ++m) {
    const int i = threadIdx.x + m * TPB;
    if (i >= n) continue;
    const long long gi = o + i;
    const double ms = p.mass[p.type[gi]];
    p.fx[gi] = f[m].x;
    p.fy[gi] = f[m].y;
    p.fz[gi] = f[m].z;
    const double v0 = p.vx[gi], v1 = p.vy[gi], v2 = p.vz[gi];
    kv[0] += ms * (v0 * v0 + v1 * v1 + v2 * v2);
    kv[1] += ms * v0;
    kv[2] += ms * v1;
    kv[3] += ms * v2;
    kv[4] += ms;
  }
  kv[8] = ev[2];  // k-space energy: each k counted by exactly one thread
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

size_t smem_bytes(int nk, int nmax) {
  return (size_t)2 * TMAX * TMAX * sizeof(float4) + (size_t)2 * nmax * sizeof(float4) + (size_t)nk * sizeof(float2) +
         (size_t)((nk + 3) & ~3) * sizeof(float) + (size_t)CH * 3 * KP * sizeof(float2) + 9 * 32 * sizeof(double);
}

using KernelFn = void (*)(BatchDev, int, int, int, int);

struct Shape {
  int tpb, mpt;
  KernelFn fn;
};

// Launch shapes per size class: (threads per CTA, atoms per thread)
const Shape kShapes[] = {
    {128, 1, k_batch<128, 1>}, {128, 2, k_batch<128, 2>}, {128, 4, k_batch<128, 4>},
    {256, 1, k_batch<256, 1>}, {256, 2, k_batch<256, 2>}, {256, 4, k_batch<256, 4>},
    {512, 1, k_batch<512, 1>}, {512, 2, k_batch<512, 2>}, {512, 4, k_batch<512, 4>},
};

}  // namespace

struct cvr_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n_rep = 0, n_types = 0;
  long long n_total = 0;
  std::vector<int> n;
  std::vector<long long> off;
  std::vector<double> L, rc_lj, rc_r;
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
  const int nmax = (c.nmax + 3) & ~3;
  s.fn<<<c.count, s.tpb, smem_bytes(b->dev.nk, nmax), st>>>(b->dev, c.first, nsteps, nmax, compute_first);
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
  b->L.assign(box_len, box_len + n_rep);
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
  if ((rc = balloc(b, &dn, n_rep)) || (rc = balloc(b, &doff, n_rep)) || (rc = balloc(b, &dorder, n_rep)) ||
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
  for (int t = 0; t < T * T; ++t) {
    b->dev.eps[t] = (float)eps[t];
    b->dev.sig[t] = (float)sigma[t];
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
          runs.push_back({a, c, z, 1, k});
      }
  b->dev.nk = (int)kint.size();
  b->dev.nruns = (int)runs.size();
  int4 *dk;
  KRunB *dr;
  if (int rc = balloc(b, &dk, kint.size())) return rc;
  if (int rc = balloc(b, &dr, runs.size())) return rc;
  cudaMemcpy(dk, kint.data(), kint.size() * sizeof(int4), cudaMemcpyHostToDevice);
  cudaMemcpy(dr, runs.data(), runs.size() * sizeof(KRunB), cudaMemcpyHostToDevice);
  b->dev.kint = dk;
  b->dev.runs = dr;
  const int sm = (int)smem_bytes(b->dev.nk, NMAX);
  for (const Shape &s : kShapes)
    if (cudaFuncSetAttribute(s.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess)
      return bfail(b, CVR_ERR_CUDA, "shared memory attribute");
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
  std::vector<double> soa(6 * N, 0.0);
  for (size_t i = 0; i < N; ++i)
    for (int a = 0; a < 3; ++a) {
      soa[a * N + i] = pos[3 * i + a];
      soa[(3 + a) * N + i] = vel ? vel[3 * i + a] : 0.0;
    }
  for (size_t i = 0; i < N; ++i)
    if (type[i] < 0 || type[i] >= b->n_types) return bfail(b, CVR_ERR_INVALID, "atom type out of range");
  cudaMemcpyAsync(b->dev.x, soa.data(), 6 * N * sizeof(double), cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync((void *)b->dev.type, type, N * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream);
  b->forces_valid = false;
  return cudaStreamSynchronize(b->stream) == cudaSuccess ? CVR_OK : bfail(b, CVR_ERR_CUDA, "upload");
}

// Autotuner: for each size class, time every shape whose atoms-per-thread
// covers the class's largest replica on 2 steps of the real state (restored
// afterwards), keep the fastest.
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
      if (s.tpb * s.mpt < c.nmax || s.tpb * s.mpt >= 4 * c.nmax + 512) continue;
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
  for (size_t i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) {
      if (pos) pos[3 * i + d] = soa[d * N + i];
      if (vel) vel[3 * i + d] = soa[(3 + d) * N + i];
      if (acc) acc[3 * i + d] = (double)a[d * N + i] * b->dev.mass_inv[t[i]];
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
    v.push_back(c.shape >= 0 ? kShapes[c.shape].mpt : 0);
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
