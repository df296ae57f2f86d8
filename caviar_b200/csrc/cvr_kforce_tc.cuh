// cvr_kforce_tc.cuh -- the k-space force of the mixed form on the
// 5th-generation tensor cores (tcgen05, sm_100a).
//
// F_i = k_e q_i sum_k k Im(A_k e^{i k.r_i}) (electrostatic_ewald_k.cpp:
// 215-218), column-regrouped as in k_kforce: for the (nx, ny) column c,
//   C = sum_m (A+ z_m + A- conj z_m),  D = sum_m m (A+ z_m - A- conj z_m),
// and F += (nx, ny) Im(P C), F_z += Im(P D) with P = X[nx] Y[ny].
// The m-sums are a contraction over k = (Re z_m, Im z_m):
//   D[atom][(c, s)] = sum_k Z[atom][k] B[(c, s)][k],  s in {Cx, Cy, Dx, Dy},
// one MMA chain per tile of 64 columns (N = 256) for 128 atoms (M = 128).
// TF32 keeps 10 mantissa bits, so both operands are split into TF32 hi and
// lo halves and each term takes hi hi + hi lo + lo hi (the dropped lo lo
// and the halves' own rounding sit near 2^-22 relative): FP32-level sums.
//
// Blocks come in clusters of two per 128 atoms: rank r takes the column
// tiles r, r + 2, ..., and rank 1 hands its partial forces to rank 0 through
// distributed shared memory (added in a fixed order), so 126 SMs work on
// 8000 atoms.  No block leaves before the cluster barrier.
// Block: 128 atoms (TMEM lane = atom) and 16 warps: warp w reads the lanes
// of atoms 32 (w % 4) .. + 31 (the TMEM lane quarter it may access) and
// the columns of quarter w / 4 of every tile, so four warps share an atom
// and hide each other's latency; their partial forces are added in quarter
// order at the end (deterministic).  Z (hi, lo), the atoms' X, Y phase
// rows for m = -kmax .. kmax (conjugates included) and per column the two
// row offsets and (nx, ny) as floats are built in shared memory, so a
// column costs one broadcast load, two table loads and ten flops in the
// epilogue; B tiles (hi + lo,
// 48 KB) arrive by bulk copy from the image k_sk_reduce writes, two buffers
// deep.  Thread 0 issues the MMAs of tile j + 1 into the second TMEM
// accumulator (2 x 256 columns) while the warps read tile j (tcgen05.ld, 32
// columns at a time) and fold it into their atoms' forces.  Every wait is
// bounded: a wait that runs out sets ERR_KSPACE_TC, the block waits
// (bounded) for what it has in flight, frees TMEM and leaves the
// accelerations untouched.
#pragma once

#include "cvr_force.cuh"

namespace cvr {

constexpr int KTC_A_BYTES = KTC_ATOMS * KTC_K * 4;        // one Z half
constexpr int KTC_B_BYTES = 2 * KTC_TILE_FLOATS * 4;      // one B tile, hi + lo
constexpr int KTC_OFF_AHI = 0;
constexpr int KTC_OFF_ALO = KTC_A_BYTES;
constexpr int KTC_OFF_B0 = 2 * KTC_A_BYTES;
constexpr int KTC_OFF_B1 = KTC_OFF_B0 + KTC_B_BYTES;
constexpr int KTC_PROWS = 2 * KTC_KPMAX - 1;              // phase rows m = -kmax .. kmax per axis
constexpr int KTC_OFF_TAB = KTC_OFF_B1 + KTC_B_BYTES;    // X rows then Y rows, atom-minor
constexpr int KTC_TAB_BYTES = 2 * KTC_PROWS * KTC_ATOMS * 8;
constexpr int KTC_MAXCOLS = KTC_PROWS * KTC_PROWS;                      // (nx, ny) columns at most
constexpr int KTC_OFF_XY = KTC_OFF_TAB + KTC_TAB_BYTES;                 // per column: X, Y row offsets, nx, ny
constexpr int KTC_OFF_RED = KTC_OFF_XY + KTC_MAXCOLS * 16;               // partial forces [3][3][128]
constexpr int KTC_OFF_PEER = KTC_OFF_RED + 9 * KTC_ATOMS * 4;           // rank 1's forces [3][128] (rank 0)
constexpr int KTC_OFF_BAR = KTC_OFF_PEER + 3 * KTC_ATOMS * 4;           // 4 mbarriers, TMEM slot, error words
constexpr int KTC_SMEM = KTC_OFF_BAR + 64;
constexpr int KTC_THREADS = 4 * KTC_ATOMS;                               // 16 warps
constexpr int KTC_QCOLS = KTC_COLS / 4;                                  // columns per warp and tile
constexpr int KTC_TMEM_COLS = 2 * KTC_N;                  // two accumulators
constexpr int KTC_SPIN = 1 << 20;                         // mbarrier polls before giving up
// instruction descriptor: D F32, A and B TF32, both K-major, N = 256, M = 128
constexpr uint32_t KTC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(KTC_N >> 3) << 17) |
                               ((uint32_t)(KTC_ATOMS >> 4) << 24);
static_assert(KTC_N % 16 == 0 && KTC_N <= 256 && KTC_K % 8 == 0, "MMA shape");
static_assert(KTC_OFF_BAR % 8 == 0 && KTC_SMEM <= 227 * 1024, "shared memory plan");

__device__ __forceinline__ uint32_t ktc_smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major without swizzle: start address,
// leading (K) core-matrix stride 128 bytes, stride (8-row group) KTC_K / 4 *
// 128 bytes, descriptor version 1.
__device__ __forceinline__ uint64_t ktc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)((KTC_K / 4 * 128) >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void ktc_mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void ktc_mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool ktc_mbar_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < KTC_SPIN; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// bulk copy global -> shared, completing on an mbarrier (no multicast)
__device__ __forceinline__ void ktc_bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void ktc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void ktc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// D (TMEM) = / += A (smem) B (smem)^T, issued by one thread
__device__ __forceinline__ void ktc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(KTC_IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}
// the mbarrier gets one arrival when every MMA this thread issued so far is done
__device__ __forceinline__ void ktc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// 32 consecutive accumulator columns of this thread's lane (and the wait for them)
__device__ __forceinline__ void ktc_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}

// kick_h != 0: the second half kick follows, as in k_kforce.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(KTC_THREADS, 1)
    k_kforce_tc(DevState<float> s, KArgs<float> a, int ntiles, double kick_h, long long *__restrict__ counters) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int al = 32 * (warp & 3) + lane;  // this thread's atom within the block (= TMEM lane)
  const int qtr = warp >> 2;              // its quarter of each tile's columns
  uint32_t rank;
  asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
  if (kick_h != 0.0 && blockIdx.x == 0 && t == 0) {
    *s.flag = 0;
    if (counters) counters[0]++;
  }
  const uint32_t sb = ktc_smem_u32(sm);
  // buffer b (local tile parity): copy-done barrier, MMA-done barrier, B tile
  auto bar_full = [&](int b) { return sb + KTC_OFF_BAR + 8u * (uint32_t)b; };
  auto bar_done = [&](int b) { return sb + KTC_OFF_BAR + 16u + 8u * (uint32_t)b; };
  auto b_tile = [&](int b) { return sb + KTC_OFF_B0 + (uint32_t)(b * KTC_B_BYTES); };
  volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(sm + KTC_OFF_BAR + 32);
  volatile int *err_word = reinterpret_cast<volatile int *>(sm + KTC_OFF_BAR + 36);
  volatile int *peer_ok = reinterpret_cast<volatile int *>(sm + KTC_OFF_BAR + 40);
  // one reading of the error word for the whole block; no block leaves
  // early (both blocks of the cluster must reach its barrier)
  if (t == 0) {
    *err_word = *s.err | ((sb & 127u) ? ERR_KSPACE_TC : 0);
    ktc_mbar_init(bar_full(0));
    ktc_mbar_init(bar_full(1));
    ktc_mbar_init(bar_done(0));
    ktc_mbar_init(bar_done(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool skip = *err_word != 0;
  // this block's tiles: rank, rank + 2, ... (local index jj, tile j = rank + 2 jj)
  const int nloc = skip ? 0 : (ntiles - (int)rank + 1) / 2;
  const int i = (blockIdx.x >> 1) * KTC_ATOMS + al;
  const bool valid = i < s.n;
  int copies = 0, issued = 0, copies_waited = 0, waited = 0;  // thread 0's pipeline counts
  bool bad = false;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  if (!skip) {
    if (t == 0)
      for (; copies < 2 && copies < nloc; ++copies) {
        ktc_mbar_expect_tx(bar_full(copies), KTC_B_BYTES);
        ktc_bulk_load(b_tile(copies), a.kimg + (size_t)(rank + 2 * copies) * 2 * KTC_TILE_FLOATS, KTC_B_BYTES,
                      bar_full(copies));
      }
    // Z of each atom (k = 2m, 2m + 1), TF32 hi and lo (quarter 0); the X
    // (quarter 1) and Y (quarter 2) phase rows; the column list (quarter 3)
    if (qtr == 0) {
      float *ahi = reinterpret_cast<float *>(sm + KTC_OFF_AHI), *alo = reinterpret_cast<float *>(sm + KTC_OFF_ALO);
      float2 z[KTC_K / 2];
#pragma unroll
      for (int m = 0; m < KTC_K / 2; ++m) {
        z[m] = make_float2(0.f, 0.f);
        if (valid && m < a.M) z[m] = a.ptab[(size_t)(2 * a.kp + m) * s.n + i];
      }
#pragma unroll
      for (int m = 0; m < KTC_K / 2; ++m) {
        const float hx = to_tf32(z[m].x), hy = to_tf32(z[m].y);
        const int o = ktc_off(al, 2 * m) / 4;
        *reinterpret_cast<float2 *>(ahi + o) = make_float2(hx, hy);
        *reinterpret_cast<float2 *>(alo + o) = make_float2(to_tf32(z[m].x - hx), to_tf32(z[m].y - hy));
      }
    } else if (qtr < 3) {
      const int d = qtr - 1;  // 0: X rows, 1: Y rows; row KTC_KPMAX - 1 + m holds e^{i 2 pi m x_d / L_d}
      float2 *tab = reinterpret_cast<float2 *>(sm + KTC_OFF_TAB) + d * KTC_PROWS * KTC_ATOMS;
      float2 x[KTC_KPMAX];
#pragma unroll
      for (int m = 0; m < KTC_KPMAX; ++m) {
        x[m] = make_float2(0.f, 0.f);
        if (valid && m <= a.kmax[d]) x[m] = a.ptab[(size_t)(d * a.kp + m) * s.n + i];
      }
#pragma unroll
      for (int m = 0; m < KTC_KPMAX; ++m) {
        tab[(KTC_KPMAX - 1 + m) * KTC_ATOMS + al] = x[m];
        if (m > 0) tab[(KTC_KPMAX - 1 - m) * KTC_ATOMS + al] = make_float2(x[m].x, -x[m].y);
      }
    } else {
      float4 *xy = reinterpret_cast<float4 *>(sm + KTC_OFF_XY);
      for (int c = t - 3 * KTC_ATOMS; c < a.ncomp; c += KTC_ATOMS) {  // the summed columns
        const int2 nn = a.xyc[c];
        const int ox = (KTC_KPMAX - 1 + nn.x) * KTC_ATOMS * 8, oy = (KTC_PROWS + KTC_KPMAX - 1 + nn.y) * KTC_ATOMS * 8;
        xy[c] = make_float4(__int_as_float(ox), __int_as_float(oy), (float)nn.x, (float)nn.y);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // Z visible to the tensor core
    if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sb + KTC_OFF_BAR + 32),
                   "r"(KTC_TMEM_COLS)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    ktc_fence_before();
    __syncthreads();
    ktc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // thread 0: the MMA chain of local tile jj into accumulator jj & 1
    auto issue = [&](int jj) {
      const uint32_t bb = b_tile(jj & 1), d = tmem + (uint32_t)((jj & 1) * KTC_N);
#pragma unroll
      for (int ks = 0; ks < KTC_K / 8; ++ks) {
        const uint64_t ah = ktc_desc(sb + KTC_OFF_AHI + 256 * ks), alo = ktc_desc(sb + KTC_OFF_ALO + 256 * ks);
        const uint64_t bh = ktc_desc(bb + 256 * ks), bl = ktc_desc(bb + KTC_TILE_FLOATS * 4 + 256 * ks);
        ktc_mma(d, ah, bh, ks > 0 ? 1u : 0u);
        ktc_mma(d, ah, bl, 1u);
        ktc_mma(d, alo, bh, 1u);
      }
      ktc_commit(bar_done(jj & 1));
      ++issued;
    };
    if (t == 0 && nloc > 0) {
      if (ktc_mbar_wait(bar_full(0), 0)) {
        ++copies_waited;
        ktc_fence_after();
        issue(0);
      } else {
        bad = true;
      }
    }
    const unsigned char *tab_al = sm + KTC_OFF_TAB + 8 * al;  // this atom's column of the phase rows
    const float4 *xy = reinterpret_cast<const float4 *>(sm + KTC_OFF_XY);
    for (int jj = 0; jj < nloc; ++jj) {
      if (t == 0 && !bad && jj + 1 < nloc) {
        if (ktc_mbar_wait(bar_full((jj + 1) & 1), ((jj + 1) >> 1) & 1)) {
          ++copies_waited;
          ktc_fence_after();
          issue(jj + 1);
        } else {
          bad = true;
        }
      }
      // thread 0's issue status first, so that no thread waits on a chain never issued
      bool ok = !__syncthreads_or(bad) && ktc_mbar_wait(bar_done(jj & 1), (jj >> 1) & 1);
      if (__syncthreads_or(!ok)) {
        bad = true;
        break;
      }
      ++waited;
      // local tile jj's B buffer is free: fetch local tile jj + 2 into it
      if (t == 0 && jj + 2 < nloc) {
        ktc_mbar_expect_tx(bar_full(jj & 1), KTC_B_BYTES);
        ktc_bulk_load(b_tile(jj & 1), a.kimg + (size_t)(rank + 2 * (jj + 2)) * 2 * KTC_TILE_FLOATS, KTC_B_BYTES,
                      bar_full(jj & 1));
        ++copies;
      }
      ktc_fence_after();
      const uint32_t tb =
          tmem + (uint32_t)((jj & 1) * KTC_N + 4 * KTC_QCOLS * qtr) + ((uint32_t)(32 * (warp & 3)) << 16);
      const int c0 = (int)(rank + 2 * jj) * KTC_COLS + KTC_QCOLS * qtr;
      for (int q = 0; q < KTC_QCOLS / 8; ++q) {
        if (c0 + 8 * q >= a.ncomp) break;
        uint32_t r[32];
        ktc_ld32(tb + 32 * q, r);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int c = c0 + 8 * q + u;
          if (c < a.ncomp) {
            const float4 ci = xy[c];
            const float2 X = *reinterpret_cast<const float2 *>(tab_al + __float_as_int(ci.x));
            const float2 Y = *reinterpret_cast<const float2 *>(tab_al + __float_as_int(ci.y));
            const float2 P = cmul(X, Y);
            const float Cx = __uint_as_float(r[4 * u]), Cy = __uint_as_float(r[4 * u + 1]);
            const float Dx = __uint_as_float(r[4 * u + 2]), Dy = __uint_as_float(r[4 * u + 3]);
            const float tt = P.x * Cy + P.y * Cx;
            fx += ci.z * tt;
            fy += ci.w * tt;
            fz += P.x * Dy + P.y * Dx;
          }
        }
      }
      ktc_fence_before();
      __syncthreads();
    }
    if (bad && t == 0) {
      // wait (bounded) for the MMA chains and copies still in flight before freeing their memory
      for (int jj = waited; jj < issued; ++jj) ktc_mbar_wait(bar_done(jj & 1), (jj >> 1) & 1);
      for (int jj = copies_waited; jj < copies; ++jj) ktc_mbar_wait(bar_full(jj & 1), (jj >> 1) & 1);
      atomicOr(s.err, ERR_KSPACE_TC);
    }
    ktc_fence_before();
    bad = __syncthreads_or(bad);  // one answer for the whole block
    if (warp == 0) {
      ktc_fence_after();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(KTC_TMEM_COLS) : "memory");
    }
  }
  const bool good = !skip && !bad;
  // the quarters' partial forces, added in quarter order
  float *red = reinterpret_cast<float *>(sm + KTC_OFF_RED);
  if (qtr > 0) {
    red[((qtr - 1) * 3 + 0) * KTC_ATOMS + al] = fx;
    red[((qtr - 1) * 3 + 1) * KTC_ATOMS + al] = fy;
    red[((qtr - 1) * 3 + 2) * KTC_ATOMS + al] = fz;
  }
  __syncthreads();
  if (qtr == 0) {
#pragma unroll
    for (int h = 0; h < 3; ++h) {
      fx += red[(h * 3 + 0) * KTC_ATOMS + al];
      fy += red[(h * 3 + 1) * KTC_ATOMS + al];
      fz += red[(h * 3 + 2) * KTC_ATOMS + al];
    }
  }
  // rank 1's tiles join rank 0's in rank 0's shared memory
  if (rank == 1) {
    uint32_t peer;
    asm("mapa.shared::cluster.u32 %0, %1, 0;" : "=r"(peer) : "r"(sb + KTC_OFF_PEER));
    if (qtr == 0) {
      asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(peer + 4u * al), "f"(fx) : "memory");
      asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(peer + 4u * (KTC_ATOMS + al)), "f"(fy) : "memory");
      asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(peer + 4u * (2 * KTC_ATOMS + al)), "f"(fz) : "memory");
    }
    if (t == 0) {
      uint32_t pok;
      asm("mapa.shared::cluster.u32 %0, %1, 0;" : "=r"(pok) : "r"(sb + KTC_OFF_BAR + 40));
      asm volatile("st.shared::cluster.s32 [%0], %1;" ::"r"(pok), "r"(good ? 1 : 0) : "memory");
    }
  }
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
  if (rank != 0 || qtr != 0 || !valid || !good || !*peer_ok) return;
  const float *pf = reinterpret_cast<const float *>(sm + KTC_OFF_PEER);
  fx += pf[al];
  fy += pf[KTC_ATOMS + al];
  fz += pf[2 * KTC_ATOMS + al];
  const int ti = s.type[i];
  const float qm = (float)(a.k_e * a.charge[ti] * s.mass_inv[ti]);
  s.ax[i] += qm * a.two_pi_over_L[0] * fx;
  s.ay[i] += qm * a.two_pi_over_L[1] * fy;
  s.az[i] += qm * a.two_pi_over_L[2] * fz;
  if (kick_h != 0.0) {
    s.vx[i] = s.vx[i] + kick_h * (double)s.ax[i];
    s.vy[i] = s.vy[i] + kick_h * (double)s.ay[i];
    s.vz[i] = s.vz[i] + kick_h * (double)s.az[i];
  }
}

}  // namespace cvr
