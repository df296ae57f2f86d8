// cvr_build.cuh -- Verlet-list build on sm_100a: PBC wrap, cell binning,
// cell-ordered re-layout, and the pair search.
//
// Replaces, in the reference (CAVIAR; paths relative to its project root):
//   Domain::fix_position                      src/caviar/objects/domain.cpp:418-468
//   exchange_ghost_single_md_domain           src/caviar/objects/atom_data/exchange_ghost_single_md_domain.cpp:26-218
//   Neighborlist::update_cell_list            src/caviar/objects/neighborlist.cpp:439-472
//   Neighborlist::update_verlet_list_from_cell_list  neighborlist.cpp:515-573
//
// The reference materialises ghost copies of atoms near the faces and bins
// owned + ghost atoms into cells of width rl.  Here no ghost is stored: an
// image is (atom j, stencil offset d), and the list entry records d.  The
// PAIR SET is nevertheless the reference's exactly: a pair (i, j, image s)
// is listed iff the reference would list it from either end -- the image of
// j exists as a reference ghost (ghost zones with the reference's
// lower-zone-first rule) and |r_i - ghost_j|^2 < rl^2 in the reference's own
// FP64 operation order, or the same with i and j swapped.  An FP32 prefilter
// on cell-local coordinates decides every candidate that is more than a
// 1e-5 relative guard band away from rl^2; the rest take the exact FP64 test.
//
// Every build kernel returns at once unless the step's rebuild flag is set,
// so the whole sequence can sit in every step of a stream or graph.
#pragma once
#include "cvr_device.cuh"

// Candidates read per round trip by the one-thread-per-atom search, and the
// minimum resident blocks it is compiled for (register budget).
#ifndef CVR_BUILD_UNROLL
#define CVR_BUILD_UNROLL 2
#endif
#ifndef CVR_BUILD_MINB
#define CVR_BUILD_MINB 8
#endif

namespace cvr {

__device__ __forceinline__ int ghost_val(double x, double gclo, double gchi, int bc) {
  // exchange_ghost_single_md_domain.cpp:59-99: lower zone first, else upper, times bc
  const int v = (x < gclo) ? -1 : ((x > gchi) ? 1 : 0);
  return v * bc;
}

// floor(a / b) for b > 0; the stencil only ever asks for -1, 0 or 1 when the
// grid has at least 2R+1 cells, so those are answered without a division.
__device__ __forceinline__ int floor_div(int a, int b) {
  if (a >= 0 && a < b) return 0;
  if (a < 0 && a >= -b) return -1;
  if (a >= b && a < 2 * b) return 1;
  const int q = a / b;
  return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

template <typename real>
__device__ __forceinline__ void cell_xyz(const DevState<real> &s, int c, int &cx, int &cy, int &cz) {
  cx = c % s.cells.nc[0];
  const int t = c / s.cells.nc[0];
  cy = t % s.cells.nc[1];
  cz = t / s.cells.nc[1];
}

// Pass 1: wrap (Domain::fix_position: one if / else-if per periodic axis),
// cell index, copy the atom to the temporaries, count atoms per cell.
template <typename real>
__global__ void k_bin_count(DevState<real> s) {
  if (*s.flag == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  double p[3] = {s.x[i], s.y[i], s.z[i]};
  int c[3];
  bool clamped = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (s.box.bc[d] == 1) {
      if (p[d] < s.box.lo[d])
        p[d] = __dadd_rn(p[d], s.box.L[d]);
      else if (p[d] > s.box.hi[d])
        p[d] = __dsub_rn(p[d], s.box.L[d]);
    }
    const double u = (p[d] - s.box.lo[d]) * s.cells.inv_w[d];
    int ci = (u >= 0.0) ? (int)fmin(u, 2.0e9) : -1;  // floor for u >= 0; NaN lands in cell 0
    clamped = clamped || ci < 0 || ci >= s.cells.nc[d];
    ci = min(max(ci, 0), s.cells.nc[d] - 1);
    c[d] = ci;
  }
  // an atom outside its cell's slab: the search must not clip rows by cell geometry
  if (clamped) *s.clamp_mark = *s.build_epoch + 1;
  const int cell = c[0] + s.cells.nc[0] * (c[1] + s.cells.nc[1] * c[2]);
  s.tx[i] = p[0];
  s.ty[i] = p[1];
  s.tz[i] = p[2];
  s.tvx[i] = s.vx[i];
  s.tvy[i] = s.vy[i];
  s.tvz[i] = s.vz[i];
  s.tid[i] = s.id[i];
  s.ttype[i] = s.type[i];
  s.tmol[i] = s.mol[i];
  s.tcell[i] = cell;
  atomicAdd(&s.cell_count[cell], 1);
}

// Exclusive scan of cell_count into cell_start, in three passes over blocks
// of 1024 cells.  cell_start[ncells] = n.
__device__ __forceinline__ int block_exclusive_scan_1024(int v, int *warp_tot, int &block_total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  block_total = warp_tot[31];
  const int before = (warp > 0) ? warp_tot[warp - 1] : 0;
  return before + x - v;
}

__global__ void __launch_bounds__(1024) k_scan_local(const int *__restrict__ flag, const int *__restrict__ in,
                                                      int *__restrict__ out, int *__restrict__ block_sums, int m) {
  if (*flag == 0) return;
  __shared__ int wt[32];
  const int i = blockIdx.x * 1024 + threadIdx.x;
  const int v = (i < m) ? in[i] : 0;
  int tot;
  const int ex = block_exclusive_scan_1024(v, wt, tot);
  if (i < m) out[i] = ex;
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_sums(const int *__restrict__ flag, int *__restrict__ block_sums, int nb,
                                                     int *__restrict__ total_out, int *__restrict__ build_epoch) {
  if (*flag == 0) return;
  if (threadIdx.x == 0) *build_epoch += 1;  // after k_bin_count, before the list search
  __shared__ int wt[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = (i < nb) ? block_sums[i] : 0;
    int tot;
    const int ex = block_exclusive_scan_1024(v, wt, tot);
    if (i < nb) block_sums[i] = ex + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total_out = carry;
}

__global__ void __launch_bounds__(1024) k_scan_add(const int *__restrict__ flag, int *__restrict__ out,
                                                    const int *__restrict__ block_sums, int m) {
  if (*flag == 0) return;
  const int i = blockIdx.x * 1024 + threadIdx.x;
  if (i < m) out[i] += block_sums[blockIdx.x];
}

// Pass 2: drop each atom into its cell's range (order inside a cell is
// fixed by k_rank below, so the atomics here do not make the result depend
// on scheduling).
template <typename real>
__global__ void k_bin_scatter(DevState<real> s) {
  if (*s.flag == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const int c = s.tcell[i];
  const int slot = s.cell_start[c] + atomicAdd(&s.cell_fill[c], 1);
  s.slot_atom[slot] = i;
}

// Pass 3: inside each cell, order atoms by id (deterministic layout).
template <typename real>
__global__ void k_rank(DevState<real> s) {
  if (*s.flag == 0) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= s.n) return;
  const int i = s.slot_atom[t];
  const int c = s.tcell[i];
  const int b = s.cell_start[c], e = s.cell_start[c + 1];
  const int key = s.tid[i];
  int rank = 0;
  for (int u = b; u < e; ++u) rank += (s.tid[s.slot_atom[u]] < key) ? 1 : 0;
  s.perm[b + rank] = i;
}

// Pass 4: gather into cell order, build the cell-local coordinates and the
// ghost-zone classification, and clear the per-cell counters for next time.
template <typename real>
__global__ void k_permute(DevState<real> s) {
  if (*s.flag == 0) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < s.cells.ncells) {
    s.cell_count[k] = 0;
    s.cell_fill[k] = 0;
  }
  if (k >= s.n) return;
  const int i = s.perm[k];
  const double p[3] = {s.tx[i], s.ty[i], s.tz[i]};
  s.x[k] = p[0];
  s.y[k] = p[1];
  s.z[k] = p[2];
  s.vx[k] = s.tvx[i];
  s.vy[k] = s.tvy[i];
  s.vz[k] = s.tvz[i];
  s.id[k] = s.tid[i];
  const int ty = s.ttype[i];
  s.type[k] = ty;
  s.mol[k] = s.tmol[i];
  const int c = s.tcell[i];
  s.cell[k] = c;
  int cc[3];
  cell_xyz(s, c, cc[0], cc[1], cc[2]);
  double loc[3];
  int code = 0, mul = 1;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double origin = s.box.lo[d] + (cc[d] + 0.5) * s.cells.w[d];
    loc[d] = p[d] - origin;
    code += (ghost_val(p[d], s.box.gclo[d], s.box.gchi[d], s.box.bc[d]) + 1) * mul;
    mul *= 3;
  }
  typename V4<real>::t q;
  q.x = (real)loc[0];
  q.y = (real)loc[1];
  q.z = (real)loc[2];
  if constexpr (sizeof(real) == 4) {
    q.w = __int_as_float(ty);
    if (s.fixed) {
      q.x = fixed_coord(p[0], s.fx_scale);
      q.y = fixed_coord(p[1], s.fx_scale);
      q.z = fixed_coord(p[2], s.fx_scale);
    }
  } else {
    q.w = (double)ty;
  }
  s.x4[k] = q;
  s.xb[k] = make_float4((float)(p[0] - s.box.ctr[0]), (float)(p[1] - s.box.ctr[1]), (float)(p[2] - s.box.ctr[2]),
                        __int_as_float(cc[0]));
  s.gcls[k] = (int8_t)code;
}

// |pa - image(pb, shift)|^2 < rl^2 in the reference's FP64 order:
// ghost = pb - val*L on shifted axes (val = -shift), dr = pa - ghost,
// dr.dr = (dx*dx + dy*dy) + dz*dz, no fused multiply-add.
__device__ __forceinline__ bool exact_within(const double pa[3], const double pb[3], const int sh[3], const DBox &b,
                                             double rl_sq) {
  double dr[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double g = sh[d] ? __dsub_rn(pb[d], __dmul_rn((double)(-sh[d]), b.L[d])) : pb[d];
    dr[d] = __dsub_rn(pa[d], g);
  }
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dr[0], dr[0]), __dmul_rn(dr[1], dr[1])), __dmul_rn(dr[2], dr[2]));
  return r2 < rl_sq;
}

// Does atom a (ghost-zone code gc) have a reference ghost at image shift sh?
__device__ __forceinline__ bool has_image(int gcode, const int sh[3]) {
  int v[3];
  v[0] = gcode % 3 - 1;
  v[1] = (gcode / 3) % 3 - 1;
  v[2] = gcode / 9 - 1;
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (sh[d] != 0 && v[d] != -sh[d]) return false;
  return true;
}

// The pair search's per-candidate test.  The FP32 prefilter works on
// box-centred coordinates: d = (xb_j + s L) - xb_i, with the image shift s
// folded into per-row constants b = s L - xb_i, so a candidate costs three
// adds and a dot product.  Candidates outside rl^2 (1 + band) are rejected;
// candidates inside rl^2 (1 - band) are accepted at once when there is no
// image shift, or when the geometry is regular (rl <= ghost_cutoff <= L/2 on
// every periodic axis: then both atoms of a pair clearly inside rl across a
// face lie in the ghost zones, so the reference has the ghost image).  The
// band is sized on the host from the FP32 rounding of the box coordinates.
// Everything else takes the reference's exact FP64 test and ghost-image rules.
template <typename real>
__device__ __forceinline__ bool in_list_slow(const DevState<real> &s, const double (&pi)[3], int gi, int j, float d2,
                                          int sx, int sy, int sz) {
  const int sh[3] = {sx, sy, sz};
  if ((sx | sy | sz) == 0) {
    const double pj[3] = {s.x[j], s.y[j], s.z[j]};
    return exact_within(pi, pj, sh, s.box, s.rl_sq);
  }
  const int gj = s.gcls[j];
  const int msh[3] = {-sx, -sy, -sz};
  const bool img_j = has_image(gj, sh);   // reference ghost of j at r_j + sL
  const bool img_i = has_image(gi, msh);  // reference ghost of i at r_i - sL
  if (!img_j && !img_i) return false;
  if (d2 <= s.rl_sq_lo) return true;
  const double pj[3] = {s.x[j], s.y[j], s.z[j]};
  return (img_j && exact_within(pi, pj, sh, s.box, s.rl_sq)) || (img_i && exact_within(pj, pi, msh, s.box, s.rl_sq));
}

__device__ __forceinline__ uint32_t list_entry(int j, int dx, int dy, int dz, int R, int S) {
  (void)S;
  return (uint32_t)j | ((uint32_t)(dx + R) << CODE_SHIFT) | ((uint32_t)(dy + R) << (CODE_SHIFT + 3)) |
         ((uint32_t)(dz + R) << (CODE_SHIFT + 6));
}

__device__ __forceinline__ size_t list_slot(int cnt, int log2_tpa, size_t stride) {
  return (size_t)(cnt >> log2_tpa) * stride + (size_t)(cnt & ((1 << log2_tpa) - 1));
}


// The same search with one WARP per atom, for systems too small to fill the
// GPU with one thread per atom: the 32 lanes take consecutive candidates of a
// stencil cell, and a ballot keeps the accepted ones in candidate order, so
// the list is identical to the one-thread-per-atom build.  Launched with 128
// threads (four warps: the per-warp piece tables); a register cap rather than
// launch bounds keeps the sweep free of spills.
template <typename real>
__global__ void __maxnreg__(80) k_build_list_warp(DevState<real> s, int count_only, int log2_tpa) {
  if (*s.flag == 0) return;
  if (blockIdx.x == 0 && threadIdx.x == 0 && !count_only) atomicAdd(s.n_builds, 1);
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= s.n) return;  // whole warp leaves together
  int cx, cy, cz;
  cell_xyz(s, s.cell[i], cx, cy, cz);
  const float4 xi = s.xb[i];
  const double pi[3] = {s.x[i], s.y[i], s.z[i]};
  const int gi = s.gcls[i];
  const int R = s.cells.R, S = s.cells.S;
  const size_t stride = (size_t)s.n_pad << log2_tpa;
  uint32_t *row = s.nlist + ((size_t)i << log2_tpa);
  const int nc0 = s.cells.nc[0], nc1 = s.cells.nc[1], nc2 = s.cells.nc[2];
  const unsigned lt = (1u << lane) - 1u;
  int cnt = 0;
  if (nc0 >= S) {
    // Row mode: the stencil's S*S rows (dz, dy), each at most three
    // contiguous atom ranges (the sx = -1, 0, +1 pieces of the unwrapped x
    // range [cx-R, cx+R]).  The lanes first load every piece's range in one
    // parallel round trip, then the warp sweeps the pieces in stencil order,
    // 32 candidates at a time (the same entries, in the same order, as the
    // cell-by-cell sweep below).
    constexpr int KP = (3 * (2 * MAX_STENCIL_R + 1) * (2 * MAX_STENCIL_R + 1) + 31) / 32;
    const int P = 3 * S * S;
    // Each row is clipped to the cells that meet the rl sphere around atom i:
    // with g_y, g_z the atom's distances to the row's y and z slabs, only
    // cells within h = sqrt(rl^2 - g_y^2 - g_z^2) of it in x can hold a
    // listed candidate.  Widened by a margin far above the FP32 rounding of
    // these few operations (gaps shrunk and h grown by 1e-3 of a cell, rl^2
    // taken at the top of the prefilter band), the clip only drops cells
    // from the two ends of a row range, so every atom keeps the same entries
    // in the same order.  f = the atom's place in its cell.  The clip needs
    // every atom inside its cell's slab, which binning breaks only when it
    // clamps a coordinate outside the box into an edge cell; such a build
    // searches whole rows.
    const float wx = (float)s.cells.w[0], wy = (float)s.cells.w[1], wz = (float)s.cells.w[2];
    const float ivx = (float)s.cells.inv_w[0];
    const float fx = (float)(pi[0] - s.box.lo[0] - cx * s.cells.w[0]);
    const float fy = (float)(pi[1] - s.box.lo[1] - cy * s.cells.w[1]);
    const float fz = (float)(pi[2] - s.box.lo[2] - cz * s.cells.w[2]);
    const float dlt = 1e-3f * fminf(wx, fminf(wy, wz));
    const float rc2 = s.rl_sq_hi;
    const bool clip = *s.clamp_mark != *s.build_epoch;
    // per piece: first candidate, length, and the list-entry bits of the
    // piece (dy, dz fields and cell_x(j) + dxc + R in the dx field, less
    // cell_x(j); wrapping 32-bit arithmetic, exact once cell_x(j) is added)
    // with the image shift (sx + 1) | (sy + 1) << 2 | (sz + 1) << 4 in the
    // low bits (the j field, zero in the entry bits)
    int pst[KP], plen[KP];
    uint32_t pcode[KP];
#pragma unroll
    for (int k = 0; k < KP; ++k) {
      const int p = 32 * k + lane;
      pst[k] = 0;
      plen[k] = 0;
      pcode[k] = 0;
      if (p < P) {
        const int r = p / 3, sx = p % 3 - 1;
        const int dz = r / S - R, dy = r % S - R;
        const int sz = floor_div(cz + dz, nc2), sy = floor_div(cy + dy, nc1);
        const float gy = fmaxf(fmaxf(dy * wy - fy, fy - (dy + 1) * wy) - dlt, 0.f);
        const float gz = fmaxf(fmaxf(dz * wz - fz, fz - (dz + 1) * wz) - dlt, 0.f);
        const float h2 = rc2 - gy * gy - gz * gz;
        int ua = cx - R, ub = cx + R;
        if (clip && !(h2 >= 0.f)) {
          ua = 1;  // the row misses the sphere
          ub = 0;
        } else if (clip) {
          const float hx = sqrtf(h2) + dlt;
          ua = cx + max(-R, min(R + 1, __float2int_rd((fx - hx) * ivx)));
          ub = cx + min(R, max(-R - 1, __float2int_rd((fx + hx) * ivx)));
        }
        if (sx < 0) ub = min(ub, -1);
        if (sx == 0) {
          ua = max(ua, 0);
          ub = min(ub, nc0 - 1);
        }
        if (sx > 0) ua = max(ua, nc0);
        const bool live = ua <= ub && (sz == 0 || s.box.bc[2]) && (sy == 0 || s.box.bc[1]) && (sx == 0 || s.box.bc[0]);
        if (live) {
          const int rowbase = nc0 * (cy + dy - sy * nc1 + nc1 * (cz + dz - sz * nc2));
          pst[k] = s.cell_start[rowbase + ua - sx * nc0];
          plen[k] = s.cell_start[rowbase + ub - sx * nc0 + 1] - pst[k];
          const int dxc = sx * nc0 - cx;  // dx = cell_x(j) + dxc
          pcode[k] = (list_entry(0, 0, dy, dz, R, S) + (uint32_t)dxc * (1u << CODE_SHIFT)) |
                     (uint32_t)((sx + 1) | ((sy + 1) << 2) | ((sz + 1) << 4));
        }
      }
    }
    // The live pieces, in stencil order, laid end to end: a per-warp table
    // in shared memory of each piece's start in that sequence, first
    // candidate, image offset and entry bits.  The warp then sweeps the
    // sequence 32 candidates at a time, so a round spans piece boundaries
    // instead of idling the lanes past the end of a short row.
    constexpr uint32_t kUnshifted = 1u | (1u << 2) | (1u << 4);
    constexpr int PMAX = 3 * (2 * MAX_STENCIL_R + 1) * (2 * MAX_STENCIL_R + 1);
    __shared__ int s_off[4][PMAX + 1];
    __shared__ float4 s_geo[4][PMAX];  // image offset bx, by, bz; first candidate (int bits)
    __shared__ uint32_t s_pc[4][PMAX];
    const int w = threadIdx.x >> 5;
    int nlive = 0, total = 0;
#pragma unroll
    for (int k = 0; k < KP; ++k) {
      const int len = plen[k];
      int incl = len;  // inclusive scan of the lengths across the lanes
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      const unsigned live = __ballot_sync(0xffffffffu, len > 0);
      if (len > 0) {
        const int q = nlive + __popc(live & lt);
        const uint32_t code = pcode[k] & 63u;
        const int sx = (int)(code & 3u) - 1, sy = (int)((code >> 2) & 3u) - 1, sz = (int)(code >> 4) - 1;
        s_off[w][q] = total + incl - len;
        s_geo[w][q] = make_float4(sx * s.box.Lf[0] - xi.x, sy * s.box.Lf[1] - xi.y, sz * s.box.Lf[2] - xi.z,
                                  __int_as_float(pst[k]));
        s_pc[w][q] = pcode[k];
      }
      nlive += __popc(live);
      total += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) s_off[w][nlive] = total;
    __syncwarp();
    int q0 = 0;  // the live piece that holds candidate `base`
    for (int base = 0; base < total; base += 32) {
      // pieces that start inside this round (after its first candidate)
      const int qt = q0 + 1 + lane;
      unsigned bit = 0u;
      if (qt < nlive) {
        const int o = s_off[w][qt];
        if (o < base + 32) bit = 1u << (o - base);
      }
      const unsigned starts = __reduce_or_sync(0xffffffffu, bit);
      const int c = base + lane;
      bool ok = false;
      int j = 0;
      float4 q = xi;
      uint32_t pc = 0;
      if (c < total) {
        const int qp = q0 + __popc(starts & ((2u << lane) - 1u));  // this lane's piece
        const float4 g = s_geo[w][qp];
        pc = s_pc[w][qp];
        j = __float_as_int(g.w) + (c - s_off[w][qp]);
        const uint32_t code = pc & 63u;
        const bool shifted = code != kUnshifted;
        if (!shifted ? j != i : true) {
          q = s.xb[j];
          const float ex = q.x + g.x, ey = q.y + g.y, ez = q.z + g.z;
          const float d2 = ex * ex + ey * ey + ez * ez;
          if (d2 < s.rl_sq_hi) {
            const bool fast_ok = !shifted || s.regular_images;
            ok = (d2 <= s.rl_sq_lo && fast_ok) ||
                 in_list_slow(s, pi, gi, j, d2, (int)(code & 3u) - 1, (int)((code >> 2) & 3u) - 1, (int)(code >> 4) - 1);
          }
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (ok && !count_only) {
        const int k2 = cnt + __popc(m & lt);
        const uint32_t ebase = pc & ~((1u << CODE_SHIFT) - 1u);
        if (k2 < s.cap)
          row[list_slot(k2, log2_tpa, stride)] = (uint32_t)j | (ebase + ((uint32_t)__float_as_int(q.w) << CODE_SHIFT));
      }
      cnt += __popc(m);
      q0 += __popc(starts);  // the piece that holds candidate base + 32
      if (q0 + 1 < nlive && s_off[w][q0 + 1] <= base + 32) ++q0;
    }
  } else
  for (int dz = -R; dz <= R; ++dz) {
    const int sz = floor_div(cz + dz, nc2);
    if (sz != 0 && !s.box.bc[2]) continue;
    const int jz = cz + dz - sz * nc2;
    const float bz = sz * s.box.Lf[2] - xi.z;
    for (int dy = -R; dy <= R; ++dy) {
      const int sy = floor_div(cy + dy, nc1);
      if (sy != 0 && !s.box.bc[1]) continue;
      const int jy = cy + dy - sy * nc1;
      const float by = sy * s.box.Lf[1] - xi.y;
      const int rowbase = nc0 * (jy + nc1 * jz);
      for (int dx = -R; dx <= R; ++dx) {
        const int sx = floor_div(cx + dx, nc0);
        if (sx != 0 && !s.box.bc[0]) continue;
        const float bx = sx * s.box.Lf[0] - xi.x;
        const bool shifted = (sx | sy | sz) != 0;
        const bool fast_ok = !shifted || s.regular_images;
        const int self = shifted ? -1 : i;
        const int cj = cx + dx - sx * nc0 + rowbase;
        const int jb = s.cell_start[cj], je = s.cell_start[cj + 1];
        for (int base = jb; base < je; base += 32) {
          const int j = base + lane;
          bool ok = false;
          if (j < je && j != self) {
            const float4 q = s.xb[j];
            const float ex = q.x + bx, ey = q.y + by, ez = q.z + bz;
            const float d2 = ex * ex + ey * ey + ez * ez;
            if (d2 < s.rl_sq_hi) ok = (d2 <= s.rl_sq_lo && fast_ok) || in_list_slow(s, pi, gi, j, d2, sx, sy, sz);
          }
          const unsigned m = __ballot_sync(0xffffffffu, ok);
          if (ok && !count_only) {
            const int k = cnt + __popc(m & lt);
            if (k < s.cap) row[list_slot(k, log2_tpa, stride)] = list_entry(j, dx, dy, dz, R, S);
          }
          cnt += __popc(m);
        }
      }
    }
  }
  if (lane == 0) {
    if (!count_only) s.ncount[i] = min(cnt, s.cap);
    if (!count_only && cnt > s.cap) atomicOr(s.err, ERR_OVERFLOW);
    atomicMax(s.max_count, cnt);
  }
}

// Pass 5: the pair search, one thread per atom over the (2R+1)^3 stencil.
// Each stencil row (fixed dy, dz) is at most two contiguous atom ranges (a
// periodic wrap in x splits it); candidates are read CVR_BUILD_UNROLL at a
// time, and a candidate's cell x index comes from xb.w.  Rows of boxes
// narrower than the stencil (nc_x < 2R+1) take the cell-by-cell path.
// With one lane per atom the list interleave is 4 (log2_tpa = 2): the pair
// kernel reads an atom's entries four at a time.  count_only = 1 only counts (used to size the list before
// the first build).
template <typename real>
__global__ void __launch_bounds__(128, CVR_BUILD_MINB) k_build_list(DevState<real> s, int count_only, int log2_tpa) {
  if (*s.flag == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x == 0 && threadIdx.x == 0 && !count_only) atomicAdd(s.n_builds, 1);
  int cnt = 0;
  if (i < s.n) {
    int cx, cy, cz;
    cell_xyz(s, s.cell[i], cx, cy, cz);
    const float4 xi = s.xb[i];
    const double pi[3] = {s.x[i], s.y[i], s.z[i]};
    const int gi = s.gcls[i];
    const int R = s.cells.R, S = s.cells.S;
    const size_t stride = (size_t)s.n_pad << log2_tpa;
    uint32_t *row = s.nlist + ((size_t)i << log2_tpa);
    const int nc0 = s.cells.nc[0], nc1 = s.cells.nc[1], nc2 = s.cells.nc[2];
    const float lo2 = s.rl_sq_lo, hi2 = s.rl_sq_hi;
    for (int dz = -R; dz <= R; ++dz) {
      const int sz = floor_div(cz + dz, nc2);
      if (sz != 0 && !s.box.bc[2]) continue;
      const int jz = cz + dz - sz * nc2;
      const float bz = sz * s.box.Lf[2] - xi.z;
      for (int dy = -R; dy <= R; ++dy) {
        const int sy = floor_div(cy + dy, nc1);
        if (sy != 0 && !s.box.bc[1]) continue;
        const int jy = cy + dy - sy * nc1;
        const float by = sy * s.box.Lf[1] - xi.y;
        const int rowbase = nc0 * (jy + nc1 * jz);
        const int parts = (nc0 >= S) ? 3 : S;
        for (int part = 0; part < parts; ++part) {
          // row mode: parts are the sx = -1, 0, +1 pieces of the unwrapped x
          // range [cx-R, cx+R]; cell mode: one stencil cell per part
          int sx, ca, cb, dxc;
          if (nc0 >= S) {
            sx = part - 1;
            int ua = cx - R, ub = cx + R;
            if (sx < 0) ub = min(ub, -1);
            if (sx == 0) {
              ua = max(ua, 0);
              ub = min(ub, nc0 - 1);
            }
            if (sx > 0) ua = max(ua, nc0);
            if (ua > ub) continue;
            ca = ua - sx * nc0;
            cb = ub - sx * nc0;
            dxc = sx * nc0 - cx;  // dx = cell_x(j) + dxc
          } else {
            const int dx = part - R;
            sx = floor_div(cx + dx, nc0);
            ca = cb = cx + dx - sx * nc0;
            dxc = dx - ca;
          }
          if (sx != 0 && !s.box.bc[0]) continue;
          const float bx = sx * s.box.Lf[0] - xi.x;
          const bool shifted = (sx | sy | sz) != 0;
          const bool fast_ok = !shifted || s.regular_images;
          const int self = shifted ? -1 : i;
          const int jb = s.cell_start[rowbase + ca];
          const int je = s.cell_start[rowbase + cb + 1];
          for (int j = jb; j < je; j += CVR_BUILD_UNROLL) {
            float4 q[CVR_BUILD_UNROLL];
#pragma unroll
            for (int u = 0; u < CVR_BUILD_UNROLL; ++u) q[u] = (j + u < je) ? s.xb[j + u] : xi;
#pragma unroll
            for (int u = 0; u < CVR_BUILD_UNROLL; ++u) {
              const int jj = j + u;
              const float ex = q[u].x + bx, ey = q[u].y + by, ez = q[u].z + bz;
              const float d2 = ex * ex + ey * ey + ez * ez;
              if (jj < je && jj != self && d2 < hi2) {
                const bool inc = (d2 <= lo2 && fast_ok) || in_list_slow(s, pi, gi, jj, d2, sx, sy, sz);
                if (inc) {
                  if (!count_only && cnt < s.cap)
                    row[list_slot(cnt, log2_tpa, stride)] = list_entry(jj, __float_as_int(q[u].w) + dxc, dy, dz, R, S);
                  ++cnt;
                }
              }
            }
          }
        }
      }
    }
    if (!count_only) {
      s.ncount[i] = min(cnt, s.cap);
      if (cnt > s.cap) atomicOr(s.err, ERR_OVERFLOW);
    }
  }
  // largest count, one atomic per warp
  int m = cnt;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(s.max_count, m);
}

}  // namespace cvr
