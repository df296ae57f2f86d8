// cvr_device.cuh -- device-side state shared by the sm_100a kernels.
//
// HBM layout (one periodic system, atoms kept in CELL ORDER, re-sorted at each
// Verlet-list build):
//   x,y,z / vx,vy,vz   FP64 SoA positions (unwrapped between builds) and velocities
//   ax,ay,az           real SoA accelerations (real = float in the mixed form, double in FP64)
//   x4                 real4 cell-local position (r - centre of the atom's build cell) with the
//                      type in .w: the only per-neighbour gather of the pair kernel (16 B mixed);
//                      in the mixed form's fixed-point mode (cubic box, see DevState::fixed) .x-.z
//                      hold the bits of u = round(r * 2^32 / L) mod 2^32 instead
//   xb                 float4 cell-local position at the last build (rebuild trigger)
//   cell,id,type,mol   int per atom; id = the caller's atom index
//   nlist              uint32 entries: atom j in bits 0-22, stencil offset dx+R, dy+R, dz+R
//                      in 3-bit fields at bits 23, 26, 29; TPA-interleaved rows:
//                      entry k of atom i at (k/TPA)*(n_pad*TPA) + i*TPA + k%TPA
//   ncount             neighbours per atom
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cvr {

enum : int { ERR_NAN = 1, ERR_OVERFLOW = 2, ERR_GEOMETRY = 4, ERR_KSPACE_TC = 8 };
constexpr int CODE_SHIFT = 23;  // first of the three 3-bit stencil-offset fields
constexpr unsigned INDEX_MASK = (1u << CODE_SHIFT) - 1u;
constexpr int MAX_STENCIL_R = 3;  // dx + R must fit in 3 bits
constexpr int MAX_TYPES = 16;
constexpr int MAX_KMAX = 31;

template <typename real> struct V4;
template <> struct V4<float> { using t = float4; };
template <> struct V4<double> { using t = double4; };

struct DBox {
  double lo[3], hi[3], L[3];
  double gclo[3], gchi[3];  // lower + ghost_cutoff, upper - ghost_cutoff (ghost zones)
  double ctr[3];            // box centre: origin of the FP32 coordinates the list search uses
  float Lf[3];
  int bc[3];
};

struct DCells {
  int nc[3];
  int ncells;
  int R;  // stencil radius in cells
  int S;  // 2R+1
  double w[3], inv_w[3];
};

// Per type-pair constants of the fused pair kernel.
template <typename real> struct PairCoef {
  real sig2, eps24, eps48, K;  // LJ: c = r2inv*s6*(eps24 - eps48*s6) + K
  real rc2;                    // LJ cutoff^2 (lj.cpp:417-420); < 0 disables LJ for the pair
  real qq;                     // k_e q_i q_j (Ewald real space)
  real e4, C0, C1;             // LJ energy: e4*(s6^2 - s6) + C1*r2 + C0
  real lam;                    // Ewald same-molecule scaling lambda (1 if unset)
  real jump2;                  // LJ jump_tol: r^2 floor of the coefficient and virial (0: off)
};

template <typename real> struct DevState {
  int n, n_pad, cap, tpa, policy, n_types;
  DBox box;
  DCells cells;
  double rl_sq;                 // (cutoff*coef)^2, FP64 list threshold
  float rl_sq_lo, rl_sq_hi;     // FP32 guard band around rl_sq for the prefilter
  float thr_sq;                 // (skin/2)^2 rebuild threshold
  int regular_images;           // rl <= ghost_cutoff <= L/2 on every periodic axis: every image pair
                                // clearly inside rl has its reference ghost (no per-pair image test)
  int fixed;                    // mixed form only: x4 holds 32-bit fixed-point coordinates, so a pair's
                                // minimum-image displacement is one wrapping int32 subtraction per axis
  double fx_scale;              // 2^32 / L (fixed-point units per length; cubic box)
  double *x, *y, *z, *vx, *vy, *vz;
  real *ax, *ay, *az;
  typename V4<real>::t *x4;
  float4 *xb;  // box-centred FP32 position at the last build, cell x index in .w (list search, rebuild trigger)
  int *cell, *id, *type, *mol;
  int8_t *gcls;                 // ghost-zone classification at build (x_val+1)+3(y_val+1)+9(z_val+1)
  // rebuild temporaries
  double *tx, *ty, *tz, *tvx, *tvy, *tvz;
  int *tid, *ttype, *tmol, *tcell;
  int *cell_count, *cell_start, *cell_fill, *slot_atom, *perm, *block_sums;
  // list
  uint32_t *nlist;
  int *ncount;
  // device flags
  int *flag;       // rebuild requested for this step
  int *err;        // sticky ERR_* bits
  int *max_count;  // largest neighbour count at the last build
  int *n_builds;
  int *build_epoch;  // advanced once per build (k_scan_sums)
  int *clamp_mark;   // build_epoch + 1 when that build's binning clamped a coordinate into an edge cell
  double *mass_inv;  // per type (device)
  double *mass;      // per type (device)
};

// erfc(x) for x >= 0 from its rational-exponential approximation
// erfc(x) = t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2), t = 1 / (1 + p x),
// absolute error below 1.5e-7 (Abramowitz & Stegun, Handbook of Mathematical
// Functions, 1964, eq. 7.1.26).  ex = exp(-x^2), which the Ewald real-space
// force needs anyway.  Used by the FP32 (mixed) kernels only.
__device__ __forceinline__ float erfc_as(float x, float ex) {
  const float t = __fdividef(1.f, fmaf(0.3275911f, x, 1.f));
  return t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f),
                  0.254829592f) * ex;
}

// 32-bit fixed-point coordinate u = round(p * 2^32 / L) mod 2^32.  The
// difference of two such coordinates, read as a signed int32, is the
// minimum-image displacement in units of L / 2^32 whenever the true
// displacement is below L / 2 (the wrap of the integer is the periodic wrap).
__device__ __forceinline__ float fixed_coord(double p, double scale) {
  return __uint_as_float((uint32_t)(unsigned long long)__double2ll_rn(p * scale));
}

}  // namespace cvr
