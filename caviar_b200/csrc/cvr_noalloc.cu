// cvr_noalloc.cu -- Ewald structure factor S(k) for callers that cannot
// allocate device memory.
//
// Who needs this: code that runs inside a host program whose allocator owns
// the GPU's memory (a framework with a caching allocator or an MD engine
// that reserves its pool up front) and may not ask the CUDA runtime for more,
// plug-ins that are forbidden to allocate after start-up, and callers that
// cannot afford the device-wide synchronisation cudaMalloc/cudaFree imply in
// the middle of their own work.  They own their input and output buffers;
// this entry point brings no buffer of its own.
//
// The per-chunk partial sums the two kernels exchange live in the file-scope
// array g_sk_scratch below instead of a cudaMalloc'd buffer.  It holds
// CVR_NOALLOC_SK_SCRATCH complex doubles (4 MiB) on every GPU that loads the
// library, for the life of the process.  Host code may not use the symbol
// g_sk_scratch as a device address (in host code it names a host-side stand-in):
// the first call on each device looks up the real address with
// cudaGetSymbolAddress, with that device current, and passes it to the
// kernels.  Make that first call before any stream capture.  The address is
// kept per device ordinal for the rest of the process, so the entry point must
// not be used again on a device after cudaDeviceReset (the module is loaded
// anew there and the kept address no longer names the array).
//
// Every call on a device shares the one array, and the array keeps the last
// call's contents.  Each call writes every partial it later reads, so nothing
// needs clearing, but two calls whose kernels overlap on the GPU (different
// streams, no ordering between them) race on the array and give wrong sums.
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/caviar_b200.h"

namespace {

constexpr int kMaxDevices = 64;
constexpr int kChunkAtoms = 64;  // atoms per shared-memory stage
constexpr int kThreads = 256;    // k-vectors per block
constexpr int kMaxK = 30;        // largest k_max per axis

// k_max <= 30 on every axis gives at most (2*30)^3 = 216000 k-vectors, one
// partial each per chunk; the array holds at least one chunk of them.
static_assert(8 * kMaxK * kMaxK * kMaxK <= CVR_NOALLOC_SK_SCRATCH, "scratch must hold one chunk at k_max 30");

// Dynamic shared memory of k_sk_noalloc_partial at k_max 30 (the largest any
// call needs): phase tables of one stage of atoms plus their charges.
constexpr size_t kMaxSmem = (size_t)kChunkAtoms * 3 * (kMaxK + 1) * 16 + kChunkAtoms * sizeof(double);

__device__ __align__(256) double2 g_sk_scratch[CVR_NOALLOC_SK_SCRATCH];

std::mutex g_lock;
double2 *g_scratch_ptr[kMaxDevices] = {nullptr};

// Index k of the used k-set -> (nx, ny, nz): the reference enumerates
// kx, ky, kz over [-kmax, kmax] (kz fastest), skips k = 0, and keeps the
// first (2kx)(2ky)(2kz) vectors (electrostatic_ewald_k/initialize.cpp:184-222).
__device__ __forceinline__ int3 k_index_to_n(int k, int kx, int ky, int kz) {
  const int ny_span = 2 * ky + 1, nz_span = 2 * kz + 1;
  const int zero = kx * ny_span * nz_span + ky * nz_span + kz;  // position of (0,0,0)
  const int m = (k < zero) ? k : k + 1;
  int3 r;
  r.x = m / (ny_span * nz_span) - kx;
  r.y = (m / nz_span) % ny_span - ky;
  r.z = m % nz_span - kz;
  return r;
}

// Partial S(k) over the atoms of one chunk (a multiple of kChunkAtoms atoms),
// one thread per k-vector; phase tables e^{i 2 pi m x_d / L_d} of a stage of
// atoms sit in shared memory.  FP64 throughout.
__global__ void __launch_bounds__(kThreads) k_sk_noalloc_partial(const double *__restrict__ pos,
                                                                 const double *__restrict__ q, int n, int chunk_atoms,
                                                                 double3 inv_L, int kx, int ky, int kz, int nk,
                                                                 double2 *__restrict__ partial) {
  extern __shared__ double2 tab[];  // [kChunkAtoms][3][kp] + charges
  const int kp = max(kx, max(ky, kz)) + 1;
  double *qs = reinterpret_cast<double *>(tab + kChunkAtoms * 3 * kp);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  int3 nv = make_int3(0, 0, 0);
  if (k < nk) nv = k_index_to_n(k, kx, ky, kz);
  const int mx = abs(nv.x), my = abs(nv.y), mz = abs(nv.z);
  double sr = 0.0, si = 0.0;
  const int a_begin = blockIdx.y * chunk_atoms;
  const int a_end = min(n, a_begin + chunk_atoms);
  for (int s0 = a_begin; s0 < a_end; s0 += kChunkAtoms) {
    const int na = min(kChunkAtoms, a_end - s0);
    __syncthreads();
    for (int t = threadIdx.x; t < kChunkAtoms * 3 * kp; t += blockDim.x) {
      const int at = t / (3 * kp), rem = t % (3 * kp), d = rem / kp, m = rem % kp;
      double2 v = make_double2(0.0, 0.0);
      if (at < na) {
        const double x = pos[3 * (size_t)(s0 + at) + d];
        const double il = (d == 0) ? inv_L.x : ((d == 1) ? inv_L.y : inv_L.z);
        const double u = (double)m * (x * il);
        double sn, cs;
        sincospi(2.0 * (u - rint(u)), &sn, &cs);
        v = make_double2(cs, sn);
      }
      tab[t] = v;
    }
    for (int t = threadIdx.x; t < kChunkAtoms; t += blockDim.x) qs[t] = (t < na) ? q[s0 + t] : 0.0;
    __syncthreads();
    if (k < nk) {
      for (int a = 0; a < na; ++a) {
        const double2 *tb = tab + a * 3 * kp;
        double2 px = tb[mx], py = tb[kp + my], pz = tb[2 * kp + mz];
        if (nv.x < 0) px.y = -px.y;
        if (nv.y < 0) py.y = -py.y;
        if (nv.z < 0) pz.y = -pz.y;
        const double2 pxy = make_double2(px.x * py.x - px.y * py.y, px.x * py.y + px.y * py.x);
        const double pr = pxy.x * pz.x - pxy.y * pz.y, pi = pxy.x * pz.y + pxy.y * pz.x;
        sr += qs[a] * pr;
        si += qs[a] * pi;
      }
    }
  }
  if (k < nk) partial[(size_t)blockIdx.y * nk + k] = make_double2(sr, si);
}

// S(k) = sum of the chunk partials, in chunk order.
__global__ void __launch_bounds__(kThreads) k_sk_noalloc_reduce(const double2 *__restrict__ partial, int nchunks,
                                                                int nk, double *__restrict__ sk) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  double sr = 0.0, si = 0.0;
  for (int c = 0; c < nchunks; ++c) {
    const double2 p = partial[(size_t)c * nk + k];
    sr += p.x;
    si += p.y;
  }
  sk[2 * (size_t)k] = sr;
  sk[2 * (size_t)k + 1] = si;
}

int say(char *err, size_t len, int code, const char *msg) {
  if (err && len) std::snprintf(err, len, "%s", msg);
  return code;
}

}  // namespace

extern "C" int cvr_structure_factor_noalloc(const double *pos, const double *q, int64_t n, const double box_len[3],
                                            int kx_max, int ky_max, int kz_max, double *sk, void *stream, char *err,
                                            size_t err_len) {
  if (err && err_len) err[0] = '\0';
  if (!pos || !q || !sk || !box_len || n <= 0 || n > (int64_t)1 << 30)
    return say(err, err_len, CVR_ERR_INVALID, "pos, q, sk, box_len must be non-null and 0 < n <= 2^30");
  if (kx_max < 0 || ky_max < 0 || kz_max < 0 || kx_max > kMaxK || ky_max > kMaxK || kz_max > kMaxK)
    return say(err, err_len, CVR_ERR_INVALID, "k_max per axis must be in [0, 30]");
  for (int d = 0; d < 3; ++d)
    if (!(box_len[d] > 0)) return say(err, err_len, CVR_ERR_INVALID, "box lengths must be positive");
  const int nk = (2 * kx_max) * (2 * ky_max) * (2 * kz_max);  // <= 216000, see kMaxK
  if (nk == 0) return CVR_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return say(err, err_len, CVR_ERR_CUDA, "no usable current CUDA device");
  double2 *scratch = nullptr;
  {
    std::lock_guard<std::mutex> g(g_lock);
    if (!g_scratch_ptr[dev]) {
      // Set-up, once per device with that device current: the array's device
      // address, and the kernel's shared-memory limit for the largest k_max
      // (set once here, so that concurrent calls never lower it for each other).
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_sk_scratch);
      if (e != cudaSuccess) return say(err, err_len, CVR_ERR_CUDA, cudaGetErrorString(e));
      e = cudaFuncSetAttribute(k_sk_noalloc_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem);
      if (e != cudaSuccess) return say(err, err_len, CVR_ERR_CUDA, cudaGetErrorString(e));
      g_scratch_ptr[dev] = static_cast<double2 *>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  // Chunks of whole stages; as many as the scratch holds, enough blocks to fill the GPU.
  const int64_t stages = (n + kChunkAtoms - 1) / kChunkAtoms;
  int64_t max_chunks = CVR_NOALLOC_SK_SCRATCH / nk;
  if (max_chunks > 65535) max_chunks = 65535;
  const int64_t want_chunks = stages < 64 ? stages : 64;
  const int64_t nchunks_target = want_chunks < max_chunks ? want_chunks : max_chunks;
  const int64_t stages_per_chunk = (stages + nchunks_target - 1) / nchunks_target;
  const int chunk_atoms = (int)(stages_per_chunk * kChunkAtoms);
  const int nchunks = (int)((n + chunk_atoms - 1) / chunk_atoms);
  const int kp = (kx_max > ky_max ? (kx_max > kz_max ? kx_max : kz_max) : (ky_max > kz_max ? ky_max : kz_max)) + 1;
  const size_t smem = (size_t)kChunkAtoms * 3 * kp * sizeof(double2) + kChunkAtoms * sizeof(double);  // <= kMaxSmem
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double3 inv_L = make_double3(1.0 / box_len[0], 1.0 / box_len[1], 1.0 / box_len[2]);
  dim3 g1((nk + kThreads - 1) / kThreads, nchunks);
  k_sk_noalloc_partial<<<g1, kThreads, smem, st>>>(pos, q, (int)n, chunk_atoms, inv_L, kx_max, ky_max, kz_max, nk,
                                                   scratch);
  k_sk_noalloc_reduce<<<(nk + kThreads - 1) / kThreads, kThreads, 0, st>>>(scratch, nchunks, nk, sk);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return say(err, err_len, CVR_ERR_CUDA, cudaGetErrorString(e));
  return CVR_OK;
}
