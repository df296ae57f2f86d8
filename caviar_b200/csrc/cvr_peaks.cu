// cvr_peaks.cu -- arithmetic-pipe peaks of the GPU this library runs on, for
// the compute side of the roofline (the HBM side is a measured copy).
//
// One kernel per precision issues independent fused multiply-adds and
// nothing else: every thread runs kChains dependency chains (enough to hide
// the FMA latency at full occupancy) for `iters` rounds, and the grid fills
// every SM with full blocks several times over.  One FMA counts as 2 flops.
// The chains are combined and stored only if the result equals an impossible
// value, so the compiler keeps every FMA and the kernel writes nothing.
#include <cuda_runtime.h>

#include "../../include/caviar_b200.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kThreads) k_fma_peak(T *sink, int iters, T b, T c) {
  T a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = (T)(threadIdx.x + k) * (T)1e-3;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
    }
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == (T)-1.2345e-30) sink[threadIdx.x] = s;  // never true for these inputs
}

template <typename T>
int measure(int device, int iters, double *tflops, double *ms_out) {
  if (cudaSetDevice(device) != cudaSuccess) return CVR_ERR_CUDA;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CVR_ERR_CUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_peak<T>, kThreads, 0) != cudaSuccess)
    return CVR_ERR_CUDA;
  const int blocks = prop.multiProcessorCount * (per_sm > 0 ? per_sm : 1) * 4;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return CVR_ERR_CUDA;
  T *sink = nullptr;  // a real buffer, although the kernels never store to it
  if (cudaMalloc(&sink, kThreads * sizeof(T)) != cudaSuccess) {
    cudaStreamDestroy(st);
    return CVR_ERR_NOMEM;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // b < 1 and c small keep every chain finite (each tends to c / (1 - b) = 0.1)
  const T b = (T)0.999, c = (T)1e-4;
  k_fma_peak<T><<<blocks, kThreads, 0, st>>>(sink, iters / 8 + 1, b, c);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0, st);
    k_fma_peak<T><<<blocks, kThreads, 0, st>>>(sink, iters, b, c);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(sink);
  if (e != cudaSuccess) return CVR_ERR_CUDA;
  const double flops = 2.0 * kChains * 16.0 * (double)iters * (double)blocks * kThreads;
  if (tflops) *tflops = flops / (best * 1e-3) / 1e12;
  if (ms_out) *ms_out = best;
  return CVR_OK;
}

}  // namespace

extern "C" int cvr_measure_fma_peak(int device, int fp64, int iters, double *tflops, double *ms) {
  if (iters <= 0) return CVR_ERR_INVALID;
  return fp64 ? measure<double>(device, iters, tflops, ms) : measure<float>(device, iters, tflops, ms);
}
