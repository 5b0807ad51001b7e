// Measured FMA throughput of the CUDA cores (FP32 and FP64 pipes).
//
// The roofline fractions of the per-centre kernels (expansion, power
// spectrum, pair adjoint, FP64 tile GEMM) need the pipe peaks of the GPU
// they run on, under its own clocks and power cap, not datasheet figures.
// This microbenchmark fills every SM with independent FMA chains (eight per
// thread, enough to cover the pipe latency at full occupancy) and times the
// launch with CUDA events on a private stream; one FMA counts as 2 flops.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"

namespace rgpu {
namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chains_kernel(T * __restrict__ out, int iters, T a, T b) {
  T x0 = T(threadIdx.x) * T(1e-3), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
  T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      x0 = fma(x0, a, b);
      x1 = fma(x1, a, b);
      x2 = fma(x2, a, b);
      x3 = fma(x3, a, b);
      x4 = fma(x4, a, b);
      x5 = fma(x5, a, b);
      x6 = fma(x6, a, b);
      x7 = fma(x7, a, b);
    }
  }
  const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  // a data-dependent store the compiler cannot drop (a = 1, b = 0 in use,
  // so s stays finite and this branch is never taken)
  if (s == T(-1.2345e30)) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename T>
double time_fma(int iters) {
  int dev = current_device(), sms = 0, per_sm = 0;
  RGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fma_chains_kernel<T>, 256, 0));
  const int blocks = sms * std::max(per_sm, 1);
  cudaStream_t st = nullptr;
  RGPU_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  DevBuf out;
  double best = 0.;
  try {
    RGPU_CUDA(cudaEventCreate(&e0));
    RGPU_CUDA(cudaEventCreate(&e1));
    out.ensure(sizeof(T) * size_t(blocks) * 256);
    const double flops = 2.0 * 64.0 * double(iters) * double(blocks) * 256.0;
    for (int rep = 0; rep < 6; ++rep) {  // the first launch warms up
      RGPU_CUDA(cudaEventRecord(e0, st));
      fma_chains_kernel<T><<<blocks, 256, 0, st>>>(out.as<T>(), iters, T(1), T(0));
      RGPU_LAUNCHED();
      RGPU_CUDA(cudaGetLastError());
      RGPU_CUDA(cudaEventRecord(e1, st));
      RGPU_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      RGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0 && ms > 0.f) best = std::max(best, flops / (double(ms) * 1e-3) / 1e12);
    }
  } catch (...) {
    cudaStreamSynchronize(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  return best;
}

}  // namespace

double measure_fma_peak(int precision) {
  return precision == RGPU_PRECISION_FP64 ? time_fma<double>(4096) : time_fma<float>(8192);
}

}  // namespace rgpu
