// Allocation-free GAP energies.
//
// e[r] = sum_n alpha_n (A_r . B_n)^zeta for FP32 device matrices A [M x K]
// and B [N x K], computed with the tcgen05 BF16x3 GEMM and its fused GAP
// epilogue (gemm_tc.cu) in its energies-only form. Every scratch buffer (the
// BF16 hi/lo splits of A and B and the per-tile energy partials) is carved
// out of one file-scope device array, and the bounded-wait status word is a
// second one, so a call never allocates device memory. It is for callers
// that must not allocate or free device memory inside a call, such as an MD
// engine's force callback running beside the engine's own kernels:
// cudaMalloc and cudaFree synchronise the whole device and would stall them.
//
// Setup: the first call on a device (with that device current) looks the
// two arrays up with cudaGetSymbolAddress and keeps their addresses for the
// life of the process. A cudaDeviceReset after that first call is not
// supported: the kept addresses would belong to the destroyed context.
// Concurrency: all calls share the one array, so calls that overlap in time
// (from several host threads or streams) race; callers serialise them.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "common.cuh"
#include "rgpu_internal.h"

namespace rgpu {
namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;  // 16 MiB

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];
static __device__ __align__(16) int g_status[4];

struct DevicePointers {
  unsigned char * scratch = nullptr;
  int * status = nullptr;
};
PerDevice<DevicePointers> g_ptrs;

// Addresses of the two arrays on the current device, looked up once.
DevicePointers setup_current_device() {
  return g_ptrs.once(current_device(), [](DevicePointers & p) {
    void * s = nullptr;
    void * w = nullptr;
    RGPU_CUDA(cudaGetSymbolAddress(&s, g_scratch));
    RGPU_CUDA(cudaGetSymbolAddress(&w, g_status));
    p.status = static_cast<int *>(w);
    p.scratch = static_cast<unsigned char *>(s);
  });
}

__global__ void sum_parts_kernel(const float * __restrict__ parts, int n_parts, int64_t M, float * __restrict__ e) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= M) return;
  float s = 0.f;
  for (int t = 0; t < n_parts; ++t) s += parts[int64_t(t) * M + r];
  e[r] = s;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

void gap_energies_noalloc(int64_t M, int64_t N, int64_t K, const float * A, const float * B, const float * alpha,
                          int zeta, float * e, cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !alpha || !e)
    throw Error(RGPU_ERR_INVALID_ARGUMENT, "bad arguments: sizes must be positive and pointers non-null");
  if (zeta < 1) throw Error(RGPU_ERR_INVALID_ARGUMENT, "zeta must be >= 1");
  auto too_big = [&](const std::string & why) {
    return Error(RGPU_ERR_CAPACITY, "GAP energies without allocation: M=" + std::to_string(M) + ", N=" +
                                        std::to_string(N) + ", K=" + std::to_string(K) + " " + why +
                                        ", above the static " + std::to_string(kScratchBytes) +
                                        " bytes of scratch");
  };
  // Each of M, N and K alone bounds a scratch term from below (4 M Kp, 4 N Kp
  // and 4 M bytes), so one beyond the array's size is rejected before any
  // product is formed; the products below then stay far inside 64 bits.
  if (M > int64_t(kScratchBytes) || N > int64_t(kScratchBytes) || K > int64_t(kScratchBytes))
    throw too_big("exceed the scratch on their own");
  const int64_t Kp = (K + 63) / 64 * 64;
  const int n_parts = int((N + kTcTileN - 1) / kTcTileN);
  // scratch layout: A hi, A lo, B hi, B lo, energy partials (the epilogue
  // runs in its energies-only form, so W needs no space)
  const size_t a_bytes = align256(size_t(M) * Kp * 2), b_bytes = align256(size_t(N) * Kp * 2);
  const size_t p_bytes = align256(size_t(n_parts) * M * 4);
  const size_t need = 2 * a_bytes + 2 * b_bytes + p_bytes;
  if (need > kScratchBytes) throw too_big("need " + std::to_string(need) + " bytes");
  const DevicePointers p = setup_current_device();
  unsigned char * s = p.scratch;
  __nv_bfloat16 * ah = reinterpret_cast<__nv_bfloat16 *>(s);
  __nv_bfloat16 * al = reinterpret_cast<__nv_bfloat16 *>(s + a_bytes);
  __nv_bfloat16 * bh = reinterpret_cast<__nv_bfloat16 *>(s + 2 * a_bytes);
  __nv_bfloat16 * bl = reinterpret_cast<__nv_bfloat16 *>(s + 2 * a_bytes + b_bytes);
  float * parts = reinterpret_cast<float *>(s + 2 * a_bytes + 2 * b_bytes);
  // Only the status word must start at zero: the splits write every padded
  // column and the epilogue every partial that is read.
  RGPU_CUDA(cudaMemsetAsync(p.status, 0, 2 * sizeof(int), st));
  split_bf16(A, M, K, K, ah, al, Kp, st);
  split_bf16(B, N, K, K, bh, bl, Kp, st);
  Bf16x3Gemm g{};
  g.M = M;
  g.N = N;
  g.K = Kp;
  g.A_hi = ah;
  g.A_lo = al;
  g.lda = Kp;
  g.B_hi = bh;
  g.B_lo = bl;
  g.ldb = Kp;
  g.epilogue = 1;
  g.W_hi = nullptr;  // energies only
  g.W_lo = nullptr;
  g.ldw = 0;
  g.alpha = alpha;
  g.zeta = zeta;
  g.e_part = parts;
  gemm_bf16x3_status(g, p.status, st);
  sum_parts_kernel<<<div_up(M, 256), 256, 0, st>>>(parts, n_parts, M, e);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
  int status[2] = {0, 0};
  RGPU_CUDA(cudaMemcpyAsync(status, p.status, sizeof(status), cudaMemcpyDeviceToHost, st));
  RGPU_CUDA(cudaStreamSynchronize(st));
  if (status[0])
    throw Error(RGPU_ERR_TIMEOUT, "tensor-core GEMM: a bounded pipeline wait gave up (stage " +
                                      std::to_string(status[1]) + ")");
}

}  // namespace rgpu
