// FP64 tile GEMM on the CUDA cores: C[r][c] = sum_k A[r][k] B(k, c), with
// the A rows addressed through a row-offset functor (plain strided rows, or
// rows gathered from a list) and the result handed to an epilogue functor
// (a plain store, or the scaled scatter of the sparse-kernel gradient
// block). B is either N x K row-major (B_NT, C = A B^T) or K x N row-major.
//
// Tile 128 x BN x 8 (BN = 128 or 64), 256 threads in a 16 x 16 grid.
// Thread (ty, tx) owns rows 32 g + 2 ty + {0, 1}, g = 0..3, and columns
// 32 g + 2 tx + {0, 1}, g < BN / 32, so every shared-memory read is a
// 16-byte vector and the 16 column pairs of a warp are contiguous (no bank
// conflicts). The next k-slice is loaded into registers while the current
// one is multiplied; shared memory is double buffered, one barrier per
// slice. BN = 64 halves the accumulators, so two blocks fit on an SM.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace rgpu {

constexpr int kDgBM = 128, kDgBN = 128, kDgBK = 8;

struct DgPlainRows {
  int64_t lda;
  __device__ __forceinline__ int64_t operator()(int64_t r) const { return r * lda; }
};

struct DgStoreC {
  double * C;
  int64_t ldc;
  __device__ __forceinline__ void operator()(int64_t r, int c, double v) const { C[r * ldc + c] = v; }
};

template <bool B_NT, int BN, class ARows, class Epi>
__global__ void __launch_bounds__(256, BN == 64 ? 2 : 1)
dgemm_kernel(int64_t M, int N, int K, const double * __restrict__ A, ARows arows,
             const double * __restrict__ B, int64_t ldb, Epi epi) {
  constexpr int JG = BN / 32;   // column groups of a thread; also B values per thread per slice
  __shared__ __align__(16) double As[2][kDgBK][kDgBM];
  __shared__ __align__(16) double Bs[2][kDgBK][BN];
  __shared__ int64_t a_off[kDgBM];
  const int t = threadIdx.x;
  const int tx = t & 15, ty = t >> 4;
  // column tiles vary fastest: the blocks that share an A row tile run
  // together, so A comes from DRAM once and the others read it from L2
  const int64_t r0 = int64_t(blockIdx.y) * kDgBM;
  const int c0 = int(blockIdx.x) * BN;
  if (t < kDgBM) a_off[t] = (r0 + t < M) ? arows(r0 + t) : int64_t(-1);
  __syncthreads();
  // global -> register loaders: A tiles 2 threads per row, 4 k each; B_NT
  // tiles (BN rows) 2 threads per row with 4 k (BN = 128) or 4 threads per
  // row with 2 k (BN = 64)
  const int lr = t >> 1, lk = (t & 1) * 4;
  const int64_t my_a = a_off[lr];
  constexpr int BK_T = JG;      // k values of a B_NT row per thread: 8 * BN / 256
  const int br = (BN == 128) ? (t >> 1) : (t >> 2);
  const int bk = (BN == 128) ? (t & 1) * 4 : (t & 3) * 2;
  const int64_t my_b = (c0 + br < N) ? int64_t(c0 + br) * ldb : int64_t(-1);
  // B (K x N) tiles: 8 k-rows of BN columns, 32 threads per row, columns 32 apart
  const int nk = t >> 5, nc = t & 31;
  double pa[4], pb[JG];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = k0 + lk + q;
      pa[q] = (my_a >= 0 && k < K) ? A[my_a + k] : 0.;
    }
    if (B_NT) {
#pragma unroll
      for (int q = 0; q < BK_T; ++q) {
        const int k = k0 + bk + q;
        pb[q] = (my_b >= 0 && k < K) ? B[my_b + k] : 0.;
      }
    } else {
      const int k = k0 + nk;
#pragma unroll
      for (int q = 0; q < JG; ++q) {
        const int c = c0 + nc + 32 * q;
        pb[q] = (k < K && c < N) ? B[int64_t(k) * ldb + c] : 0.;
      }
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) As[buf][lk + q][lr] = pa[q];
    if (B_NT) {
#pragma unroll
      for (int q = 0; q < BK_T; ++q) Bs[buf][bk + q][br] = pb[q];
    } else {
#pragma unroll
      for (int q = 0; q < JG; ++q) Bs[buf][nk][nc + 32 * q] = pb[q];
    }
  };
  double acc[8][2 * JG];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 2 * JG; ++j) acc[i][j] = 0.;
  load(0);
  store(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < K; k0 += kDgBK) {
    const bool more = k0 + kDgBK < K;
    if (more) load(k0 + kDgBK);
#pragma unroll
    for (int kk = 0; kk < kDgBK; ++kk) {
      double a[8], b[2 * JG];
      const double2 * ar = reinterpret_cast<const double2 *>(&As[buf][kk][0]);
      const double2 * bs = reinterpret_cast<const double2 *>(&Bs[buf][kk][0]);
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const double2 va = ar[16 * g + ty];
        a[2 * g] = va.x, a[2 * g + 1] = va.y;
      }
#pragma unroll
      for (int g = 0; g < JG; ++g) {
        const double2 vb = bs[16 * g + tx];
        b[2 * g] = vb.x, b[2 * g + 1] = vb.y;
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 2 * JG; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (more) {
      store(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t r = r0 + 32 * (i >> 1) + 2 * ty + (i & 1);
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 2 * JG; ++j) {
      const int c = c0 + 32 * (j >> 1) + 2 * tx + (j & 1);
      if (c < N) epi(r, c, acc[i][j]);
    }
  }
}

template <bool B_NT, class ARows, class Epi, int BN = kDgBN>
void launch_dgemm(int64_t M, int N, int K, const double * A, ARows arows, const double * B, int64_t ldb,
                  Epi epi, cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  const int64_t row_tiles = (M + kDgBM - 1) / kDgBM;
  const int col_tiles = div_up(N, BN);
  if (row_tiles > 65535 || col_tiles > 0x7fffffff)
    throw Error(RGPU_ERR_CAPACITY, "FP64 GEMM: too many rows for one launch");
  const dim3 grid{static_cast<unsigned>(col_tiles), static_cast<unsigned>(row_tiles), 1u};
  dgemm_kernel<B_NT, BN><<<grid, 256, 0, st>>>(M, N, K, A, arows, B, ldb, epi);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

}  // namespace rgpu
