// Sparse GAP kernel matrices for training, in FP64 (the reference's
// arithmetic):
//   K_NM energy rows    models/sparse_kernels.hh:104-131 (target Structure),
//                       :165-191 (target Atom);
//   K_NM gradient rows  models/sparse_kernels.hh:258-499 (with the negative
//                       stress rows of :405-425, :470-482);
//   K_MM                models/sparse_kernels.hh:141-156 with
//                       models/sparse_points.hh:144-170.
//
// The dot products X T^T and T T^T run through the FP64 tile GEMM of
// gemm.cu. The gradient block is one gathered GEMM per central species and
// chunk of pairs: its A rows are the materialised dX_i/dr_j[c] (3 rows per
// pair, pairs listed by the species of their centre), its B rows the sparse
// points of that species. The epilogue scales each entry by
// zeta (X_i . T_m)^(zeta-1), adds it into row 3j + c of the output and, for
// the stress rows, reduces r_ji (x) entry over the tile's rows of one
// structure before one atomic add per (structure, Voigt entry, column).
#include <cuda_runtime.h>

#include "common.cuh"

namespace rgpu {
namespace {

__global__ void knm_rows_kernel(int64_t rows, int M, const double * __restrict__ K, int zeta,
                                const int32_t * __restrict__ center_of_row, int64_t row0,
                                const int32_t * __restrict__ center_struct, int atom_target,
                                const int32_t * __restrict__ ucol, double * __restrict__ out,
                                int64_t ldo) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= rows * M) return;
  const int64_t r = i / M;
  const int m = int(i - r * M);
  const double v = pow_zeta_d(K[i], zeta);
  const int64_t ci = center_of_row[row0 + r];
  if (atom_target)
    out[ci * ldo + ucol[m]] = v;
  else
    atomicAdd(&out[int64_t(center_struct[ci]) * ldo + ucol[m]], v);
}

// W = zeta k^(zeta-1); exactly 1 for zeta = 1, where the reference skips the
// factor (models/sparse_kernels.hh:320-331, :393-396).
__global__ void kernel_weight_kernel(int64_t n, double * __restrict__ K, int zeta) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  K[i] = zeta > 1 ? double(zeta) * pow_zeta_d(K[i], zeta - 1) : 1.;
}

__global__ void kmm_scatter_kernel(int M, const double * __restrict__ K, int zeta,
                                   const int32_t * __restrict__ ucol, double * __restrict__ out,
                                   int64_t ldo) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= int64_t(M) * M) return;
  const int a = int(i / M), b = int(i - int64_t(a) * M);
  out[int64_t(ucol[a]) * ldo + ucol[b]] = pow_zeta_d(K[i], zeta);
}

constexpr int kDT = 64, kDK = 16;

// Gathered GEMM of the gradient block: tile of 64 (pair, component) rows x
// 64 sparse points, 256 threads with a 4 x 4 register tile each.
template <bool STRESS>
__global__ void __launch_bounds__(256)
knm_derivative_kernel(const KnmDerArgs a) {
  // As/Bs during the main loop; the scaled 64 x 64 tile in the stress epilogue
  __shared__ double sm[kDT * (kDT + 1)];
  __shared__ int64_t a_off[kDT];
  __shared__ int32_t r_struct[kDT];
  __shared__ double r_vec[kDT][3];
  double (*As)[kDT + 1] = reinterpret_cast<double (*)[kDT + 1]>(sm);
  double (*Bs)[kDT + 1] = reinterpret_cast<double (*)[kDT + 1]>(sm + kDK * (kDT + 1));
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t n_rows = 3 * a.n_list;
  const int64_t r0 = int64_t(blockIdx.x) * kDT;
  const int c0 = int(blockIdx.y) * kDT;
  if (threadIdx.x < kDT) {
    const int64_t gr = r0 + threadIdx.x;
    int64_t off = -1;
    if (gr < n_rows) {
      const int64_t k = gr / 3;
      const int c = int(gr - 3 * k);
      const int64_t pl = a.list[2 * k];
      off = (pl * 3 + c) * int64_t(a.D);
      if (STRESS) {
        const int64_t p = a.p_base + pl;
        const double r = a.pair_dist[p];
        // r_ji = r_i - r_j = -r * dir
        r_vec[threadIdx.x][0] = -r * a.pair_dir[3 * p];
        r_vec[threadIdx.x][1] = -r * a.pair_dir[3 * p + 1];
        r_vec[threadIdx.x][2] = -r * a.pair_dir[3 * p + 2];
        r_struct[threadIdx.x] = a.center_struct[a.list[2 * k + 1]];
      }
    }
    a_off[threadIdx.x] = off;
  }
  __syncthreads();
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.;
  for (int k0 = 0; k0 < a.D; k0 += kDK) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = threadIdx.x + q * 256;
      const int r = idx / kDK, k = idx % kDK;
      const int64_t off = a_off[r];
      As[k][r] = (off >= 0 && k0 + k < a.D) ? a.dX[off + k0 + k] : 0.;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = threadIdx.x + q * 256;
      const int c = idx / kDK, k = idx % kDK;
      const int gc = c0 + c;
      Bs[k][c] = (gc < a.M && k0 + k < a.D) ? a.T[int64_t(gc) * a.ldt + k0 + k] : 0.;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kDK; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[k][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[k][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += av[i] * bv[j];
    }
    __syncthreads();
  }
  // epilogue: scale by W, add into the atom rows, keep the tile for the stress
  double (*V)[kDT + 1] = reinterpret_cast<double (*)[kDT + 1]>(sm);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rl = ty + 16 * i;
    const int64_t gr = r0 + rl;
    const bool row_ok = gr < n_rows;
    int64_t k = 0, ci = 0, wrow = 0, j = 0;
    int c = 0;
    if (row_ok) {
      k = gr / 3;
      c = int(gr - 3 * k);
      ci = a.list[2 * k + 1];
      wrow = int64_t(a.row_of_center[ci]) - a.row0;
      j = a.pair_j[a.p_base + a.list[2 * k]];
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int cl = tx + 16 * jj;
      const int gc = c0 + cl;
      double v = 0.;
      if (row_ok && gc < a.M) {
        v = acc[i][jj] * a.W[wrow * a.M + gc];
        atomicAdd(&a.out[(3 * j + c) * a.ldo + a.ucol[gc]], v);
      }
      if (STRESS) V[rl][cl] = v;
    }
  }
  if (!STRESS) return;
  __syncthreads();
  // Voigt xx, yy, zz, yz, xz, xy: entry e takes component c_of[e] of the
  // pair term times r_ji[d_of[e]] (models/sparse_kernels.hh:405-425)
  const int64_t rem = n_rows - r0;
  const int rows_here = rem < kDT ? int(rem) : kDT;
  for (int t = threadIdx.x; t < 6 * kDT; t += blockDim.x) {
    const int cl = t % kDT, e = t / kDT;
    const int gc = c0 + cl;
    if (gc >= a.M) continue;
    const int c_of = e < 3 ? e : (e == 3 ? 2 : (e == 4 ? 0 : 1));
    const int d_of = e < 3 ? e : (e == 3 ? 1 : (e == 4 ? 2 : 0));
    double sum = 0.;
    int cur = -1;
    for (int rl = 0; rl < rows_here; ++rl) {
      if (int((r0 + rl) % 3) != c_of) continue;
      const int sidx = r_struct[rl];
      if (sidx != cur) {
        if (cur >= 0) atomicAdd(&a.out[(a.stress_row0 + 6 * int64_t(cur) + e) * a.ldo + a.ucol[gc]], sum);
        cur = sidx;
        sum = 0.;
      }
      sum += r_vec[rl][d_of] * V[rl][cl];
    }
    if (cur >= 0) atomicAdd(&a.out[(a.stress_row0 + 6 * int64_t(cur) + e) * a.ldo + a.ucol[gc]], sum);
  }
}

}  // namespace

void launch_knm_rows(int64_t rows, int M, const double * K, int zeta, const int32_t * center_of_row,
                     int64_t row0, const int32_t * center_struct, bool atom_target, const int32_t * ucol,
                     double * out, int64_t ldo, cudaStream_t st) {
  if (rows <= 0 || M <= 0) return;
  knm_rows_kernel<<<div_up(rows * M, 256), 256, 0, st>>>(rows, M, K, zeta, center_of_row, row0, center_struct,
                                                        int(atom_target), ucol, out, ldo);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

void launch_kernel_weight(int64_t n, double * K, int zeta, cudaStream_t st) {
  if (n <= 0) return;
  kernel_weight_kernel<<<div_up(n, 256), 256, 0, st>>>(n, K, zeta);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

void launch_kmm_scatter(int M, const double * K, int zeta, const int32_t * ucol, double * out, int64_t ldo,
                        cudaStream_t st) {
  if (M <= 0) return;
  kmm_scatter_kernel<<<div_up(int64_t(M) * M, 256), 256, 0, st>>>(M, K, zeta, ucol, out, ldo);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

void launch_knm_derivative(const KnmDerArgs & a, cudaStream_t st) {
  if (a.n_list <= 0 || a.M <= 0) return;
  const int64_t row_tiles = (3 * a.n_list + kDT - 1) / kDT;
  const int col_tiles = div_up(a.M, kDT);
  if (row_tiles > 0x7fffffff || col_tiles > 65535)
    throw Error(RGPU_ERR_CAPACITY, "kernel gradient block: too many rows or sparse points for one launch");
  const dim3 grid{static_cast<unsigned>(row_tiles), static_cast<unsigned>(col_tiles), 1u};
  if (a.pair_dist)
    knm_derivative_kernel<true><<<grid, 256, 0, st>>>(a);
  else
    knm_derivative_kernel<false><<<grid, 256, 0, st>>>(a);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

}  // namespace rgpu
