// Sparse GAP kernel matrices for training, in FP64 (the reference's
// arithmetic):
//   K_NM energy rows    models/sparse_kernels.hh:104-131 (target Structure),
//                       :165-191 (target Atom);
//   K_NM gradient rows  models/sparse_kernels.hh:258-499 (with the negative
//                       stress rows of :405-425, :470-482);
//   K_MM                models/sparse_kernels.hh:141-156 with
//                       models/sparse_points.hh:144-170.
//
// All products run through the FP64 tile GEMM of dgemm.cuh. The gradient
// block is one gathered GEMM per central species and chunk of pairs: its A
// rows are the materialised dX_i/dr_j[c] (3 rows per pair, pairs listed by
// the species of their centre), its B rows the sparse points of that
// species; the epilogue scales each entry by zeta (X_i . T_m)^(zeta-1) and
// adds it into row 3j + c of the output. The stress rows come from a second,
// smaller GEMM over 6 virial rows per centre (sum over its pairs of r_ji
// times dX_i/dr_j), whose epilogue adds into the centre's structure.
#include <cuda_runtime.h>

#include "common.cuh"
#include "dgemm.cuh"

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

// A rows of the gradient block: row 3k + c is dX_i/dr_j[c] of pair list[2k].
struct PairRows {
  const int32_t * list;
  int D;
  __device__ __forceinline__ int64_t operator()(int64_t r) const {
    const int64_t k = r / 3;
    return (int64_t(list[2 * k]) * 3 + (r - 3 * k)) * D;
  }
};

// Entry (3k + c, m): scaled by zeta k_im^(zeta-1) and added into row 3j + c.
struct PairScatter {
  const int32_t * list;
  int64_t p_base, row0;
  const int32_t * row_of_center;
  const double * W;
  int M;
  const int32_t * pair_j;
  const int32_t * ucol;
  double * out;
  int64_t ldo;
  __device__ __forceinline__ void operator()(int64_t r, int m, double v) const {
    const int64_t k = r / 3;
    const int c = int(r - 3 * k);
    const int64_t ci = list[2 * k + 1];
    const double w = W[(int64_t(row_of_center[ci]) - row0) * M + m];
    const int64_t j = pair_j[p_base + list[2 * k]];
    atomicAdd(&out[(3 * j + c) * ldo + ucol[m]], v * w);
  }
};

// Entry (6k + e, m) of the stress GEMM: scaled like the pair entries and
// added into Voigt row e of the centre's structure.
struct StressScatter {
  const int32_t * centres;
  int64_t row0, stress_row0;
  const int32_t * row_of_center;
  const double * W;
  int M;
  const int32_t * center_struct;
  const int32_t * ucol;
  double * out;
  int64_t ldo;
  __device__ __forceinline__ void operator()(int64_t r, int m, double v) const {
    const int64_t k = r / 6;
    const int e = int(r - 6 * k);
    const int64_t ci = centres[k];
    const double w = W[(int64_t(row_of_center[ci]) - row0) * M + m];
    atomicAdd(&out[(stress_row0 + 6 * int64_t(center_struct[ci]) + e) * ldo + ucol[m]], v * w);
  }
};

// Virial rows of a centre i: V[e][d] = sum over its pairs of r_ji[a_e] *
// dX_i/dr_j[b_e][d], Voigt e = xx, yy, zz, yz, xz, xy with (a, b) = (x, x),
// (y, y), (z, z), (y, z), (z, x), (x, y) (models/sparse_kernels.hh:405-425).
// Contracting V with T_m gives the stress entries of the centre, since the
// scale zeta k_im^(zeta-1) is the same for all its pairs.
__global__ void __launch_bounds__(256)
virial_rows_kernel(const int32_t * __restrict__ centres, int64_t n, const int64_t * __restrict__ pair_off,
                   int64_t p_base, const double * __restrict__ pair_dist, const double * __restrict__ pair_dir,
                   const double * __restrict__ dX, int D, double * __restrict__ V) {
  constexpr int kMaxP = 64;
  __shared__ double rv[kMaxP][3];
  const int64_t k = blockIdx.x;
  if (k >= n) return;
  const int64_t ci = centres[k];
  const int64_t p0 = pair_off[ci], p1 = pair_off[ci + 1];
  double * out = V + k * 6 * int64_t(D);
  for (int d = threadIdx.x; d < D; d += blockDim.x)
#pragma unroll
    for (int e = 0; e < 6; ++e) out[int64_t(e) * D + d] = 0.;
  for (int64_t q0 = p0; q0 < p1; q0 += kMaxP) {
    const int np = p1 - q0 < kMaxP ? int(p1 - q0) : kMaxP;
    __syncthreads();
    if (threadIdx.x < np) {
      const int64_t p = q0 + threadIdx.x;
      const double r = pair_dist[p];
      rv[threadIdx.x][0] = -r * pair_dir[3 * p];
      rv[threadIdx.x][1] = -r * pair_dir[3 * p + 1];
      rv[threadIdx.x][2] = -r * pair_dir[3 * p + 2];
    }
    __syncthreads();
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
      double v[6] = {0., 0., 0., 0., 0., 0.};
      for (int q = 0; q < np; ++q) {
        const double * g = dX + (q0 + q - p_base) * 3 * int64_t(D) + d;
        const double gx = g[0], gy = g[D], gz = g[2 * int64_t(D)];
        v[0] += rv[q][0] * gx;
        v[1] += rv[q][1] * gy;
        v[2] += rv[q][2] * gz;
        v[3] += rv[q][1] * gz;
        v[4] += rv[q][2] * gx;
        v[5] += rv[q][0] * gy;
      }
#pragma unroll
      for (int e = 0; e < 6; ++e) out[int64_t(e) * D + d] += v[e];
    }
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
  PairScatter epi{a.list, a.p_base, a.row0, a.row_of_center, a.W, a.M, a.pair_j, a.ucol, a.out, a.ldo};
  // 128 x 64 tiles: two blocks per SM (3 % faster than 128 x 128 here)
  launch_dgemm<true, PairRows, PairScatter, 64>(3 * a.n_list, a.M, a.D, a.dX, PairRows{a.list, a.D}, a.T, a.ldt,
                                                epi, st);
}

void launch_knm_stress(const KnmStressArgs & a, cudaStream_t st) {
  if (a.n_centres <= 0 || a.M <= 0) return;
  virial_rows_kernel<<<unsigned(a.n_centres), 256, 0, st>>>(a.centres, a.n_centres, a.pair_off, a.p_base,
                                                          a.pair_dist, a.pair_dir, a.dX, a.D, a.V);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
  StressScatter epi{a.centres, a.row0, a.stress_row0, a.row_of_center, a.W, a.M, a.center_struct, a.ucol,
                    a.out, a.ldo};
  launch_dgemm<true>(6 * a.n_centres, a.M, a.D, a.V, DgPlainRows{a.D}, a.T, a.ldt, epi, st);
}

}  // namespace rgpu
