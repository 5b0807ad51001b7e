// Dense contractions of the GAP model.
//
// Forward, per central species s:  k = X_s T_s^T,  e_i = sum_m alpha_m k^zeta,
// W = alpha zeta k^(zeta-1)   (models/sparse_kernels.hh:104-131,
// models/sparse_kernel_predict.hh:130-145, models/kernels.hh:48-61).
// Backward: dE/dX_s = W T_s (the "sparse_point_scaled" contraction of
// models/sparse_kernel_predict.hh:141-143, done for all centres at once).
//
// Two implementations:
//  * FP64 SIMT tiles for the plain path (the reference's arithmetic,
//    dgemm.cuh);
//  * TF32 tensor-core tiles (mma.sync m16n8k8) with FP32 accumulation for
//    the fast path, optionally as a 3-term split (hi*hi + hi*lo + lo*hi) that
//    carries ~21 mantissa bits. The forward epilogue fuses k^zeta, the
//    per-row energy partials and W, so k never touches HBM.
#include <cuda_runtime.h>

#include "common.cuh"
#include "dgemm.cuh"

namespace rgpu {
namespace {

__device__ __forceinline__ float pow_zeta_f(float v, int z) {
  float r = 1.f;
  for (int i = 0; i < z; ++i) r *= v;
  return r;
}

__global__ void gap_pointwise_fp64_kernel(int64_t rows, int M, const double * __restrict__ Km,
                                          int64_t ldk, const double * __restrict__ alpha, int zeta,
                                          double * __restrict__ W, int64_t ldw,
                                          double * __restrict__ e_row) {
  int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (r >= rows) return;
  double e = 0.;
  for (int m = lane; m < M; m += 32) {
    double k = Km[r * ldk + m];
    e += alpha[m] * pow_zeta_d(k, zeta);
    W[r * ldw + m] = alpha[m] * (zeta * pow_zeta_d(k, zeta - 1));
  }
  e = warp_sum(e);
  if (lane == 0) e_row[r] = e;
}

// ------------------------------------------------------ TF32 tensor-core GEMM
constexpr int kBM = 128, kBN = 128, kBKt = 32, kStages = 3, kLdS = kBKt + 4;
constexpr size_t kTf32Smem = size_t(kStages) * 2 * kBM * kLdS * sizeof(float);

__device__ __forceinline__ void cp_async16(void * smem, const void * gmem, int src_bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void mma_tf32(float * c, const uint32_t * a, const uint32_t * b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t tf32_bits(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

template <bool SPLIT>
__global__ void __launch_bounds__(256)
gemm_tf32_kernel(Tf32GemmArgs g) {
  extern __shared__ __align__(16) float sm[];
  float * As = sm;                                  // [stages][BM][LdS]
  float * Bs = sm + size_t(kStages) * kBM * kLdS;   // [stages][BN][LdS]
  __shared__ float row_e[kBM];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int wm = (wid >> 2) * 64, wn = (wid & 3) * 32;
  const int64_t n0 = int64_t(blockIdx.x) * kBN, m0 = int64_t(blockIdx.y) * kBM;
  if (g.epilogue == 1 && tid < kBM) row_e[tid] = 0.f;

  auto load_stage = [&](int stage, int64_t k0) {
    float * as = As + size_t(stage) * kBM * kLdS;
    float * bs = Bs + size_t(stage) * kBN * kLdS;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int idx = tid + q * 256;  // 1024 chunks of 16 B per operand
      int r = idx >> 3, cchunk = (idx & 7) * 4;
      int64_t ga = m0 + r;
      const float * src = g.A + (ga < g.M ? ga : 0) * g.lda + k0 + cchunk;
      cp_async16(as + r * kLdS + cchunk, src, ga < g.M ? 16 : 0);
      int64_t gb = n0 + r;
      const float * srcb = g.B + (gb < g.N ? gb : 0) * g.ldb + k0 + cchunk;
      cp_async16(bs + r * kLdS + cchunk, srcb, gb < g.N ? 16 : 0);
    }
  };

  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.f;

  const int nk = int(g.K / kBKt);
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) load_stage(s, int64_t(s) * kBKt);
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<kStages - 2>();
    __syncthreads();
    {
      int nxt = kt + kStages - 1;
      if (nxt < nk) load_stage(nxt % kStages, int64_t(nxt) * kBKt);
      cp_commit();
    }
    const float * as = As + size_t(kt % kStages) * kBM * kLdS;
    const float * bs = Bs + size_t(kt % kStages) * kBN * kLdS;
#pragma unroll
    for (int kk = 0; kk < kBKt; kk += 8) {
      uint32_t ah[4][4], bh[4][2];
      uint32_t al[4][4], bl[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float * p = as + (wm + i * 16 + gid) * kLdS + kk + tig;
        float f[4] = {p[0], p[8 * kLdS], p[4], p[8 * kLdS + 4]};
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          ah[i][v] = tf32_bits(f[v]);
          if (SPLIT) al[i][v] = tf32_bits(f[v] - __uint_as_float(ah[i][v]));
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float * p = bs + (wn + j * 8 + gid) * kLdS + kk + tig;
        float f[2] = {p[0], p[4]};
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          bh[j][v] = tf32_bits(f[v]);
          if (SPLIT) bl[j][v] = tf32_bits(f[v] - __uint_as_float(bh[j][v]));
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (SPLIT) {
            mma_tf32(acc[i][j], al[i], bh[j]);
            mma_tf32(acc[i][j], ah[i], bl[j]);
          }
          mma_tf32(acc[i][j], ah[i], bh[j]);
        }
    }
  }
  cp_wait<0>();

  if (g.epilogue == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int64_t r = m0 + wm + i * 16 + gid + h * 8;
          int64_t c = n0 + wn + j * 8 + tig * 2;
          if (r < g.M && c < g.N) {
            float2 v = make_float2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
            *reinterpret_cast<float2 *>(g.C + r * g.ldc + c) = v;
          }
        }
    return;
  }
  // GAP forward epilogue
  float re[4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i) re[i][0] = re[i][1] = 0.f;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int64_t r = m0 + wm + i * 16 + gid + h * 8;
        int64_t c = n0 + wn + j * 8 + tig * 2;
        float w2[2];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          float k = acc[i][j][2 * h + v];
          float al = (c + v < g.N) ? g.alpha[c + v] : 0.f;
          re[i][h] += al * pow_zeta_f(k, g.zeta);
          w2[v] = al * (float(g.zeta) * pow_zeta_f(k, g.zeta - 1));
        }
        if (r < g.M && c < g.ldc) *reinterpret_cast<float2 *>(g.C + r * g.ldc + c) = make_float2(w2[0], w2[1]);
      }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v = re[i][h];
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      re[i][h] = v;
    }
  __syncthreads();
  if (tig == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int h = 0; h < 2; ++h) atomicAdd(&row_e[wm + i * 16 + gid + h * 8], re[i][h]);
  }
  __syncthreads();
  if (tid < kBM) {
    int64_t r = m0 + tid;
    if (r < g.M) g.e_part[int64_t(blockIdx.x) * g.M + r] = row_e[tid];
  }
}

__global__ void energy_reduce_kernel(int64_t rows, int n_parts, const float * __restrict__ e_part,
                                     int64_t ld, const double * __restrict__ e_row, int64_t row0,
                                     const int32_t * __restrict__ center_of_row,
                                     const int32_t * __restrict__ center_struct,
                                     double * __restrict__ E) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double e = 0.;
  int key = -1;
  if (r < rows) {
    if (e_row) {
      e = e_row[r];
    } else {
      for (int t = 0; t < n_parts; ++t) e += double(e_part[int64_t(t) * ld + r]);
    }
    key = center_struct[center_of_row[row0 + r]];
  }
  // the warp's rows of one structure are summed first, so a structure with
  // many centres (one large box) takes one atomic per warp, not per row
  const int lane = threadIdx.x & 31;
  double sum = 0.;
  int leader = 32;
#pragma unroll 4
  for (int src = 0; src < 32; ++src) {
    const double v = __shfl_sync(0xffffffffu, e, src);
    const int k = __shfl_sync(0xffffffffu, key, src);
    if (k == key) {
      sum += v;
      leader = min(leader, src);
    }
  }
  if (key >= 0 && leader == lane) atomicAdd(&E[key], sum);
}

// Plain path: gradients[j] += dX_i(pair) . t_i, one warp per pair.
__global__ void force_contract_kernel(int64_t p_first, int64_t np, int D, int64_t p_base,
                                      const int64_t * __restrict__ pair_center,
                                      const int32_t * __restrict__ pair_j,
                                      const int32_t * __restrict__ row_of_center,
                                      const double * __restrict__ dX, const double * __restrict__ t,
                                      int64_t ldt, double * __restrict__ grad,
                                      const double * __restrict__ pair_dist,
                                      const double * __restrict__ pair_dir,
                                      const int32_t * __restrict__ center_struct,
                                      double * __restrict__ stress) {
  int64_t q = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (q >= np) return;
  int64_t p = p_first + q;
  int64_t ci = pair_center[q];
  const double * tr = t + size_t(row_of_center[ci]) * ldt;
  const double * g = dX + size_t(p - p_base) * 3 * D;
  double s[3] = {0., 0., 0.};
  for (int d = lane; d < D; d += 32) {
    double tv = tr[d];
    s[0] += g[d] * tv;
    s[1] += g[D + d] * tv;
    s[2] += g[2 * D + d] * tv;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) s[c] = warp_sum(s[c]);
  if (lane == 0) {
    int64_t j = pair_j[p];
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(&grad[3 * j + c], s[c]);
    // r_ji (x) dE_i/dr_j, Voigt xx yy zz yz xz xy
    // (models/sparse_kernel_predict.hh:355-366); the self pair has r_ji = 0
    if (stress && pair_dist[p] > 0.) {
      const double r = pair_dist[p];
      const double rx = -r * pair_dir[3 * p], ry = -r * pair_dir[3 * p + 1], rz = -r * pair_dir[3 * p + 2];
      double * st = stress + 6 * size_t(center_struct[ci]);
      atomicAdd(st + 0, rx * s[0]);
      atomicAdd(st + 4, rz * s[0]);
      atomicAdd(st + 1, ry * s[1]);
      atomicAdd(st + 5, rx * s[1]);
      atomicAdd(st + 2, rz * s[2]);
      atomicAdd(st + 3, ry * s[2]);
    }
  }
}

__global__ void pair_center2_kernel(int64_t c0, int64_t c1, const int64_t * __restrict__ pair_off,
                                    int64_t p_first, int64_t * __restrict__ pc) {
  int64_t ci = c0 + int64_t(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (ci >= c1) return;
  for (int64_t p = pair_off[ci] + (threadIdx.x & 31); p < pair_off[ci + 1]; p += 32)
    pc[p - p_first] = ci;
}

}  // namespace

void gemm_nt_fp64(int64_t M, int64_t N, int64_t K, const double * A, int64_t lda, const double * B,
                  int64_t ldb, double * C, int64_t ldc, cudaStream_t st) {
  launch_dgemm<true>(M, int(N), int(K), A, DgPlainRows{lda}, B, ldb, DgStoreC{C, ldc}, st);
}
void gemm_nn_fp64(int64_t M, int64_t N, int64_t K, const double * A, int64_t lda, const double * B,
                  int64_t ldb, double * C, int64_t ldc, cudaStream_t st) {
  launch_dgemm<false>(M, int(N), int(K), A, DgPlainRows{lda}, B, ldb, DgStoreC{C, ldc}, st);
}

void launch_gap_pointwise_fp64(int64_t rows, int M, const double * Kmat, int64_t ldk,
                               const double * alpha, int zeta, double * W, int64_t ldw,
                               double * e_row, cudaStream_t st) {
  if (rows <= 0) return;
  gap_pointwise_fp64_kernel<<<div_up(rows * 32, 256), 256, 0, st>>>(rows, M, Kmat, ldk, alpha, zeta,
                                                                   W, ldw, e_row);
  RGPU_LAUNCHED();
}

bool g_tf32_split = true;

void gemm_tf32(const Tf32GemmArgs & g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0) return;
  if (g.K % kBKt != 0) throw Error(RGPU_ERR_INVALID_ARGUMENT, "TF32 GEMM: K must be a multiple of 32");
  dim3 grid(div_up(g.N, kBN), div_up(g.M, kBM));
  if (g_tf32_split) {
    RGPU_CUDA(cudaFuncSetAttribute(gemm_tf32_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(kTf32Smem)));
    gemm_tf32_kernel<true><<<grid, 256, kTf32Smem, st>>>(g);
  } else {
    RGPU_CUDA(cudaFuncSetAttribute(gemm_tf32_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(kTf32Smem)));
    gemm_tf32_kernel<false><<<grid, 256, kTf32Smem, st>>>(g);
  }
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

void launch_energy_reduce(int64_t rows, int n_parts, const float * e_part, int64_t ld,
                          const double * e_row_fp64, int64_t row0, const int32_t * center_of_row,
                          const int32_t * center_struct, double * energies, cudaStream_t st) {
  if (rows <= 0) return;
  energy_reduce_kernel<<<div_up(rows, 256), 256, 0, st>>>(rows, n_parts, e_part, ld, e_row_fp64, row0,
                                                         center_of_row, center_struct, energies);
  RGPU_LAUNCHED();
}

void launch_force_contract_fp64(const FeatureDims & fd, int64_t c0, int64_t c1, int64_t p_base,
                                const int64_t * pair_off, const int32_t * pair_j,
                                const int32_t * row_of_center, const double * dX, const double * t,
                                int64_t ldt, double * grad, cudaStream_t st, const double * pair_dist,
                                const double * pair_dir, const int32_t * center_struct, double * stress) {
  if (c1 <= c0) return;
  int64_t p_first = 0, p_last = 0;
  RGPU_CUDA(cudaMemcpyAsync(&p_first, pair_off + c0, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RGPU_CUDA(cudaMemcpyAsync(&p_last, pair_off + c1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RGPU_CUDA(cudaStreamSynchronize(st));
  const int64_t np = p_last - p_first;
  if (np <= 0) return;
  // per host thread and per device: another device's buffer is not memory this launch may use
  static thread_local PerDevice<DevBuf> pc_tab;
  DevBuf & pc = pc_tab.at(current_device());
  pc.ensure(sizeof(int64_t) * np);
  pair_center2_kernel<<<div_up(c1 - c0, 8), 256, 0, st>>>(c0, c1, pair_off, p_first, pc.as<int64_t>());
  RGPU_LAUNCHED();
  force_contract_kernel<<<div_up(np * 32, 256), 256, 0, st>>>(p_first, np, fd.D, p_base,
                                                             pc.as<int64_t>(), pair_j, row_of_center,
                                                             dX, t, ldt, grad, pair_dist, pair_dir,
                                                             center_struct, stress);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

}  // namespace rgpu
