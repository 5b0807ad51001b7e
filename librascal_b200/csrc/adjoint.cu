// Adjoint force kernel of the fast path.
//
// Given dE/dc^i (from the power-spectrum backward), the force contribution of
// pair (i, j) is g_ij = sum_{n,lm} dE/dc^i_{type_j, n lm} * d c^i_{n lm}/d r_j,
// where d c^i / d r_j = (dRI f_c + RI df_c) Y r^ + RI f_c / r grad Y is
// recomputed here from the spline and the spherical-harmonics recurrence
// instead of being stored (the reference materialises it per pair,
// calculator_spherical_expansion.hh:2306-2366, and contracts it in
// models/sparse_kernel_predict.hh:147-172). The contraction is reordered as
//   g = r^ * sum_lm A_lm Y_lm + f_c / r * sum_lm B_lm grad Y_lm,
//   A_lm = sum_n E_{n lm} (dRI f_c + RI df_c)_{n l},  B_lm = sum_n E_{n lm} RI_{n l}.
// Forces follow the reference's accumulation (sparse_kernel_predict.hh:
// 257-263): F_j -= g_ij for every pair (folded onto the real atom) and
// F_i += g_ij unless j is a periodic image of i (the rule of
// calculator_spherical_expansion.hh:2354-2358).
#include <cuda_runtime.h>

#include "common.cuh"

namespace rgpu {
namespace {

constexpr int kWarps = 4;

__device__ __forceinline__ float fc_cos_f(double r, double rc, double sw) {
  if (r <= (rc - sw)) return 1.f;
  if (r > rc) return 0.f;
  double rs = 3.14159265358979323846264338327950288 * (r - rc + sw) / sw;
  return float(0.5 * (1. + cos(rs)));
}
__device__ __forceinline__ float dfc_cos_f(double r, double rc, double sw) {
  if (r <= (rc - sw)) return 0.f;
  if (r > rc) return 0.f;
  double rs = 3.14159265358979323846264338327950288 * (r - rc + sw) / sw;
  return float(-0.5 * 3.14159265358979323846264338327950288 / sw * sin(rs));
}

template <int L>
__global__ void __launch_bounds__(kWarps * 32)
pair_adjoint_kernel(ExpansionArgs a, const float * __restrict__ dC, double * __restrict__ F) {
  constexpr int K = (L + 1) * (L + 1);
  constexpr int L1 = L + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int W = a.fd.W, n = a.fd.n, S = a.fd.S, nK = a.fd.nK;
  float * Es = reinterpret_cast<float *>(smem_raw) + size_t(wid) * (S * nK + 2 * W * 32);
  float * RI = Es + S * nK;
  float * P1 = RI + W * 32;
  for (int64_t ci = int64_t(blockIdx.x) * kWarps + wid; ci < a.n_centers;
       ci += int64_t(gridDim.x) * kWarps) {
    const float * Ei = dC + size_t(ci) * S * nK;
    for (int e = lane; e < S * nK; e += 32) Es[e] = Ei[e];
    __syncwarp();
    const int64_t p_lo = a.pair_off[ci] + 1, p_hi = a.pair_off[ci + 1];
    const int32_t self_atom = a.center_atom[ci];
    float fi[3] = {0.f, 0.f, 0.f};
    for (int64_t p = p_lo + lane; p < p_hi; p += 32) {
      const double r = a.pair_dist[p];
      const int32_t j = a.pair_j[p];
      const int s = a.species_lut[a.types[j]];
      const float fc = fc_cos_f(r, a.rc, a.sw), dfc = dfc_cos_f(r, a.rc, a.sw);
      // RI and dRI of this pair (dRI is turned into p1 = dRI fc + RI dfc)
      {
        SplinePos q = spline_pos(a.sp, r);
        const float aa = float(q.a), bb = float(q.b);
        const float ca = aa * aa - 1.f, cb = bb * bb - 1.f;
        const float ea = 3.f * aa * aa - 1.f, eb = 3.f * bb * bb - 1.f;
        const float ih = float(a.sp.inv_h);
        const float * y0 = a.sp.yf + size_t(q.k) * W;
        const float * d0 = a.sp.y2hf + size_t(q.k) * W;
        for (int c = 0; c < W; ++c) {
          const float yy0 = __ldg(y0 + c), yy1 = __ldg(y0 + W + c);
          const float dd0 = __ldg(d0 + c), dd1 = __ldg(d0 + W + c);
          const float ri = aa * (yy0 + ca * dd0) + bb * (yy1 + cb * dd1);
          const float dri = (yy1 - yy0 - ea * dd0 + eb * dd1) * ih;
          RI[c * 32 + lane] = ri;
          P1[c * 32 + lane] = dri * fc + ri * dfc;
        }
      }
      const float * E = Es + s * nK;
      float sY = 0.f, sd[3] = {0.f, 0.f, 0.f};
      const float dx = float(a.pair_dir[3 * p]), dy = float(a.pair_dir[3 * p + 1]),
                  dz = float(a.pair_dir[3 * p + 2]);
      spherical_harmonics<L, true, float>(dx, dy, dz, [&](int lm, float y, float gx, float gy,
                                                          float gz) {
        int l = 0;
#pragma unroll
        for (int ll = 1; ll <= L; ++ll) l += (lm >= ll * ll);
        float A = 0.f, B = 0.f;
        for (int nn = 0; nn < n; ++nn) {
          const float ev = E[nn * K + lm];
          A += ev * P1[(nn * L1 + l) * 32 + lane];
          B += ev * RI[(nn * L1 + l) * 32 + lane];
        }
        sY += A * y;
        sd[0] += B * gx;
        sd[1] += B * gy;
        sd[2] += B * gz;
      });
      const float fr = fc / float(r);
      const float g[3] = {dx * sY + fr * sd[0], dy * sY + fr * sd[1], dz * sY + fr * sd[2]};
#pragma unroll
      for (int c = 0; c < 3; ++c) atomicAdd(&F[3 * size_t(j) + c], -double(g[c]));
      if (j != self_atom) {
        fi[0] += g[0];
        fi[1] += g[1];
        fi[2] += g[2];
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) fi[c] = warp_sum(fi[c]);
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) atomicAdd(&F[3 * size_t(self_atom) + c], double(fi[c]));
    }
    __syncwarp();
  }
}

}  // namespace

void launch_pair_adjoint_fp32(const ExpansionArgs & a, const float * dC, double * forces,
                              cudaStream_t st) {
  if (a.n_centers == 0) return;
  sph_constants_tu();
  const size_t smem = size_t(kWarps) * (size_t(a.fd.S) * a.fd.nK + 2 * a.fd.W * 32) * sizeof(float);
  int grid = int(std::min<int64_t>((a.n_centers + kWarps - 1) / kWarps, 148 * 16));
#define RGPU_ADJ_CASE(LL)                                                                   \
  case LL:                                                                                  \
    RGPU_CUDA(cudaFuncSetAttribute(pair_adjoint_kernel<LL>,                                 \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))); \
    pair_adjoint_kernel<LL><<<grid, kWarps * 32, smem, st>>>(a, dC, forces);                \
    break;
  switch (a.fd.L) {
    RGPU_ADJ_CASE(0)
    RGPU_ADJ_CASE(1)
    RGPU_ADJ_CASE(2)
    RGPU_ADJ_CASE(3)
    RGPU_ADJ_CASE(4)
    RGPU_ADJ_CASE(5)
    RGPU_ADJ_CASE(6)
    RGPU_ADJ_CASE(7)
    RGPU_ADJ_CASE(8)
    RGPU_ADJ_CASE(9)
    RGPU_ADJ_CASE(10)
    RGPU_ADJ_CASE(11)
    RGPU_ADJ_CASE(12)
    default:
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_angular above 12 is not supported on the GPU");
  }
#undef RGPU_ADJ_CASE
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

}  // namespace rgpu
