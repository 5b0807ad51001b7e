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

constexpr int kThreads = 128;

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

constexpr int kMaxN = 16;  // largest max_radial of the register-staged path

// One thread per pair (pairs of many centres share a warp, so no lane idles
// when centres have few neighbours). Per l, the n radial values RI and
// p1 = dRI f_c + RI df_c are staged in registers; the spherical-harmonics
// recurrence then streams (Y, grad Y) for that l.
template <int L>
__global__ void __launch_bounds__(kThreads)
pair_adjoint_kernel(ExpansionArgs a, const int32_t * __restrict__ pair_center, int64_t n_pairs,
                    const float * __restrict__ dC, double * __restrict__ F) {
  constexpr int K = (L + 1) * (L + 1);
  constexpr int L1 = L + 1;
  const int W = a.fd.W, n = a.fd.n, S = a.fd.S, nK = a.fd.nK;
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n_pairs;
       p += int64_t(gridDim.x) * blockDim.x) {
    const int32_t ci = pair_center[p];
    if (p == a.pair_off[ci]) continue;  // self pair: carried by the other pairs' F_i terms
    const int32_t self_atom = a.center_atom[ci];
    const double r = a.pair_dist[p];
    const int32_t j = a.pair_j[p];
    const int s = a.species_lut[a.types[j]];
    const float fc = fc_cos_f(r, a.rc, a.sw), dfc = dfc_cos_f(r, a.rc, a.sw);
    const SplinePos q = spline_pos(a.sp, r);
    const float aa = float(q.a), bb = float(q.b);
    const float ca = aa * aa - 1.f, cb = bb * bb - 1.f;
    const float ea = 3.f * aa * aa - 1.f, eb = 3.f * bb * bb - 1.f;
    const float ih = float(a.sp.inv_h);
    const float * y0 = a.sp.yf + size_t(q.k) * W;
    const float * d0 = a.sp.y2hf + size_t(q.k) * W;
    const float * E = dC + (size_t(ci) * S + s) * nK;
    float rl[kMaxN], pl[kMaxN];
    float sY = 0.f, sd0 = 0.f, sd1 = 0.f, sd2 = 0.f;
    const float dx = float(a.pair_dir[3 * p]), dy = float(a.pair_dir[3 * p + 1]),
                dz = float(a.pair_dir[3 * p + 2]);
    spherical_harmonics<L, true, float>(
        dx, dy, dz,
        [&](int lm, float y, float gx, float gy, float gz) {
          float A = 0.f, B = 0.f;
#pragma unroll
          for (int nn = 0; nn < kMaxN; ++nn) {
            if (nn < n) {
              const float ev = __ldg(E + nn * K + lm);
              A += ev * pl[nn];
              B += ev * rl[nn];
            }
          }
          sY += A * y;
          sd0 += B * gx;
          sd1 += B * gy;
          sd2 += B * gz;
        },
        [&](int l) {
#pragma unroll
          for (int nn = 0; nn < kMaxN; ++nn) {
            if (nn < n) {
              const int c = nn * L1 + l;
              const float yy0 = __ldg(y0 + c), yy1 = __ldg(y0 + W + c);
              const float dd0 = __ldg(d0 + c), dd1 = __ldg(d0 + W + c);
              const float ri = aa * (yy0 + ca * dd0) + bb * (yy1 + cb * dd1);
              const float dri = (yy1 - yy0 - ea * dd0 + eb * dd1) * ih;
              rl[nn] = ri;
              pl[nn] = dri * fc + ri * dfc;
            }
          }
        });
    const float fr = fc / float(r);
    const float g0 = dx * sY + fr * sd0, g1 = dy * sY + fr * sd1, g2 = dz * sY + fr * sd2;
    atomicAdd(&F[3 * size_t(j) + 0], -double(g0));
    atomicAdd(&F[3 * size_t(j) + 1], -double(g1));
    atomicAdd(&F[3 * size_t(j) + 2], -double(g2));
    if (j != self_atom) {
      atomicAdd(&F[3 * size_t(self_atom) + 0], double(g0));
      atomicAdd(&F[3 * size_t(self_atom) + 1], double(g1));
      atomicAdd(&F[3 * size_t(self_atom) + 2], double(g2));
    }
  }
}

}  // namespace

void launch_pair_adjoint_fp32(const ExpansionArgs & a, const int32_t * pair_center, int64_t n_pairs,
                              const float * dC, double * forces, cudaStream_t st) {
  if (a.n_centers == 0 || n_pairs == 0) return;
  sph_constants_tu();
  if (a.fd.n > kMaxN) throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_radial above 16 is not supported on the fast path");
  const int grid = int(std::min<int64_t>((n_pairs + kThreads - 1) / kThreads, int64_t(148) * 64));
#define RGPU_ADJ_CASE(LL)                                                                            \
  case LL:                                                                                           \
    pair_adjoint_kernel<LL><<<grid, kThreads, 0, st>>>(a, pair_center, n_pairs, dC, forces);         \
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
