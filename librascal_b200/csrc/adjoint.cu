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

#include <algorithm>

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
// p1 = dRI f_c + RI df_c are staged in registers (NV >= n of them); the
// spherical-harmonics recurrence then streams (Y, grad Y) for that l.
// dE/dc of the pair's centre is read as dC[i][lm][s*n + n'], n contiguous
// values per lm (float4 loads when n == NV). With STRESS, the pair's
// r_ji (x) g_ij (Voigt xx yy zz yz xz xy, the reference's
// sparse_kernel_predict.hh:355-366) is summed per structure as well.
template <int L, int NV, bool STRESS>
// 5 resident blocks per SM (96 registers, a few bytes of spills at L = 6)
// measured faster than 4 (128 registers) or 6 (more spills)
__global__ void __launch_bounds__(kThreads, 5)
pair_adjoint_kernel(ExpansionArgs a, const int32_t * __restrict__ pair_center, int64_t n_pairs,
                    const float * __restrict__ dC, double * __restrict__ F,
                    const int32_t * __restrict__ center_struct, double * __restrict__ stress) {
  constexpr int K = (L + 1) * (L + 1);
  constexpr int L1 = L + 1;
  const int W = a.fd.W, n = a.fd.n, Sn = a.fd.S * a.fd.n;
  const bool vec = (n == NV);
  const int lane = threadIdx.x & 31;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  // the list's own total bounds the loop (below n_pairs when the list was
  // built to a capacity)
  {
    const int64_t listed = a.pair_off[a.n_centers];
    if (listed < n_pairs) n_pairs = listed;
  }
  // the loop bound is warp-uniform: the F_i sums below shuffle across lanes
  for (int64_t base = int64_t(blockIdx.x) * blockDim.x + threadIdx.x - lane; base < n_pairs; base += stride) {
    const int64_t p = base + lane;
    const int32_t ci = p < n_pairs ? pair_center[p] : -1;
    float g0 = 0.f, g1 = 0.f, g2 = 0.f;
    float t6[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int32_t j = -1, self_atom = -1;
    // the self pair carries no force of its own: the other pairs' F_i terms do
    if (ci >= 0 && p != a.pair_off[ci]) {
      self_atom = a.center_atom[ci];
      const double r = a.pair_dist[p];
      j = a.pair_j[p];
      const int s = a.species_lut[a.types[j]];
      float fc = fc_cos_f(r, a.rc, a.sw), dfc = dfc_cos_f(r, a.rc, a.sw);
      if (a.rs.on) {
        const double u = rs_value(a.rs, r);
        const double cosw = 0.5 * (1. + cos(3.14159265358979323846264338327950288 * (r - a.rc + a.sw) / a.sw));
        const double sr = (r <= a.rc - a.sw) ? 1.0 : (r > a.rc ? 0.0 : cosw);
        dfc = float(rs_grad(a.rs, r) * sr + u * double(dfc));
        fc = float(u * sr);
      }
      const SplinePos q = spline_pos(a.sp, r);
      const float aa = float(q.a), bb = float(q.b);
      const float ca = aa * aa - 1.f, cb = bb * bb - 1.f;
      const float ea = 3.f * aa * aa - 1.f, eb = 3.f * bb * bb - 1.f;
      const float ih = float(a.sp.inv_h);
      // interval k of the spline: (y_k, y2h_k, y_k+1, y2h_k+1) per channel
      const float4 * q4 = a.sp.q4f + size_t(q.k) * W;
      const float * E = dC + size_t(ci) * Sn * K + s * n;
      float rl[NV], pl[NV];
      float sY = 0.f, sd0 = 0.f, sd1 = 0.f, sd2 = 0.f;
      const float dx = float(a.pair_dir[3 * p]), dy = float(a.pair_dir[3 * p + 1]),
                  dz = float(a.pair_dir[3 * p + 2]);
      spherical_harmonics<L, true, float>(
          dx, dy, dz,
          [&](int lm, float y, float gx, float gy, float gz) {
            float A = 0.f, B = 0.f;
            const float * El = E + lm * Sn;
            if (vec) {
              const float4 * E4 = reinterpret_cast<const float4 *>(El);
#pragma unroll
              for (int qq = 0; qq < NV / 4; ++qq) {
                const float4 ev = __ldg(E4 + qq);
                A += ev.x * pl[4 * qq] + ev.y * pl[4 * qq + 1] + ev.z * pl[4 * qq + 2] + ev.w * pl[4 * qq + 3];
                B += ev.x * rl[4 * qq] + ev.y * rl[4 * qq + 1] + ev.z * rl[4 * qq + 2] + ev.w * rl[4 * qq + 3];
              }
            } else {
#pragma unroll
              for (int nn = 0; nn < NV; ++nn) {
                if (nn < n) {
                  const float ev = __ldg(El + nn);
                  A += ev * pl[nn];
                  B += ev * rl[nn];
                }
              }
            }
            sY += A * y;
            sd0 += B * gx;
            sd1 += B * gy;
            sd2 += B * gz;
          },
          [&](int l) {
#pragma unroll
            for (int nn = 0; nn < NV; ++nn) {
              if (nn < n) {
                const float4 t = __ldg(q4 + nn * L1 + l);
                const float ri = aa * (t.x + ca * t.y) + bb * (t.z + cb * t.w);
                const float dri = (t.z - t.x - ea * t.y + eb * t.w) * ih;
                rl[nn] = ri;
                pl[nn] = dri * fc + ri * dfc;
              } else {
                rl[nn] = 0.f;
                pl[nn] = 0.f;
              }
            }
          });
      const float fr = fc / float(r);
      g0 = dx * sY + fr * sd0;
      g1 = dy * sY + fr * sd1;
      g2 = dz * sY + fr * sd2;
      if constexpr (STRESS) {
        const float rf = float(r), rx = -rf * dx, ry = -rf * dy, rz = -rf * dz;
        t6[0] = rx * g0;
        t6[1] = ry * g1;
        t6[2] = rz * g2;
        t6[3] = ry * g2;
        t6[4] = rz * g0;
        t6[5] = rx * g1;
      }
      atomicAdd(&F[3 * size_t(j) + 0], -double(g0));
      atomicAdd(&F[3 * size_t(j) + 1], -double(g1));
      atomicAdd(&F[3 * size_t(j) + 2], -double(g2));
    }
    // F_i += g unless j is a periodic image of i: the centre's pairs are
    // consecutive lanes, so a segmented warp scan leaves each run's sum in
    // its last lane and one atomic per run and component remains.
    float h0 = (j >= 0 && j != self_atom) ? g0 : 0.f;
    float h1 = (j >= 0 && j != self_atom) ? g1 : 0.f;
    float h2 = (j >= 0 && j != self_atom) ? g2 : 0.f;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const float u0 = __shfl_up_sync(0xffffffffu, h0, off);
      const float u1 = __shfl_up_sync(0xffffffffu, h1, off);
      const float u2 = __shfl_up_sync(0xffffffffu, h2, off);
      const int32_t cu = __shfl_up_sync(0xffffffffu, ci, off);
      if (lane >= off && cu == ci) {
        h0 += u0;
        h1 += u1;
        h2 += u2;
      }
    }
    const int32_t cn = __shfl_down_sync(0xffffffffu, ci, 1);
    if (ci >= 0 && (lane == 31 || cn != ci)) {
      const int32_t ia = a.center_atom[ci];
      atomicAdd(&F[3 * size_t(ia) + 0], double(h0));
      atomicAdd(&F[3 * size_t(ia) + 1], double(h1));
      atomicAdd(&F[3 * size_t(ia) + 2], double(h2));
    }
    if constexpr (STRESS) {
      // structures are consecutive runs of centres, hence of lanes
      const int32_t sid = ci >= 0 ? center_struct[ci] : -1;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int32_t su = __shfl_up_sync(0xffffffffu, sid, off);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          const float u = __shfl_up_sync(0xffffffffu, t6[k], off);
          if (lane >= off && su == sid) t6[k] += u;
        }
      }
      const int32_t sn = __shfl_down_sync(0xffffffffu, sid, 1);
      if (sid >= 0 && (lane == 31 || sn != sid))
#pragma unroll
        for (int k = 0; k < 6; ++k) atomicAdd(&stress[6 * size_t(sid) + k], double(t6[k]));
    }
  }
}

}  // namespace

void launch_pair_adjoint_fp32(const ExpansionArgs & a, const int32_t * pair_center, int64_t n_pairs,
                              const float * dC, double * forces, cudaStream_t st,
                              const int32_t * center_struct, double * stress) {
  if (a.n_centers == 0 || n_pairs == 0) return;
  sph_constants_tu();
  if (a.fd.n > kMaxN) throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_radial above 16 is not supported on the fast path");
  const TileConfig cfg = tile_config(a.fd.S, a.fd.n, a.fd.L);
  const int threads = std::min(cfg.adj_threads, kThreads);
  int dev = 0, sms = 148;
  RGPU_CUDA(cudaGetDevice(&dev));
  RGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid =
      int(std::min<int64_t>((n_pairs + threads - 1) / threads, int64_t(sms) * cfg.adj_blocks_per_sm));
#define RGPU_ADJ_LAUNCH(LL, NVV)                                                                     \
  if (stress)                                                                                        \
    pair_adjoint_kernel<LL, NVV, true><<<grid, threads, 0, st>>>(a, pair_center, n_pairs, dC, forces,  \
                                                                  center_struct, stress);            \
  else                                                                                               \
    pair_adjoint_kernel<LL, NVV, false><<<grid, threads, 0, st>>>(a, pair_center, n_pairs, dC,        \
                                                                   forces, nullptr, nullptr);
#define RGPU_ADJ_CASE(LL)                                                                            \
  case LL:                                                                                           \
    if (a.fd.n <= 8) {                                                                               \
      RGPU_ADJ_LAUNCH(LL, 8)                                                                         \
    } else {                                                                                         \
      RGPU_ADJ_LAUNCH(LL, 16)                                                                        \
    }                                                                                                \
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
#undef RGPU_ADJ_LAUNCH
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

}  // namespace rgpu
