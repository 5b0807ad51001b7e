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

#ifndef RGPU_ADJ_L0
#define RGPU_ADJ_L0 0
#define RGPU_ADJ_L1 12
#define RGPU_ADJ_DISPATCH
#endif

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
  const bool vec = (n & 3) == 0;  // dE/dc rows of n floats as 16-byte loads
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
    {
      // the lanes of one centre bring its dE/dc row (Sn K floats, read
      // below one lm at a time) towards L2 together, before the spline and
      // Y_lm work, so that the reads below wait on L2 rather than DRAM
      const unsigned same = __match_any_sync(0xffffffffu, ci);
      if (ci >= 0) {
        const int rank = __popc(same & lanemask_lt()), run = __popc(same);
        const char * row = reinterpret_cast<const char *>(dC + size_t(ci) * Sn * K);
        const int lines = (Sn * K * 4 + 127) >> 7;
        for (int k = rank; k < lines; k += run)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(row + (size_t(k) << 7)));
      }
    }
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
                if (4 * qq < n) {
                  const float4 ev = __ldg(E4 + qq);
                  A = fmaf(ev.w, pl[4 * qq + 3],
                           fmaf(ev.z, pl[4 * qq + 2], fmaf(ev.y, pl[4 * qq + 1], fmaf(ev.x, pl[4 * qq], A))));
                  B = fmaf(ev.w, rl[4 * qq + 3],
                           fmaf(ev.z, rl[4 * qq + 2], fmaf(ev.y, rl[4 * qq + 1], fmaf(ev.x, rl[4 * qq], B))));
                }
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

// One instantiation per (L, NV): compiled in the translation unit that owns
// L (the library builds this file once per range of L, in parallel, since
// each instantiation unrolls the spherical-harmonics recurrence).
template <int L>
void adjoint_launch(const ExpansionArgs & a, const int32_t * pair_center, int64_t n_pairs, const float * dC,
                    double * forces, cudaStream_t st, const int32_t * center_struct, double * stress, int grid,
                    int threads) {
  sph_constants_tu();  // this translation unit's copy of the constants
  if (a.fd.n <= 8) {
    if (stress)
      pair_adjoint_kernel<L, 8, true><<<grid, threads, 0, st>>>(a, pair_center, n_pairs, dC, forces, center_struct,
                                                              stress);
    else
      pair_adjoint_kernel<L, 8, false><<<grid, threads, 0, st>>>(a, pair_center, n_pairs, dC, forces, nullptr,
                                                               nullptr);
  } else {
    if (stress)
      pair_adjoint_kernel<L, 16, true><<<grid, threads, 0, st>>>(a, pair_center, n_pairs, dC, forces,
                                                               center_struct, stress);
    else
      pair_adjoint_kernel<L, 16, false><<<grid, threads, 0, st>>>(a, pair_center, n_pairs, dC, forces, nullptr,
                                                                nullptr);
  }
}

}  // namespace

// Launch of the adjoint kernels of one L. Each translation unit
// instantiates it for its own range of L (explicit instantiation below); the
// dispatch refers to the others through extern declarations.
template <int L>
void adjoint_launch_l(const ExpansionArgs & a, const int32_t * pc, int64_t np, const float * dC, double * F,
                      cudaStream_t st, const int32_t * cs, double * S, int grid, int threads) {
  adjoint_launch<L>(a, pc, np, dC, F, st, cs, S, grid, threads);
}

#define RGPU_ADJ_SIG(LL)                                                                                  \
  void adjoint_launch_l<LL>(const ExpansionArgs &, const int32_t *, int64_t, const float *, double *,     \
                            cudaStream_t, const int32_t *, double *, int, int)
#define RGPU_ADJ_INST(LL)                                             \
  template RGPU_ADJ_SIG(LL);
#define RGPU_ADJ_EXTERN(LL)                                           \
  extern template RGPU_ADJ_SIG(LL);
#if RGPU_ADJ_L0 <= 0 && 0 <= RGPU_ADJ_L1
RGPU_ADJ_INST(0)
#else
RGPU_ADJ_EXTERN(0)
#endif
#if RGPU_ADJ_L0 <= 1 && 1 <= RGPU_ADJ_L1
RGPU_ADJ_INST(1)
#else
RGPU_ADJ_EXTERN(1)
#endif
#if RGPU_ADJ_L0 <= 2 && 2 <= RGPU_ADJ_L1
RGPU_ADJ_INST(2)
#else
RGPU_ADJ_EXTERN(2)
#endif
#if RGPU_ADJ_L0 <= 3 && 3 <= RGPU_ADJ_L1
RGPU_ADJ_INST(3)
#else
RGPU_ADJ_EXTERN(3)
#endif
#if RGPU_ADJ_L0 <= 4 && 4 <= RGPU_ADJ_L1
RGPU_ADJ_INST(4)
#else
RGPU_ADJ_EXTERN(4)
#endif
#if RGPU_ADJ_L0 <= 5 && 5 <= RGPU_ADJ_L1
RGPU_ADJ_INST(5)
#else
RGPU_ADJ_EXTERN(5)
#endif
#if RGPU_ADJ_L0 <= 6 && 6 <= RGPU_ADJ_L1
RGPU_ADJ_INST(6)
#else
RGPU_ADJ_EXTERN(6)
#endif
#if RGPU_ADJ_L0 <= 7 && 7 <= RGPU_ADJ_L1
RGPU_ADJ_INST(7)
#else
RGPU_ADJ_EXTERN(7)
#endif
#if RGPU_ADJ_L0 <= 8 && 8 <= RGPU_ADJ_L1
RGPU_ADJ_INST(8)
#else
RGPU_ADJ_EXTERN(8)
#endif
#if RGPU_ADJ_L0 <= 9 && 9 <= RGPU_ADJ_L1
RGPU_ADJ_INST(9)
#else
RGPU_ADJ_EXTERN(9)
#endif
#if RGPU_ADJ_L0 <= 10 && 10 <= RGPU_ADJ_L1
RGPU_ADJ_INST(10)
#else
RGPU_ADJ_EXTERN(10)
#endif
#if RGPU_ADJ_L0 <= 11 && 11 <= RGPU_ADJ_L1
RGPU_ADJ_INST(11)
#else
RGPU_ADJ_EXTERN(11)
#endif
#if RGPU_ADJ_L0 <= 12 && 12 <= RGPU_ADJ_L1
RGPU_ADJ_INST(12)
#else
RGPU_ADJ_EXTERN(12)
#endif
#undef RGPU_ADJ_EXTERN
#undef RGPU_ADJ_INST
#undef RGPU_ADJ_SIG

#ifdef RGPU_ADJ_DISPATCH
void launch_pair_adjoint_fp32(const ExpansionArgs & a, const int32_t * pair_center, int64_t n_pairs,
                              const float * dC, double * forces, cudaStream_t st,
                              const int32_t * center_struct, double * stress) {
  if (a.n_centers == 0 || n_pairs == 0) return;
  if (a.fd.n > kMaxN) throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_radial above 16 is not supported on the fast path");
  const TileConfig cfg = tile_config(a.fd.S, a.fd.n, a.fd.L);
  const int threads = std::min(cfg.adj_threads, kThreads);
  int dev = 0, sms = 148;
  RGPU_CUDA(cudaGetDevice(&dev));
  RGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid =
      int(std::min<int64_t>((n_pairs + threads - 1) / threads, int64_t(sms) * cfg.adj_blocks_per_sm));
#define RGPU_ADJ_CASE(LL)                                                                        \
  case LL:                                                                                       \
    adjoint_launch_l<LL>(a, pair_center, n_pairs, dC, forces, st, center_struct, stress, grid, threads); \
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
#endif

}  // namespace rgpu
