// Power spectrum, FP32 fast path: forward (x and its BF16 hi/lo split for
// the tensor-core GEMMs) and the adjoint dE/dx -> dE/dc.
//
// Same contractions as powerspectrum.cu (calculator_spherical_invariants.hh:
// 747-794 forward, 588-652 and 796-921 for the gradient it replaces), laid
// out for the SIMT pipes: the centre's coefficients sit in shared memory as
// [species][n][l-block padded to a multiple of 4], so every length-(2l+1)
// product over m is a few 16-byte loads; work items are ordered with l
// slowest, so a warp shares l (uniform trip counts, broadcast loads) and the
// dot products are unrolled per l.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace rgpu {
namespace {

constexpr int kThreads = 256;
constexpr float kSqrt2f = 1.41421356237309504880f;

__host__ __device__ constexpr int pad4(int x) { return (x + 3) & ~3; }
// padded offset of block l: sum_{l' < l} pad4(2l'+1)
__host__ __device__ constexpr int offp(int l) {
  int o = 0;
  for (int i = 0; i < l; ++i) o += pad4(2 * i + 1);
  return o;
}
// row stride of the padded layout: the block sum rounded so that stride/4
// is odd (conflict-free 16-byte loads across 8 consecutive rows)
__host__ __device__ constexpr int row_stride(int L) {
  int s = offp(L + 1);
  return ((s / 4) % 2 == 1) ? s : s + 4;
}

struct Keys {
  int8_t ka[kMaxSpecies * (kMaxSpecies + 1) / 2];
  int8_t kb[kMaxSpecies * (kMaxSpecies + 1) / 2];
  int16_t kid[kMaxSpecies][kMaxSpecies];
};
__device__ __forceinline__ void make_keys(Keys & t, int S) {
  if (threadIdx.x == 0) {
    int k = 0;
    for (int a = 0; a < S; ++a)
      for (int b = a; b < S; ++b) {
        t.ka[k] = int8_t(a);
        t.kb[k] = int8_t(b);
        t.kid[a][b] = t.kid[b][a] = int16_t(k);
        ++k;
      }
  }
}

__device__ __forceinline__ float block_sum_f(float v, float * red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  float t = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.f;
  if (wid == 0) t = warp_sum(t);
  if (threadIdx.x == 0) red[0] = t;
  __syncthreads();
  return red[0];
}

// Source index (l^2 + m) of every padded column, -1 for padding.
template <int L>
struct PadMap {
  int8_t src[row_stride(L)];
  constexpr PadMap() : src() {
    int c = 0;
    for (int l = 0; l <= L; ++l)
      for (int m = 0; m < pad4(2 * l + 1); ++m) src[c++] = int8_t(m < 2 * l + 1 ? l * l + m : -1);
    for (; c < row_stride(L); ++c) src[c] = -1;
  }
};

// Load c^i (S x n x K, K = (L+1)^2) into the padded layout.
template <int L>
__device__ __forceinline__ void load_padded(const float * __restrict__ Ci, float * Cp, int S, int n) {
  constexpr int K = (L + 1) * (L + 1), RS = row_stride(L);
  constexpr PadMap<L> pm;
  __shared__ int8_t src[RS];
  if (threadIdx.x < RS) src[threadIdx.x] = pm.src[threadIdx.x];
  __syncthreads();
  for (int e = threadIdx.x; e < S * n * RS; e += blockDim.x) {
    const int row = e / RS, c = e - row * RS;
    const int s = src[c];
    Cp[e] = (s >= 0) ? Ci[row * K + s] : 0.f;
  }
}

template <int Q>
__device__ __forceinline__ float dot4(const float4 * a, const float * b) {
  const float4 * b4 = reinterpret_cast<const float4 *>(b);
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const float4 y = b4[q];
    s += a[q].x * y.x + a[q].y * y.y + a[q].z * y.z + a[q].w * y.w;
  }
  return s;
}

template <int L, int l>
__device__ __forceinline__ float fwd_task(const float * Cp, float * Ps, const Keys & kt, int S, int n,
                                          int n1, int n2, int blk, int out) {
  constexpr int RS = row_stride(L), Q = pad4(2 * l + 1) / 4, O = offp(l);
  const float lf = rsqrtf(float(2 * l + 1));
  float ss = 0.f;
  for (int sa = 0; sa < S; ++sa) {
    float4 c1[Q];
    const float4 * p1 = reinterpret_cast<const float4 *>(Cp + (sa * n + n1) * RS + O);
#pragma unroll
    for (int q = 0; q < Q; ++q) c1[q] = p1[q];
    for (int sb = sa; sb < S; ++sb) {
      float v = dot4<Q>(c1, Cp + (sb * n + n2) * RS + O) * lf;
      if (sa < sb) v *= kSqrt2f;
      Ps[kt.kid[sa][sb] * blk + out] = v;
      ss += v * v;
    }
  }
  return ss;
}

template <int L, int l>
__device__ __forceinline__ float fwd_dispatch(int lrt, const float * Cp, float * Ps, const Keys & kt, int S,
                                              int n, int n1, int n2, int blk, int out) {
  if constexpr (l > L) {
    return 0.f;
  } else {
    if (lrt == l) return fwd_task<L, l>(Cp, Ps, kt, S, n, n1, n2, blk, out);
    return fwd_dispatch<L, l + 1>(lrt, Cp, Ps, kt, S, n, n1, n2, blk, out);
  }
}

template <int L>
__global__ void __launch_bounds__(kThreads)
ps_fwd_f32_kernel(PsArgs a, const float * __restrict__ C, float * __restrict__ X,
                  __nv_bfloat16 * __restrict__ Xh, __nv_bfloat16 * __restrict__ Xl,
                  float * __restrict__ norm_out) {
  constexpr int L1 = L + 1, RS = row_stride(L);
  extern __shared__ __align__(16) float smf[];
  const FeatureDims fd = a.fd;
  const int n = fd.n, S = fd.S, nn2 = n * n, blk = nn2 * L1;
  float * Cp = smf;                        // [S*n][RS]
  float * Ps = Cp + size_t(S) * n * RS;    // [D]
  __shared__ Keys kt;
  __shared__ float red[32];
  make_keys(kt, S);
  const int64_t ci = blockIdx.x;
  load_padded<L>(C + size_t(ci) * S * fd.nK, Cp, S, n);
  __syncthreads();
  float ss = 0.f;
  for (int t = threadIdx.x; t < blk; t += blockDim.x) {
    const int l = t / nn2;
    const int r = t - l * nn2;
    const int n1 = r / n, n2 = r - n1 * n;
    ss += fwd_dispatch<L, 0>(l, Cp, Ps, kt, S, n, n1, n2, blk, r * L1 + l);
  }
  ss = block_sum_f(ss, red);
  const float nrm = sqrtf(ss);
  const bool do_norm = a.normalize && nrm > 0.f;
  const float rinv = do_norm ? 1.f / nrm : 1.f;
  const size_t roff = size_t(a.row_of_center[ci]) * fd.Dpad;
  for (int d0 = threadIdx.x * 4; d0 < fd.Dpad; d0 += blockDim.x * 4) {
    float v[4];
    if (d0 + 4 <= fd.D) {
      const float4 p = *reinterpret_cast<const float4 *>(Ps + d0);
      v[0] = p.x;
      v[1] = p.y;
      v[2] = p.z;
      v[3] = p.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i] = (d0 + i < fd.D) ? Ps[d0 + i] : 0.f;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] *= rinv;
    if (X) *reinterpret_cast<float4 *>(X + roff + d0) = make_float4(v[0], v[1], v[2], v[3]);
    __align__(8) __nv_bfloat16 h[4], lo[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      h[i] = __float2bfloat16_rn(v[i]);
      lo[i] = __float2bfloat16_rn(v[i] - __bfloat162float(h[i]));
    }
    *reinterpret_cast<uint2 *>(Xh + roff + d0) = *reinterpret_cast<uint2 *>(h);
    *reinterpret_cast<uint2 *>(Xl + roff + d0) = *reinterpret_cast<uint2 *>(lo);
  }
  if (threadIdx.x == 0) norm_out[ci] = a.normalize ? nrm : 1.f;
}

// ---------------------------------------------------------------- backward
template <int L, int l>
__device__ __forceinline__ void bwd_task(const float * Cp, const float * Gs, const Keys & kt, int S, int n,
                                         int sa, int n1, int blk, float * __restrict__ out) {
  constexpr int L1 = L + 1, RS = row_stride(L), Q = pad4(2 * l + 1) / 4, O = offp(l), M = 2 * l + 1;
  float4 acc[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) acc[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int sb = 0; sb < S; ++sb) {
    const float * gk = Gs + size_t(kt.kid[sa][sb]) * blk + l;
    const float w = (sa == sb) ? 1.f : kSqrt2f;
    for (int n2 = 0; n2 < n; ++n2) {
      float h;
      if (sa < sb)
        h = gk[(n1 * n + n2) * L1];
      else if (sa > sb)
        h = gk[(n2 * n + n1) * L1];
      else
        h = gk[(n1 * n + n2) * L1] + gk[(n2 * n + n1) * L1];
      h *= w;
      const float4 * cb = reinterpret_cast<const float4 *>(Cp + (sb * n + n2) * RS + O);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const float4 c = cb[q];
        acc[q].x += h * c.x;
        acc[q].y += h * c.y;
        acc[q].z += h * c.z;
        acc[q].w += h * c.w;
      }
    }
  }
  const float lf = rsqrtf(float(M));
  const float * av = reinterpret_cast<const float *>(acc);
#pragma unroll
  for (int m = 0; m < M; ++m) out[l * l + m] = av[m] * lf;
}

template <int L, int l>
__device__ __forceinline__ void bwd_dispatch(int lrt, const float * Cp, const float * Gs, const Keys & kt, int S,
                                             int n, int sa, int n1, int blk, float * out) {
  if constexpr (l <= L) {
    if (lrt == l)
      bwd_task<L, l>(Cp, Gs, kt, S, n, sa, n1, blk, out);
    else
      bwd_dispatch<L, l + 1>(lrt, Cp, Gs, kt, S, n, sa, n1, blk, out);
  }
}

template <int L>
__global__ void __launch_bounds__(kThreads)
ps_bwd_f32_kernel(PsArgs a, const float * __restrict__ C, const __nv_bfloat16 * __restrict__ Xh,
                  const __nv_bfloat16 * __restrict__ Xl, const float * __restrict__ norm,
                  const float * __restrict__ dX, float * __restrict__ dC) {
  constexpr int L1 = L + 1, RS = row_stride(L);
  extern __shared__ __align__(16) float smf[];
  const FeatureDims fd = a.fd;
  const int n = fd.n, S = fd.S, blk = n * n * L1, Sn = S * n;
  float * Cp = smf;
  float * Gs = Cp + size_t(S) * n * RS;
  __shared__ Keys kt;
  __shared__ float red[32];
  make_keys(kt, S);
  const int64_t ci = blockIdx.x;
  const int64_t row = a.row_of_center[ci];
  load_padded<L>(C + size_t(ci) * S * fd.nK, Cp, S, n);
  // x = hi + lo, g = dE/dx; the projection of the normalisation backward
  const uint4 * xh4 = reinterpret_cast<const uint4 *>(Xh + size_t(row) * fd.Dpad);
  const uint4 * xl4 = reinterpret_cast<const uint4 *>(Xl + size_t(row) * fd.Dpad);
  const float4 * g4 = reinterpret_cast<const float4 *>(dX + size_t(row) * fd.Dpad);
  float dot = 0.f;
  for (int c8 = threadIdx.x; c8 * 8 < fd.Dpad; c8 += blockDim.x) {
    const uint4 hv = xh4[c8], lv = xl4[c8];
    const __nv_bfloat16 * hb = reinterpret_cast<const __nv_bfloat16 *>(&hv);
    const __nv_bfloat16 * lb = reinterpret_cast<const __nv_bfloat16 *>(&lv);
    const float4 ga = g4[2 * c8], gb = g4[2 * c8 + 1];
    const float gv[8] = {ga.x, ga.y, ga.z, ga.w, gb.x, gb.y, gb.z, gb.w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float x = __bfloat162float(hb[i]) + __bfloat162float(lb[i]);
      dot += x * gv[i];
      const int d = c8 * 8 + i;
      if (d < fd.D) Gs[d] = x;
    }
  }
  dot = a.normalize ? block_sum_f(dot, red) : 0.f;
  const float invn = 1.f / norm[ci];
  for (int c8 = threadIdx.x; c8 * 8 < fd.Dpad; c8 += blockDim.x) {
    const float4 ga = g4[2 * c8], gb = g4[2 * c8 + 1];
    const float gv[8] = {ga.x, ga.y, ga.z, ga.w, gb.x, gb.y, gb.z, gb.w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int d = c8 * 8 + i;
      if (d < fd.D) Gs[d] = (gv[i] - Gs[d] * dot) * invn;
    }
  }
  __syncthreads();
  float * Ci_out = dC + size_t(ci) * S * fd.nK;
  for (int t = threadIdx.x; t < Sn * L1; t += blockDim.x) {
    const int l = t / Sn;
    const int r = t - l * Sn;
    const int sa = r / n, n1 = r - sa * n;
    bwd_dispatch<L, 0>(l, Cp, Gs, kt, S, n, sa, n1, blk, Ci_out + sa * fd.nK + n1 * fd.K);
  }
}

template <int L>
size_t fwd_smem(const FeatureDims & fd) {
  return sizeof(float) * (size_t(fd.S) * fd.n * row_stride(L) + fd.D + 4);
}

}  // namespace

void launch_ps_fwd_fp32(const PsArgs & a, const float * C, float * X, __nv_bfloat16 * Xh,
                        __nv_bfloat16 * Xl, float * norm, cudaStream_t st) {
  if (a.n_centers == 0) return;
  if (!Xh || !Xl) throw Error(RGPU_ERR_INVALID_ARGUMENT, "FP32 power spectrum needs the BF16 outputs");
#define RGPU_PSF_CASE(LL)                                                                                     \
  case LL: {                                                                                                  \
    const size_t smem = fwd_smem<LL>(a.fd);                                                                   \
    RGPU_CUDA(cudaFuncSetAttribute(ps_fwd_f32_kernel<LL>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                   int(smem)));                                                               \
    ps_fwd_f32_kernel<LL><<<int(a.n_centers), kThreads, smem, st>>>(a, C, X, Xh, Xl, norm);                 \
    break;                                                                                                    \
  }
  switch (a.fd.L) {
    RGPU_PSF_CASE(0)
    RGPU_PSF_CASE(1)
    RGPU_PSF_CASE(2)
    RGPU_PSF_CASE(3)
    RGPU_PSF_CASE(4)
    RGPU_PSF_CASE(5)
    RGPU_PSF_CASE(6)
    RGPU_PSF_CASE(7)
    RGPU_PSF_CASE(8)
    RGPU_PSF_CASE(9)
    RGPU_PSF_CASE(10)
    RGPU_PSF_CASE(11)
    RGPU_PSF_CASE(12)
    default:
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_angular above 12 is not supported on the GPU");
  }
#undef RGPU_PSF_CASE
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

void launch_ps_bwd_fp32(const PsArgs & a, const float * C, const __nv_bfloat16 * Xh, const __nv_bfloat16 * Xl,
                        const float * norm, const float * dX, float * dC, cudaStream_t st) {
  if (a.n_centers == 0) return;
#define RGPU_PSB_CASE(LL)                                                                                     \
  case LL: {                                                                                                  \
    const size_t smem = fwd_smem<LL>(a.fd);                                                                   \
    RGPU_CUDA(cudaFuncSetAttribute(ps_bwd_f32_kernel<LL>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                   int(smem)));                                                               \
    ps_bwd_f32_kernel<LL><<<int(a.n_centers), kThreads, smem, st>>>(a, C, Xh, Xl, norm, dX, dC);            \
    break;                                                                                                    \
  }
  switch (a.fd.L) {
    RGPU_PSB_CASE(0)
    RGPU_PSB_CASE(1)
    RGPU_PSB_CASE(2)
    RGPU_PSB_CASE(3)
    RGPU_PSB_CASE(4)
    RGPU_PSB_CASE(5)
    RGPU_PSB_CASE(6)
    RGPU_PSB_CASE(7)
    RGPU_PSB_CASE(8)
    RGPU_PSB_CASE(9)
    RGPU_PSB_CASE(10)
    RGPU_PSB_CASE(11)
    RGPU_PSB_CASE(12)
    default:
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_angular above 12 is not supported on the GPU");
  }
#undef RGPU_PSB_CASE
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

}  // namespace rgpu
