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
constexpr int kMaxN = 16;  // largest max_radial of the FP32 backward
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

// Output (key, n1, n2, l) goes to Ps[key * n^2 + out] with
// out = l * P * n^2 + n2 * n + n1 (the fast column order).
template <int L, int l>
__device__ __forceinline__ float fwd_task(const float * Cp, float * Ps, const Keys & kt, int S, int n,
                                          int n1, int n2, int kstride, int out) {
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
      Ps[kt.kid[sa][sb] * kstride + out] = v;
      ss += v * v;
    }
  }
  return ss;
}

template <int L, int l>
__device__ __forceinline__ float fwd_dispatch(int lrt, const float * Cp, float * Ps, const Keys & kt, int S,
                                              int n, int n1, int n2, int kstride, int out) {
  if constexpr (l > L) {
    return 0.f;
  } else {
    if (lrt == l) return fwd_task<L, l>(Cp, Ps, kt, S, n, n1, n2, kstride, out);
    return fwd_dispatch<L, l + 1>(lrt, Cp, Ps, kt, S, n, n1, n2, kstride, out);
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
  float * Ps = Cp + size_t(S) * n * RS;    // [D], fast column order
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
    const int n2 = r / n, n1 = r - n2 * n;  // consecutive lanes: consecutive n1 and Ps words
    ss += fwd_dispatch<L, 0>(l, Cp, Ps, kt, S, n, n1, n2, nn2, l * fd.P * nn2 + r);
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
// Quotient x / d for a runtime divisor d >= 1, exact whenever x * d < 2^32
// (multiply by the rounded-up reciprocal 2^32 / d).
struct FastDiv {
  uint32_t d, m;
  FastDiv() = default;
  __host__ __device__ explicit FastDiv(uint32_t dd) : d(dd), m(dd > 1 ? 0xFFFFFFFFu / dd + 1u : 0u) {}
  __device__ __forceinline__ uint32_t div(uint32_t x) const { return d > 1 ? __umulhi(x, m) : x; }
};

struct BwdShape {
  FastDiv n, P, npair, Snp;  // n, key count, n(n-1)/2, S n(n-1)/2
  int LS;                    // floats per H_l block in shared memory
  bool vec;                  // n and S n multiples of 4: 16-byte stores of 4 n1
};

// dE/dc_{i l m} = lf_l sum_j H_l[i][j] c_{j l m} for one row i = (a, n1);
// H_l is read from the transposed slot H_l[j][i], so the 32 lanes of a warp
// (consecutive i) read 32 consecutive words while the c_j loads broadcast.
template <int L, int l>
__device__ __forceinline__ void bwd_task(const float * Cp, const float * Hs, int LS, int Sn, int i,
                                         float * __restrict__ out) {
  constexpr int RS = row_stride(L), Q = pad4(2 * l + 1) / 4, O = offp(l), M = 2 * l + 1;
  float4 acc[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) acc[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  const float * h = Hs + l * LS + i;
  const float * cb = Cp + O;
#pragma unroll 4
  for (int j = 0; j < Sn; ++j) {
    const float hv = h[j * Sn];
    const float4 * c4 = reinterpret_cast<const float4 *>(cb + j * RS);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const float4 c = c4[q];
      acc[q].x += hv * c.x;
      acc[q].y += hv * c.y;
      acc[q].z += hv * c.z;
      acc[q].w += hv * c.w;
    }
  }
  const float lf = rsqrtf(float(M));
  const float * av = reinterpret_cast<const float *>(acc);
#pragma unroll
  for (int m = 0; m < M; ++m) out[(l * l + m) * Sn + i] = av[m] * lf;
}

template <int L, int l>
__device__ __forceinline__ void bwd_dispatch(int lrt, const float * Cp, const float * Hs, int LS, int Sn, int i,
                                             float * out) {
  if constexpr (l <= L) {
    if (lrt == l)
      bwd_task<L, l>(Cp, Hs, LS, Sn, i, out);
    else
      bwd_dispatch<L, l + 1>(lrt, Cp, Hs, LS, Sn, i, out);
  }
}

// One CTA per centre. The projected gradient G = (g - x (x.g)) / |p| (x as
// BF16 hi + lo, g = dE/dx, both in the fast column order) is formed in two
// passes over the row: the first reduces x.g, the second (an L2 re-read)
// scatters G into the symmetric matrices
//   H_l[(a n1)][(b n2)] = s_ab G_(ab)(n1 n2 l)   (a < b, both triangles)
//   H_l[(a n1)][(a n2)] = G(n1 n2 l) + G(n2 n1 l)
// then each thread computes one (l, row) of dE/dc = lf_l H_l c_l.
template <int L>
__global__ void __launch_bounds__(kThreads)
ps_bwd_f32_kernel(PsArgs a, BwdShape bs, const float * __restrict__ C, const __nv_bfloat16 * __restrict__ Xh,
                  const __nv_bfloat16 * __restrict__ Xl, const float * __restrict__ norm,
                  const float * __restrict__ dX, float * __restrict__ dC) {
  constexpr int L1 = L + 1, RS = row_stride(L), K = L1 * L1;
  extern __shared__ __align__(16) float smf[];
  const FeatureDims fd = a.fd;
  const int n = fd.n, S = fd.S, Sn = S * n, LS = bs.LS, P = fd.P;
  float * Cp = smf;             // [Sn][RS]
  float * Hs = Cp + Sn * RS;    // H_l[j][i] at l*LS + j*Sn + i
  __shared__ Keys kt;
  __shared__ float red[32];
  __shared__ int8_t pair_n1[kMaxN * (kMaxN - 1) / 2], pair_n2[kMaxN * (kMaxN - 1) / 2];
  make_keys(kt, S);
  if (threadIdx.x < n * n) {
    const int n1 = threadIdx.x / n, n2 = threadIdx.x - n1 * n;
    if (n1 < n2) {
      const int p = n1 * (2 * n - n1 - 1) / 2 + (n2 - n1 - 1);
      pair_n1[p] = int8_t(n1);
      pair_n2[p] = int8_t(n2);
    }
  }
  const int64_t ci = blockIdx.x;
  const int64_t row = a.row_of_center[ci];
  load_padded<L>(C + size_t(ci) * S * fd.nK, Cp, S, n);
  const uint2 * xh = reinterpret_cast<const uint2 *>(Xh + size_t(row) * fd.Dpad);
  const uint2 * xl = reinterpret_cast<const uint2 *>(Xl + size_t(row) * fd.Dpad);
  const float4 * g4 = reinterpret_cast<const float4 *>(dX + size_t(row) * fd.Dpad);
  const int nq = (fd.D + 3) >> 2;
  float dot = 0.f;
  if (a.normalize) {
    for (int c = threadIdx.x; c < nq; c += blockDim.x) {
      const uint2 hv = xh[c], lv = xl[c];
      const float4 gq = g4[c];
      const __nv_bfloat16 * hb = reinterpret_cast<const __nv_bfloat16 *>(&hv);
      const __nv_bfloat16 * lb = reinterpret_cast<const __nv_bfloat16 *>(&lv);
      dot += (__bfloat162float(hb[0]) + __bfloat162float(lb[0])) * gq.x;
      dot += (__bfloat162float(hb[1]) + __bfloat162float(lb[1])) * gq.y;
      dot += (__bfloat162float(hb[2]) + __bfloat162float(lb[2])) * gq.z;
      dot += (__bfloat162float(hb[3]) + __bfloat162float(lb[3])) * gq.w;
    }
    dot = block_sum_f(dot, red);  // padding columns are zero in x and g
  }
  const float invn = 1.f / norm[ci];
  for (int c = threadIdx.x; c < nq; c += blockDim.x) {
    const uint2 hv = __ldcs(xh + c), lv = __ldcs(xl + c);
    const float4 gq = __ldcs(g4 + c);
    const __nv_bfloat16 * hb = reinterpret_cast<const __nv_bfloat16 *>(&hv);
    const __nv_bfloat16 * lb = reinterpret_cast<const __nv_bfloat16 *>(&lv);
    const float gv[4] = {gq.x, gq.y, gq.z, gq.w};
    float G[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) G[e] = (gv[e] - (__bfloat162float(hb[e]) + __bfloat162float(lb[e])) * dot) * invn;
    // decode the first column of the chunk: ((l*P + key)*n + n2)*n + n1
    const uint32_t d0 = 4u * uint32_t(c);
    const uint32_t q1 = bs.n.div(d0);
    int n1 = int(d0 - q1 * bs.n.d);
    const uint32_t q2 = bs.n.div(q1);
    int n2 = int(q1 - q2 * bs.n.d);
    const uint32_t q3 = bs.P.div(q2);
    int key = int(q2 - q3 * bs.P.d);
    int l = int(q3);
    if (bs.vec) {
      // the 4 columns share (l, key, n2) and n1 % 4 == 0: one 16-byte store
      // for H[(b n2)][(a n1..n1+3)], four for the mirrored column
      const int sa = kt.ka[key], sb = kt.kb[key];
      const int i = sa * n + n1, j = sb * n + n2;
      float * Hl = Hs + l * LS;
      if (sa != sb) {
        float v[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) v[e] = kSqrt2f * G[e];
        *reinterpret_cast<float4 *>(Hl + j * Sn + i) = make_float4(v[0], v[1], v[2], v[3]);
#pragma unroll
        for (int e = 0; e < 4; ++e) Hl[(i + e) * Sn + j] = v[e];
      } else {
        float v[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) v[e] = (n1 + e == n2) ? 2.f * G[e] : G[e];
        *reinterpret_cast<float4 *>(Hl + j * Sn + i) = make_float4(v[0], v[1], v[2], v[3]);
      }
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (int(d0) + e < fd.D) {
          const int sa = kt.ka[key], sb = kt.kb[key];
          const int i = sa * n + n1, j = sb * n + n2;
          float * Hl = Hs + l * LS;
          if (sa != sb) {
            Hl[j * Sn + i] = kSqrt2f * G[e];
            Hl[i * Sn + j] = kSqrt2f * G[e];
          } else {
            Hl[j * Sn + i] = (n1 == n2) ? 2.f * G[e] : G[e];
          }
        }
        if (++n1 == n) {
          n1 = 0;
          if (++n2 == n) {
            n2 = 0;
            if (++key == P) {
              key = 0;
              ++l;
            }
          }
        }
      }
    }
  }
  __syncthreads();
  // same-species blocks: H[(a n1)][(a n2)] = H[(a n2)][(a n1)] = G(n1 n2) + G(n2 n1)
  const int nsym = L1 * int(bs.Snp.d);
  for (int t = threadIdx.x; t < nsym; t += blockDim.x) {
    const uint32_t l = bs.Snp.div(uint32_t(t));
    const uint32_t r = uint32_t(t) - l * bs.Snp.d;
    const uint32_t sa = bs.npair.div(r);
    const int p = int(r - sa * bs.npair.d);
    const int i = int(sa) * n + pair_n1[p], j = int(sa) * n + pair_n2[p];
    float * Hl = Hs + l * LS;
    const float s = Hl[j * Sn + i] + Hl[i * Sn + j];
    Hl[j * Sn + i] = s;
    Hl[i * Sn + j] = s;
  }
  __syncthreads();
  float * out = dC + size_t(ci) * Sn * K;
  for (int t = threadIdx.x; t < L1 * Sn; t += blockDim.x) {
    const int lr = t / Sn;
    bwd_dispatch<L, 0>(L - lr, Cp, Hs, LS, Sn, t - lr * Sn, out);
  }
}

template <int L>
size_t fwd_smem(const FeatureDims & fd) {
  return sizeof(float) * (size_t(fd.S) * fd.n * row_stride(L) + fd.D + 4);
}

BwdShape bwd_shape(const FeatureDims & fd) {
  BwdShape b;
  const uint32_t n = uint32_t(fd.n), Sn = uint32_t(fd.S) * n, npair = n * (n - 1) / 2;
  b.n = FastDiv(n);
  b.P = FastDiv(uint32_t(fd.P));
  b.npair = FastDiv(npair > 0 ? npair : 1u);
  b.Snp = FastDiv(npair > 0 ? uint32_t(fd.S) * npair : 1u);
  if (npair == 0) b.Snp.d = 0;  // no off-diagonal pairs: the symmetrisation loop is empty
  // a multiple of 4 (16-byte rows) that is not a multiple of 32, so the
  // L+1 blocks start on different banks
  b.LS = int((Sn * Sn + 3) / 4 * 4);
  if (b.LS % 32 == 0) b.LS += 4;
  b.vec = (n % 4 == 0) && (Sn % 4 == 0);
  return b;
}

template <int L>
size_t bwd_smem(const FeatureDims & fd, const BwdShape & b) {
  return sizeof(float) * (size_t(fd.S) * fd.n * row_stride(L) + size_t(L + 1) * b.LS);
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
  if (a.fd.n > kMaxN) throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_radial above 16 is not supported on the fast path");
  const BwdShape bs = bwd_shape(a.fd);
  constexpr size_t kMaxSmem = 227 * 1024 - 2048;
#define RGPU_PSB_CASE(LL)                                                                                     \
  case LL: {                                                                                                  \
    const size_t smem = bwd_smem<LL>(a.fd, bs);                                                               \
    if (smem > kMaxSmem)                                                                                      \
      throw Error(RGPU_ERR_INVALID_ARGUMENT,                                                                  \
                  "species x max_radial too large for the FP32 power-spectrum backward; use FP64");           \
    RGPU_CUDA(cudaFuncSetAttribute(ps_bwd_f32_kernel<LL>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                   int(smem)));                                                               \
    ps_bwd_f32_kernel<LL><<<int(a.n_centers), kThreads, smem, st>>>(a, bs, C, Xh, Xl, norm, dX, dC);          \
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
