// Power spectrum, FP32 fast path: forward (the unnormalised p as a BF16
// hi/lo split for the tensor-core GEMMs, plus 1/|p| per row, which the GEMM
// epilogue and the backward apply) and the adjoint dE/dx -> dE/dc.
//
// Same contractions as powerspectrum.cu (calculator_spherical_invariants.hh:
// 747-794 forward, 588-652 and 796-921 for the gradient it replaces), laid
// out for the SIMT pipes: the centre's coefficients sit in shared memory as
// [species][n][l-block padded to a multiple of 4], so every length-(2l+1)
// product over m is a few 16-byte loads; work items are ordered with l
// slowest, so a warp shares l (uniform trip counts, broadcast loads) and the
// dot products are unrolled per l.
#include <algorithm>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace rgpu {
namespace {

constexpr int kThreads = 256;
constexpr int kBwdThreads = 320;  // 16 column groups x 20 row pairs at L = 6, S n = 40
constexpr int kMaxN = 16;  // largest max_radial of the FP32 backward
constexpr float kSqrt2f = 1.41421356237309504880f;

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

// Copy c^i, already in the padded row layout [S*n][row_stride(L)] of the
// FP32 expansion, into shared memory. Starts with a barrier so that tables
// the block wrote before are visible afterwards.
template <int L>
__device__ __forceinline__ void load_padded(const float * __restrict__ Ci, float * Cp, int S, int n) {
  constexpr int RS = row_stride(L);
  __syncthreads();
  const float4 * src = reinterpret_cast<const float4 *>(Ci);
  float4 * dst = reinterpret_cast<float4 *>(Cp);
  for (int e = threadIdx.x; e < S * n * (RS / 4); e += blockDim.x) dst[e] = __ldg(src + e);
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

// Output (key, n1, n2, l) is column key * n^2 + out of the row, with
// out = l * P * n^2 + n2 * n + n1 (the fast column order): the 32 lanes of a
// warp (consecutive n1, n2) store 32 consecutive columns for every key.
// Values are the unnormalised p; the row's 1/|p| is applied by the consumers.
template <int L, int l>
__device__ __forceinline__ float fwd_task(const float * Cp, const Keys & kt, int S, int n, int n1, int n2,
                                          int kstride, int out, float * __restrict__ X,
                                          __nv_bfloat16 * __restrict__ Xh, __nv_bfloat16 * __restrict__ Xl) {
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
      const int pos = kt.kid[sa][sb] * kstride + out;
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      Xh[pos] = h;
      Xl[pos] = __float2bfloat16_rn(v - __bfloat162float(h));
      if (X) X[pos] = v;
      ss += v * v;
    }
  }
  return ss;
}

template <int L, int l>
__device__ __forceinline__ float fwd_dispatch(int lrt, const float * Cp, const Keys & kt, int S, int n, int n1,
                                              int n2, int kstride, int out, float * X, __nv_bfloat16 * Xh,
                                              __nv_bfloat16 * Xl) {
  if constexpr (l > L) {
    return 0.f;
  } else {
    if (lrt == l) return fwd_task<L, l>(Cp, kt, S, n, n1, n2, kstride, out, X, Xh, Xl);
    return fwd_dispatch<L, l + 1>(lrt, Cp, kt, S, n, n1, n2, kstride, out, X, Xh, Xl);
  }
}

// Two consecutive radial indices n1, n1+1 (n1 even) of one (l, n2): each
// c_b load feeds both dot products, and the two outputs are consecutive
// columns, stored as packed bf16 pairs (4-byte stores).
template <int L, int l>
__device__ __forceinline__ float fwd_task2(const float * Cp, const Keys & kt, int S, int n, int n1, int n2,
                                           int kstride, int out, float * __restrict__ X,
                                           __nv_bfloat16 * __restrict__ Xh, __nv_bfloat16 * __restrict__ Xl) {
  constexpr int RS = row_stride(L), Q = pad4(2 * l + 1) / 4, O = offp(l);
  const float lf = rsqrtf(float(2 * l + 1));
  float ss = 0.f;
  for (int sa = 0; sa < S; ++sa) {
    float4 ca[Q], cb[Q];
    const float4 * pa = reinterpret_cast<const float4 *>(Cp + (sa * n + n1) * RS + O);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      ca[q] = pa[q];
      cb[q] = pa[q + RS / 4];
    }
    for (int sb = sa; sb < S; ++sb) {
      const float4 * p2 = reinterpret_cast<const float4 *>(Cp + (sb * n + n2) * RS + O);
      float va = 0.f, vb = 0.f;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const float4 y = p2[q];
        va += ca[q].x * y.x + ca[q].y * y.y + ca[q].z * y.z + ca[q].w * y.w;
        vb += cb[q].x * y.x + cb[q].y * y.y + cb[q].z * y.z + cb[q].w * y.w;
      }
      const float sc = (sa < sb) ? lf * kSqrt2f : lf;
      va *= sc;
      vb *= sc;
      const int pos = kt.kid[sa][sb] * kstride + out;
      const __nv_bfloat162 hh = __floats2bfloat162_rn(va, vb);
      const float2 hf = __bfloat1622float2(hh);
      *reinterpret_cast<__nv_bfloat162 *>(Xh + pos) = hh;
      *reinterpret_cast<__nv_bfloat162 *>(Xl + pos) = __floats2bfloat162_rn(va - hf.x, vb - hf.y);
      if (X) *reinterpret_cast<float2 *>(X + pos) = make_float2(va, vb);
      ss += va * va + vb * vb;
    }
  }
  return ss;
}

template <int L, int l>
__device__ __forceinline__ float fwd_dispatch2(int lrt, const float * Cp, const Keys & kt, int S, int n, int n1,
                                               int n2, int kstride, int out, float * X, __nv_bfloat16 * Xh,
                                               __nv_bfloat16 * Xl) {
  if constexpr (l > L) {
    return 0.f;
  } else {
    if (lrt == l) return fwd_task2<L, l>(Cp, kt, S, n, n1, n2, kstride, out, X, Xh, Xl);
    return fwd_dispatch2<L, l + 1>(lrt, Cp, kt, S, n, n1, n2, kstride, out, X, Xh, Xl);
  }
}

// p of a centre's row as a BF16 hi/lo split (and in FP32 when X is given),
// straight from the dot products to HBM, and the row's scale 1/|p| (1
// without normalisation). Persistent: each block loops over centres.
template <int L>
__global__ void __launch_bounds__(kThreads)
ps_fwd_f32_kernel(PsArgs a, const float * __restrict__ C, float * __restrict__ X,
                  __nv_bfloat16 * __restrict__ Xh, __nv_bfloat16 * __restrict__ Xl,
                  float * __restrict__ row_scale) {
  constexpr int L1 = L + 1, RS = row_stride(L);
  extern __shared__ __align__(16) float smf[];
  const FeatureDims fd = a.fd;
  const int n = fd.n, S = fd.S, nn2 = n * n, blk = nn2 * L1;
  float * Cp = smf;  // [S*n][RS]
  __shared__ Keys kt;
  __shared__ float red[32];
  make_keys(kt, S);
  const bool paired = (n % 2) == 0;
  const int half = n / 2;
  for (int64_t ci = blockIdx.x; ci < a.n_centers; ci += gridDim.x) {
    const int64_t row = a.row_of_center[ci];
    load_padded<L>(C + size_t(ci) * S * n * RS, Cp, S, n);
    __syncthreads();
    const size_t roff = size_t(row) * fd.Dpad;
    float * Xr = X ? X + roff : nullptr;
    __nv_bfloat16 * hr = Xh + roff;
    __nv_bfloat16 * lr = Xl + roff;
    float ss = 0.f;
    if (paired) {
      // tasks (l, n2, n1 pair): consecutive lanes store consecutive pairs
      for (int t = threadIdx.x; t < L1 * n * half; t += blockDim.x) {
        const int l = t / (n * half);
        const int r = t - l * (n * half);
        const int n2 = r / half, n1 = 2 * (r - n2 * half);
        ss += fwd_dispatch2<L, 0>(l, Cp, kt, S, n, n1, n2, nn2, l * fd.P * nn2 + n2 * n + n1, Xr, hr, lr);
      }
    } else {
      for (int t = threadIdx.x; t < blk; t += blockDim.x) {
        const int l = t / nn2;
        const int r = t - l * nn2;
        const int n2 = r / n, n1 = r - n2 * n;  // consecutive lanes: consecutive n1 and columns
        ss += fwd_dispatch<L, 0>(l, Cp, kt, S, n, n1, n2, nn2, l * fd.P * nn2 + r, Xr, hr, lr);
      }
    }
    for (int d = fd.D + threadIdx.x; d < fd.Dpad; d += blockDim.x) {
      hr[d] = __float2bfloat16_rn(0.f);
      lr[d] = __float2bfloat16_rn(0.f);
      if (Xr) Xr[d] = 0.f;
    }
    ss = block_sum_f(ss, red);  // ends with a barrier: Cp may be refilled
    if (threadIdx.x == 0) {
      const float nrm = sqrtf(ss);
      row_scale[row] = (a.normalize && nrm > 0.f) ? 1.f / nrm : 1.f;
    }
  }
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
  int SnP;                   // row stride of H_l: S n rounded up to even
  int LS;                    // floats per H_l block in shared memory
  bool vec;                  // n and S n multiples of 4: 16-byte stores of 4 n1
};

// One CTA per centre. The projected gradient G = (g - x (x.g)) / |p| (x as
// BF16 hi + lo, g = dE/dx, both in the fast column order) is formed in two
// passes over the row: the first reduces x.g, the second (an L2 re-read)
// scatters G into the symmetric matrices
//   H_l[(a n1)][(b n2)] = s_ab G_(ab)(n1 n2 l)   (a < b, both triangles)
//   H_l[(a n1)][(a n2)] = G(n1 n2 l) + G(n2 n1 l)
// then each thread computes one (l, row) of dE/dc = lf_l H_l c_l.
template <int L>
__global__ void __launch_bounds__(kBwdThreads, 4)
ps_bwd_f32_kernel(PsArgs a, BwdShape bs, const float * __restrict__ C, const __nv_bfloat16 * __restrict__ Xh,
                  const __nv_bfloat16 * __restrict__ Xl, const float * __restrict__ row_scale,
                  const float * __restrict__ dX, float * __restrict__ dC) {
  constexpr int L1 = L + 1, RS = row_stride(L), K = L1 * L1;
  extern __shared__ __align__(16) float smf[];
  const FeatureDims fd = a.fd;
  const int n = fd.n, S = fd.S, Sn = S * n, SnP = bs.SnP, LS = bs.LS, P = fd.P;
  float * Cp = smf;             // [Sn][RS]
  float * Hs = Cp + Sn * RS;    // H_l[j][i] at l*LS + j*SnP + i
  __shared__ Keys kt;
  __shared__ float red[32];
  __shared__ int8_t pair_n1[kMaxN * (kMaxN - 1) / 2], pair_n2[kMaxN * (kMaxN - 1) / 2];
  // column groups of the contraction: every 4-wide chunk q of every padded
  // l-block, l descending; group g covers padded columns grp_off[g] + 0..3
  constexpr int kG = offp(L + 1) / 4;
  __shared__ int8_t grp_l[kG];
  __shared__ int16_t grp_off[kG];
  for (int t = threadIdx.x; t < kG; t += blockDim.x) {
    int g = t, l = L;
    while (g >= pad4(2 * l + 1) / 4) {
      g -= pad4(2 * l + 1) / 4;
      --l;
    }
    grp_l[t] = int8_t(l);
    grp_off[t] = int16_t(offp_rt(l) + 4 * g);
  }
  make_keys(kt, S);
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
    const int n1 = t / n, n2 = t - n1 * n;
    if (n1 < n2) {
      const int p = n1 * (2 * n - n1 - 1) / 2 + (n2 - n1 - 1);
      pair_n1[p] = int8_t(n1);
      pair_n2[p] = int8_t(n2);
    }
  }
  // persistent: the tables above serve every centre of this block
  for (int64_t ci = blockIdx.x; ci < a.n_centers; ci += gridDim.x) {
  const int64_t row = a.row_of_center[ci];
  load_padded<L>(C + size_t(ci) * S * n * RS, Cp, S, n);
  const uint2 * xh = reinterpret_cast<const uint2 *>(Xh + size_t(row) * fd.Dpad);
  const uint2 * xl = reinterpret_cast<const uint2 *>(Xl + size_t(row) * fd.Dpad);
  const float4 * g4 = reinterpret_cast<const float4 *>(dX + size_t(row) * fd.Dpad);
  const int nq = (fd.D + 3) >> 2;
  const float rs = row_scale[row];  // x = rs * p; G = rs * (g - x (x.g))
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
    dot = block_sum_f(dot, red) * rs;  // padding columns are zero in p and g
  }
  for (int c = threadIdx.x; c < nq; c += blockDim.x) {
    const uint2 hv = __ldcs(xh + c), lv = __ldcs(xl + c);
    const float4 gq = __ldcs(g4 + c);
    const __nv_bfloat16 * hb = reinterpret_cast<const __nv_bfloat16 *>(&hv);
    const __nv_bfloat16 * lb = reinterpret_cast<const __nv_bfloat16 *>(&lv);
    const float gv[4] = {gq.x, gq.y, gq.z, gq.w};
    float G[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) G[e] = (gv[e] - (__bfloat162float(hb[e]) + __bfloat162float(lb[e])) * rs * dot) * rs;
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
        *reinterpret_cast<float4 *>(Hl + j * SnP + i) = make_float4(v[0], v[1], v[2], v[3]);
#pragma unroll
        for (int e = 0; e < 4; ++e) Hl[(i + e) * SnP + j] = v[e];
      } else {
        float v[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) v[e] = (n1 + e == n2) ? 2.f * G[e] : G[e];
        *reinterpret_cast<float4 *>(Hl + j * SnP + i) = make_float4(v[0], v[1], v[2], v[3]);
      }
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (int(d0) + e < fd.D) {
          const int sa = kt.ka[key], sb = kt.kb[key];
          const int i = sa * n + n1, j = sb * n + n2;
          float * Hl = Hs + l * LS;
          if (sa != sb) {
            Hl[j * SnP + i] = kSqrt2f * G[e];
            Hl[i * SnP + j] = kSqrt2f * G[e];
          } else {
            Hl[j * SnP + i] = (n1 == n2) ? 2.f * G[e] : G[e];
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
    const float s = Hl[j * SnP + i] + Hl[i * SnP + j];
    Hl[j * SnP + i] = s;
    Hl[i * SnP + j] = s;
  }
  __syncthreads();
  // dE/dc_{i l m} = lf_l sum_j H_l[i][j] c_{j l m}: each task is one pair of
  // rows (2ip, 2ip+1) and one 4-wide column group (l, q). H_l is read from
  // the transposed slots H_l[j][2ip..2ip+1] (consecutive lanes: consecutive
  // 8-byte words), c_j from the broadcast 16-byte chunk of the padded tile.
  float * out = dC + size_t(ci) * Sn * K;
  const int NP = (Sn + 1) >> 1;
  for (int t = threadIdx.x; t < kG * NP; t += blockDim.x) {
    const int g = t / NP;
    const int ip = t - g * NP;
    const int l = grp_l[g];
    const float * h = Hs + l * LS + 2 * ip;
    const float * cb = Cp + grp_off[g];
    float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
#pragma unroll 4
    for (int j = 0; j < Sn; ++j) {
      const float2 hv = *reinterpret_cast<const float2 *>(h + j * SnP);
      const float4 c = *reinterpret_cast<const float4 *>(cb + j * RS);
      a0.x += hv.x * c.x;
      a0.y += hv.x * c.y;
      a0.z += hv.x * c.z;
      a0.w += hv.x * c.w;
      a1.x += hv.y * c.x;
      a1.y += hv.y * c.y;
      a1.z += hv.y * c.z;
      a1.w += hv.y * c.w;
    }
    const int M = 2 * l + 1, m0 = grp_off[g] - offp_rt(l);
    const float lf = rsqrtf(float(M));
    const float v0[4] = {a0.x, a0.y, a0.z, a0.w}, v1[4] = {a1.x, a1.y, a1.z, a1.w};
    const int i = 2 * ip;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (m0 + e < M) {
        float * o = out + (l * l + m0 + e) * Sn + i;
        o[0] = v0[e] * lf;
        if (i + 1 < Sn) o[1] = v1[e] * lf;
      }
    }
  }
  }
}

template <int L>
size_t fwd_smem(const FeatureDims & fd) {
  return sizeof(float) * size_t(fd.S) * fd.n * row_stride(L);
}

BwdShape bwd_shape(const FeatureDims & fd) {
  BwdShape b;
  const uint32_t n = uint32_t(fd.n), Sn = uint32_t(fd.S) * n, npair = n * (n - 1) / 2;
  b.n = FastDiv(n);
  b.P = FastDiv(uint32_t(fd.P));
  b.npair = FastDiv(npair > 0 ? npair : 1u);
  b.Snp = FastDiv(npair > 0 ? uint32_t(fd.S) * npair : 1u);
  if (npair == 0) b.Snp.d = 0;  // no off-diagonal pairs: the symmetrisation loop is empty
  b.SnP = int(Sn + (Sn & 1u));
  // a multiple of 4 (16-byte rows) that is not a multiple of 32, so the
  // L+1 blocks start on different banks
  b.LS = int((Sn * uint32_t(b.SnP) + 3) / 4 * 4);
  if (b.LS % 32 == 0) b.LS += 4;
  b.vec = (n % 4 == 0) && (Sn % 4 == 0);
  return b;
}

template <int L>
size_t bwd_smem(const FeatureDims & fd, const BwdShape & b) {
  return sizeof(float) * (size_t(fd.S) * fd.n * row_stride(L) + size_t(L + 1) * b.LS);
}

// Blocks of a persistent kernel: as many as fit on the device at once (at
// most one per centre).
template <class Kern>
int persistent_grid(Kern k, int threads, size_t smem, int64_t n_centers) {
  int dev = 0, sms = 0, per_sm = 0;
  RGPU_CUDA(cudaGetDevice(&dev));
  RGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem));
  return int(std::max<int64_t>(1, std::min<int64_t>(n_centers, int64_t(sms) * std::max(per_sm, 1))));
}

}  // namespace

void launch_ps_fwd_fp32(const PsArgs & a, const float * C, float * X, __nv_bfloat16 * Xh,
                        __nv_bfloat16 * Xl, float * row_scale, cudaStream_t st) {
  if (a.n_centers == 0) return;
  if (!Xh || !Xl) throw Error(RGPU_ERR_INVALID_ARGUMENT, "FP32 power spectrum needs the BF16 outputs");
  const int threads = std::min(tile_config(a.fd.S, a.fd.n, a.fd.L).psf_threads, kThreads);
#define RGPU_PSF_CASE(LL)                                                                                     \
  case LL: {                                                                                                  \
    const size_t smem = fwd_smem<LL>(a.fd);                                                                   \
    RGPU_CUDA(cudaFuncSetAttribute(ps_fwd_f32_kernel<LL>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                   int(smem)));                                                               \
    ps_fwd_f32_kernel<LL><<<persistent_grid(ps_fwd_f32_kernel<LL>, threads, smem, a.n_centers), threads,     \
                            smem, st>>>(a, C, X, Xh, Xl, row_scale);                                          \
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

void launch_ps_fwd_fast(const PsArgs & a, const float * C, float * X, __nv_bfloat16 * Xh, __nv_bfloat16 * Xl,
                        float * row_scale, cudaStream_t st) {
  if (!X && tile_config(a.fd.S, a.fd.n, a.fd.L).psf_tc && ps_fwd_tc_supported(a.fd))
    launch_ps_fwd_tc(a, C, Xh, Xl, row_scale, st);
  else
    launch_ps_fwd_fp32(a, C, X, Xh, Xl, row_scale, st);
}

void launch_ps_bwd_fp32(const PsArgs & a, const float * C, const __nv_bfloat16 * Xh, const __nv_bfloat16 * Xl,
                        const float * row_scale, const float * dX, float * dC, cudaStream_t st) {
  if (a.n_centers == 0) return;
  if (a.fd.n > kMaxN) throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_radial above 16 is not supported on the fast path");
  const BwdShape bs = bwd_shape(a.fd);
  constexpr size_t kMaxSmem = 227 * 1024 - 2048;
  const int threads = std::min(tile_config(a.fd.S, a.fd.n, a.fd.L).psb_threads, kBwdThreads);
#define RGPU_PSB_CASE(LL)                                                                                     \
  case LL: {                                                                                                  \
    const size_t smem = bwd_smem<LL>(a.fd, bs);                                                               \
    if (smem > kMaxSmem)                                                                                      \
      throw Error(RGPU_ERR_INVALID_ARGUMENT,                                                                  \
                  "species x max_radial too large for the FP32 power-spectrum backward; use FP64");           \
    RGPU_CUDA(cudaFuncSetAttribute(ps_bwd_f32_kernel<LL>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                   int(smem)));                                                               \
    ps_bwd_f32_kernel<LL><<<persistent_grid(ps_bwd_f32_kernel<LL>, threads, smem, a.n_centers),               \
                            threads, smem, st>>>(a, bs, C, Xh, Xl, row_scale, dX, dC);                        \
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
