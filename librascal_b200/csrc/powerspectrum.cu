// SOAP power spectrum: forward, plain-path gradients, and the adjoint
// (backward) used by the fast force path.
//
// p_{(a<=b) n1 n2 l} = lf_l s_ab sum_m c_{a n1 lm} c_{b n2 lm},
//   lf_l = 1/sqrt(2l+1), s_ab = sqrt(2) for a < b else 1,
// x = p / |p|  (calculator_spherical_invariants.hh:747-794,
// property_block_sparse.hh:470-478). Gradients: :796-921 and the
// normalisation update :588-652. Dense layout per row: key (a<=b) major,
// then n1, n2, l (the reference's block layout (n1*n+n2, l), keys sorted).
#include <cuda_runtime.h>

#include "common.cuh"

namespace rgpu {
namespace {

constexpr int kThreads = 256;
constexpr double kSqrt2 = 1.41421356237309504880168872420969808;

struct KeyTables {
  int8_t ka[kMaxSpecies * (kMaxSpecies + 1) / 2];
  int8_t kb[kMaxSpecies * (kMaxSpecies + 1) / 2];
  int16_t kid[kMaxSpecies][kMaxSpecies];
};
__device__ __forceinline__ void build_keys(KeyTables & t, int S) {
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

template <typename T>
__device__ __forceinline__ T block_sum(T v, T * red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  T t = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : T(0);
  if (wid == 0) t = warp_sum(t);
  if (threadIdx.x == 0) red[0] = t;
  __syncthreads();
  T out = red[0];
  return out;
}

__device__ __forceinline__ void decode(int d, int n, int L1, int blk, int & k, int & n1, int & n2,
                                       int & l) {
  k = d / blk;
  int r = d - k * blk;
  n1 = r / (n * L1);
  r -= n1 * n * L1;
  n2 = r / L1;
  l = r - n2 * L1;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
ps_fwd_kernel(PsArgs a, const T * __restrict__ C, T * __restrict__ X, __nv_bfloat16 * __restrict__ Xh,
              __nv_bfloat16 * __restrict__ Xl, T * __restrict__ norm_out, bool inv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const FeatureDims fd = a.fd;
  T * Cs = reinterpret_cast<T *>(smem_raw);
  T * Ps = Cs + fd.S * fd.nK;
  __shared__ KeyTables kt;
  __shared__ T red[32];
  __shared__ T lfs[kMaxL + 1];
  build_keys(kt, fd.S);
  const int64_t ci = blockIdx.x;
  const T * Ci = C + size_t(ci) * fd.S * fd.nK;
  for (int e = threadIdx.x; e < fd.S * fd.nK; e += blockDim.x) Cs[e] = Ci[e];
  const int n = fd.n, S = fd.S, L1 = fd.L + 1, nn2 = n * n, blk = nn2 * L1;
  // 1/sqrt(2l+1) (calculator_spherical_invariants.hh:62-69)
  if (threadIdx.x < L1) lfs[threadIdx.x] = T(1.0 / sqrt(double(2 * threadIdx.x + 1)));
  __syncthreads();
  // task t = (l, n1, n2) with l slowest, so a warp shares l (uniform trip
  // counts; the c^a and c^b reads are a few broadcast addresses per warp)
  T ss = T(0);
  for (int t = threadIdx.x; t < blk; t += blockDim.x) {
    const int l = t / nn2;
    const int r = t - l * nn2;
    const int n1 = r / n, n2 = r - n1 * n;
    const int off = l * l, cnt = 2 * l + 1;
    const T lf = lfs[l];
    const int out = r * L1 + l;
    for (int sa = 0; sa < S; ++sa) {
      const T * c1 = Cs + sa * fd.nK + n1 * fd.K + off;
      for (int sb = sa; sb < S; ++sb) {
        const T * c2 = Cs + sb * fd.nK + n2 * fd.K + off;
        T s = T(0);
        for (int m = 0; m < cnt; ++m) s += c1[m] * c2[m];
        T v = s * lf;
        if (sa < sb) v *= T(kSqrt2);
        Ps[kt.kid[sa][sb] * blk + out] = v;
        ss += v * v;
      }
    }
  }
  ss = block_sum(ss, red);
  const T nrm = sqrt(ss);
  const size_t roff = size_t(a.row_of_center[ci]) * fd.Dpad;
  const bool do_norm = a.normalize && fabs(double(nrm)) > 0.;
  const T rinv = do_norm ? T(1) / nrm : T(1);
  // 8 consecutive outputs per thread: 16-byte BF16 stores
  for (int d0 = threadIdx.x * 8; d0 < fd.Dpad; d0 += blockDim.x * 8) {
    T v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int d = d0 + i;
      v[i] = d < fd.D ? Ps[d] : T(0);
      if (do_norm) v[i] = (sizeof(T) == 8) ? v[i] / nrm : v[i] * rinv;
    }
    if (X) {
#pragma unroll
      for (int i = 0; i < 8; ++i) X[roff + d0 + i] = v[i];
    }
    if (Xh) {  // BF16 hi/lo pair for the tensor-core GEMMs
      __align__(16) __nv_bfloat16 h[8], lo[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        h[i] = __float2bfloat16_rn(float(v[i]));
        lo[i] = __float2bfloat16_rn(float(v[i]) - __bfloat162float(h[i]));
      }
      *reinterpret_cast<uint4 *>(Xh + roff + d0) = *reinterpret_cast<uint4 *>(h);
      *reinterpret_cast<uint4 *>(Xl + roff + d0) = *reinterpret_cast<uint4 *>(lo);
    }
  }
  if (threadIdx.x == 0) {
    T nn = a.normalize ? nrm : T(1);
    norm_out[ci] = inv ? T(1) / nn : nn;
  }
}

// Plain path: d x / d r for every pair of centres [c0, c1); one block per
// pair, two passes (projection dot, then the normalised gradient).
__global__ void __launch_bounds__(kThreads)
ps_grad_kernel(PsArgs a, ExpansionArgs e, int64_t c0, int64_t p_base, int64_t p_first,
               const int64_t * __restrict__ pair_center, const double * __restrict__ C,
               const double * __restrict__ X, const double * __restrict__ inv_norm,
               const double * __restrict__ dCp, const double * __restrict__ dCs,
               double * __restrict__ dX) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const FeatureDims fd = a.fd;
  const int64_t p = p_first + blockIdx.x;
  const int64_t ci = pair_center[p - p_first];
  const bool self = (p == e.pair_off[ci]);
  double * Cs = reinterpret_cast<double *>(smem_raw);
  double * Gs = Cs + fd.S * fd.nK;  // gradient blocks [S][3][nK] (self) or [1][3][nK]
  __shared__ KeyTables kt;
  __shared__ double red[32];
  __shared__ double dots[3];
  build_keys(kt, fd.S);
  const int nK3 = 3 * fd.nK;
  for (int i = threadIdx.x; i < fd.S * fd.nK; i += blockDim.x) Cs[i] = C[size_t(ci) * fd.S * fd.nK + i];
  int gsp = -1;  // gradient species of a non-self pair
  if (self) {
    const double * src = dCs + size_t(ci - c0) * fd.S * nK3;
    for (int i = threadIdx.x; i < fd.S * nK3; i += blockDim.x) Gs[i] = src[i];
  } else {
    gsp = e.species_lut[e.types[e.pair_j[p]]];
    const double * src = dCp + size_t(p - p_base) * nK3;
    for (int i = threadIdx.x; i < nK3; i += blockDim.x) Gs[i] = src[i];
  }
  __syncthreads();
  const int L1 = fd.L + 1, blk = fd.n * fd.n * L1;
  const double invn = inv_norm[ci];
  const double * xr = X + size_t(a.row_of_center[ci]) * fd.Dpad;
  // gradient block of species s for component c, or null when zero
  auto gblk = [&](int s, int c) -> const double * {
    if (self) return Gs + size_t(s) * nK3 + c * fd.nK;
    return (s == gsp) ? Gs + c * fd.nK : nullptr;
  };
  auto grad_p = [&](int d, int c) -> double {
    int k, n1, n2, l;
    decode(d, fd.n, L1, blk, k, n1, n2, l);
    const int sa = kt.ka[k], sb = kt.kb[k];
    const double * ga = gblk(sa, c);
    const double * gb = gblk(sb, c);
    if (!ga && !gb) return 0.;
    const double lf = 1.0 / sqrt(double(2 * l + 1));
    double v = 0.;
    const int o = l * l;
    if (ga) {  // grad c^a_{n1} c^b_{n2}
      double s = 0.;
      const double * g1 = ga + n1 * fd.K + o;
      const double * c2 = Cs + sb * fd.nK + n2 * fd.K + o;
      for (int m = 0; m < 2 * l + 1; ++m) s += g1[m] * c2[m];
      v += s * lf;
    }
    if (gb) {  // c^a_{n1} grad c^b_{n2}
      double s = 0.;
      const double * g2 = gb + n2 * fd.K + o;
      const double * c1 = Cs + sa * fd.nK + n1 * fd.K + o;
      for (int m = 0; m < 2 * l + 1; ++m) s += g2[m] * c1[m];
      v += s * lf;
    }
    if (sa != sb) v *= kSqrt2;
    return v;
  };
  if (a.normalize) {
    for (int c = 0; c < 3; ++c) {
      double s = 0.;
      for (int d = threadIdx.x; d < fd.D; d += blockDim.x) s += (grad_p(d, c) * invn) * xr[d];
      s = block_sum(s, red);
      if (threadIdx.x == 0) dots[c] = s;
    }
    __syncthreads();
  }
  double * out = dX + size_t(p - p_base) * 3 * fd.D;
  for (int c = 0; c < 3; ++c) {
    const double dot = a.normalize ? dots[c] : 0.;
    for (int d = threadIdx.x; d < fd.D; d += blockDim.x) {
      double g = grad_p(d, c);
      if (a.normalize) {
        g *= invn;
        g -= dot * xr[d];
      }
      out[size_t(c) * fd.D + d] = g;
    }
  }
}

__global__ void pair_center_kernel(int64_t c0, int64_t c1, const int64_t * __restrict__ pair_off,
                                   int64_t p_first, int64_t * __restrict__ pc) {
  int64_t ci = c0 + int64_t(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (ci >= c1) return;
  for (int64_t p = pair_off[ci] + (threadIdx.x & 31); p < pair_off[ci + 1]; p += 32)
    pc[p - p_first] = ci;
}

}  // namespace

// FP64 kernels; compiled with --fmad=false (the FP32 path is in ps_fast.cu).
#ifndef RGPU_PART_FP32
void launch_ps_fwd_fp64(const PsArgs & a, const double * C, double * X, double * inv_norm,
                        cudaStream_t st) {
  if (a.n_centers == 0) return;
  size_t smem = sizeof(double) * (size_t(a.fd.S) * a.fd.nK + a.fd.D);
  RGPU_CUDA(cudaFuncSetAttribute(ps_fwd_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)));
  ps_fwd_kernel<double><<<int(a.n_centers), kThreads, smem, st>>>(a, C, X, nullptr, nullptr, inv_norm, true);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}
#endif

#ifndef RGPU_PART_FP32
void launch_ps_grad_fp64(const PsArgs & a, const ExpansionArgs & e, int64_t c0, int64_t c1,
                         int64_t p_base, const double * C, const double * X,
                         const double * inv_norm, const double * dCp, const double * dCs,
                         double * dX, cudaStream_t st) {
  if (c1 <= c0) return;
  int64_t p_first = 0, p_last = 0;
  RGPU_CUDA(cudaMemcpyAsync(&p_first, e.pair_off + c0, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RGPU_CUDA(cudaMemcpyAsync(&p_last, e.pair_off + c1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RGPU_CUDA(cudaStreamSynchronize(st));
  const int64_t np = p_last - p_first;
  if (np <= 0) return;
  // map each pair of the chunk back to its centre (stored just after dX)
  // per host thread and per device: another device's buffer is not memory this launch may use
  static thread_local PerDevice<DevBuf> pc_tab;
  DevBuf & pc = pc_tab.at(current_device());
  pc.ensure(sizeof(int64_t) * np);
  pair_center_kernel<<<div_up(c1 - c0, 8), 256, 0, st>>>(c0, c1, e.pair_off, p_first, pc.as<int64_t>());
  RGPU_LAUNCHED();
  size_t smem = sizeof(double) * (size_t(a.fd.S) * a.fd.nK + size_t(a.fd.S) * 3 * a.fd.nK);
  RGPU_CUDA(cudaFuncSetAttribute(ps_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  ps_grad_kernel<<<int(np), kThreads, smem, st>>>(a, e, c0, p_base, p_first, pc.as<int64_t>(), C, X,
                                                  inv_norm, dCp, dCs, dX);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}
#endif


}  // namespace rgpu
