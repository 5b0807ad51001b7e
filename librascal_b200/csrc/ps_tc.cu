// Power-spectrum forward on the 5th-generation tensor cores.
//
// p_(ab)(n1 n2 l) = lf s_ab sum_m c_(a n1 lm) c_(b n2 lm) (lf = (2l+1)^-1/2,
// s_ab = sqrt2 for a < b; calculator_spherical_invariants.hh:747-794) is,
// for each l, the Gram matrix C_l C_l^T of the centre's S n x (2l+1) block of
// coefficients. Centres are taken T = floor(128 / (S n)) at a time: their
// C_l blocks are stacked into one 128-row operand A_l (BF16 hi/lo split,
// K = 2l+1 padded to 16 per MMA step) and tcgen05 computes A_l A_l^T, a
// 128 x 128 FP32 accumulator in TMEM, as the 3-term product
// hi hi^T + hi lo^T + lo hi^T. Only the T diagonal (S n x S n) blocks are
// used: the other products pair rows of different centres.
//
// One CTA of 4 warps per tile of centres, persistent over tiles:
//   * all warps convert the tile's FP32 coefficient rows into the operand
//     layout (K-major, no swizzle: 8-row x 16-byte core matrices, the two
//     K halves of a 16-wide step 128 bytes apart, 8-row groups Kpad*16 bytes
//     apart);
//   * thread 0 issues the MMAs of l + 1 into one TMEM buffer while the
//     warps drain l from the other (two 128-column buffers);
//   * each warp reads its 32 rows (tcgen05.ld, 32 lanes x 4 columns at a
//     time), keeps the upper triangle J >= I of its own centre's block,
//     scales, splits into BF16 hi/lo and writes the centre's packed l-block
//     (the layout of rgpu_internal.h) into shared memory, from where the
//     block is copied to HBM with 16-byte stores;
//   * |p|^2 is summed per centre and 1/|p| stored per row, as the SIMT
//     forward does.
// Every mbarrier wait is bounded; a wait that gives up records it in the
// tensor-core status word, the CTA waits for the MMAs it issued and frees
// TMEM before it ends.
//
// Measured against the FP32-pipe forward (ps_fast.cu) on the molecule
// clusters (S n = 40): 9.1 against 1.95 ms, and 8.2 against 1.56 ms at the
// bulk shape (S n = 24), with forces within 3e-5 of it. The multiply-adds it
// moves to the tensor cores are a small part of the forward (about 25
// GFLOP per step, 0.35 ms at the FP32 rate); what remains per element (the
// conversion into the operand layout, the per-lane choice of the diagonal
// block, scaling, the BF16 split and the stores) runs on 8 warps per SM,
// since two 256-column TMEM buffers and 80 KB of shared memory allow two
// CTAs. The tile configuration keeps the FP32-pipe forward by default
// (psf_tc = 0); the autotuner measures both.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "tcgen05.cuh"

namespace rgpu {
using namespace tc;
TcStatus * tc_status_word();  // gemm_tc.cu: the current device's status word

namespace {

constexpr int kThreads = 128;
constexpr int kRows = 128;        // MMA M and N
constexpr int kTmemCols = 256;    // two 128-column accumulators
constexpr float kSqrt2 = 1.41421356237309504880f;
constexpr size_t kMinSmem = 80 * 1024;  // at most two CTAs (2 x 256 TMEM columns) per SM

__host__ __device__ constexpr int kpad16(int l) { return (2 * l + 1 + 15) / 16 * 16; }
// byte offset of the hi tile of l; the lo tile follows it
__host__ __device__ constexpr int op_off(int l) {
  int o = 0;
  for (int i = 0; i < l; ++i) o += 2 * kRows * kpad16(i) * 2;
  return o;
}
__device__ __forceinline__ int op_off_rt(int l) {
  int o = 0;
  for (int i = 0; i < l; ++i) o += 2 * kRows * kpad16(i) * 2;
  return o;
}
// element (r, k) of a K-major, no-swizzle operand with Kp columns
__device__ __forceinline__ int op_elem(int r, int k, int Kp) {
  return ((r >> 3) * (Kp * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2) >> 1;
}
__device__ __forceinline__ uint64_t desc_noswizzle(uint32_t addr, int Kp) {
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3FFF);
  d |= uint64_t(128 >> 4) << 16;             // leading byte offset: next 8 K elements
  d |= uint64_t((Kp * 16) >> 4) << 32;       // stride byte offset: next 8 rows
  d |= uint64_t(1) << 46;                    // descriptor version
  return d;                                  // layout type 0: no swizzle
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float * v) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

struct TcPsPlan {
  int T;         // centres per tile
  int ops;       // bytes of the operand tiles
  int stage;     // bytes of one staging buffer: T x 4 ntile x (hi, lo) BF16
  int ntile;     // 2 x 2 tiles of one l-block of a row
};

template <int L>
__global__ void __launch_bounds__(kThreads, 1)
ps_fwd_tc_kernel(PsArgs a, TcPsPlan plan, const float * __restrict__ C, __nv_bfloat16 * __restrict__ Xh,
                 __nv_bfloat16 * __restrict__ Xl, float * __restrict__ row_scale, TcStatus * status) {
  constexpr int RS = row_stride(L), OL = offp(L + 1);
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char * ops = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) &
                                                          ~uintptr_t(127));
  __nv_bfloat16 * stage0 = reinterpret_cast<__nv_bfloat16 *>(ops + plan.ops);
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ float nrm_s[kRows];
  const FeatureDims fd = a.fd;
  const int n = fd.n, S = fd.S, Sn = S * n, T = plan.T;
  const int blk = 4 * plan.ntile;  // one l-block of a row in staging (tiles in task order)
  // task table: row pair i, column pair j and the segment's tiles per l in
  // .x = i | j << 8 | T << 16, the tile's first column at l = L in .y
  int2 * tab = reinterpret_cast<int2 *>(ops + plan.ops + 2 * plan.stage);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  // the operand tiles start at zero: rows beyond T S n and columns beyond
  // 2l + 1 are never written again; so do the staging buffers, whose zero
  // entries (below the diagonal of the diagonal tiles, and the l-block
  // padding) no epilogue writes
  for (int e = threadIdx.x; e < (plan.ops + 2 * plan.stage) / 16; e += blockDim.x)
    reinterpret_cast<uint4 *>(ops)[e] = make_uint4(0u, 0u, 0u, 0u);
  for (int r = threadIdx.x; r < plan.ntile; r += blockDim.x) {
    int j = int((sqrtf(8.f * float(r) + 1.f) - 1.f) * 0.5f);
    while (j > 0 && j * (j + 1) / 2 > r) --j;
    while ((j + 1) * (j + 2) / 2 <= r) ++j;
    const int i = r - j * (j + 1) / 2;
    int base, lstep;
    tile_column(fd, i, j, base, lstep);
    tab[r] = make_int2(int(uint32_t(i) | (uint32_t(j) << 8) | (uint32_t(lstep / 4) << 16)), base);
  }
  const int padD = fd.lenD - 4 * (L + 1) * fd.TD, padO = fd.lenO - 4 * (L + 1) * fd.TO;
  const int nD = fd.G * padD, npad = nD + fd.G * (fd.G - 1) / 2 * padO;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(uint32_t(kTmemCols)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  constexpr uint32_t idesc = make_idesc(kRows, kRows);
  uint32_t uses[2] = {0u, 0u};     // commits of each buffer waited for (every thread)
  uint32_t commits[2] = {0u, 0u};  // commits issued to each buffer (thread 0)
  bool ok = true;

  const int64_t n_tiles = (a.n_centers + T - 1) / T;
  for (int64_t tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
    const int64_t c0 = tile * T;
    const int nt = int(std::min<int64_t>(T, a.n_centers - c0));
    // 1. coefficient rows of the tile -> BF16 hi/lo operands of every l
    for (int e = threadIdx.x; e < T * Sn * (OL / 4); e += blockDim.x) {
      const int r = e / (OL / 4), q = e - r * (OL / 4);
      const int t = r / Sn;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (t < nt) v = __ldg(reinterpret_cast<const float4 *>(C + (size_t(c0) * Sn + r) * RS) + q);
      const int col = 4 * q;
      int l = 0;
      while (col >= offp_rt(l + 1)) ++l;
      const int m0 = col - offp_rt(l), M = 2 * l + 1, Kp = kpad16(l);
      __nv_bfloat16 * hi = reinterpret_cast<__nv_bfloat16 *>(ops + op_off_rt(l));
      __nv_bfloat16 * lo = hi + kRows * Kp;
      const float x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (m0 + k < M) {
          const __nv_bfloat16 h = __float2bfloat16_rn(x[k]);
          const int idx = op_elem(r, m0 + k, Kp);
          hi[idx] = h;
          lo[idx] = __float2bfloat16_rn(x[k] - __bfloat162float(h));
        }
      }
    }
    if (threadIdx.x < kRows) nrm_s[threadIdx.x] = 0.f;
    fence_proxy_async_smem();  // the operands are read by the tensor cores
    __syncthreads();
    auto issue = [&](int l) {
      const int b = l & 1, Kp = kpad16(l);
      const uint32_t hi = smem_u32(ops + op_off_rt(l));
      const uint32_t lo = hi + uint32_t(kRows * Kp * 2);
      const uint32_t d = tmem + uint32_t(b * kRows);
      tc_fence_after();
      for (int s = 0; s < Kp / 16; ++s) {
        const uint32_t o = uint32_t(s) * 256u;  // 16 K elements = two core matrices
        mma_bf16(d, desc_noswizzle(hi + o, Kp), desc_noswizzle(hi + o, Kp), idesc, s > 0 ? 1u : 0u);
        mma_bf16(d, desc_noswizzle(hi + o, Kp), desc_noswizzle(lo + o, Kp), idesc, 1u);
        mma_bf16(d, desc_noswizzle(lo + o, Kp), desc_noswizzle(hi + o, Kp), idesc, 1u);
      }
      mma_commit(&bar[b]);
      ++commits[b];
    };
    if (threadIdx.x == 0) issue(0);
    // per-thread row: centre t, row my_i = a n + n1 of its Gram block (species a)
    const int r = warp * 32 + lane;
    const int my_t = r / Sn, my_i = r - my_t * Sn;
    const int my_a = my_i / n;
    const bool row_ok = my_t < nt;
    const int t_lo = (warp * 32) / Sn, t_hi = std::min((warp * 32 + 31) / Sn, nt - 1);
    float nrm = 0.f;
    for (int l = 0; l <= L; ++l) {
      const int b = l & 1;
      if (threadIdx.x == 0 && l + 1 <= L) issue(l + 1);
      const bool w = mbar_wait(&bar[b], uses[b] & 1u, status, 21);
      ok = __syncthreads_and(w) != 0;
      ++uses[b];
      if (!ok) break;
      tc_fence_after();
      __nv_bfloat16 * sh = stage0 + size_t(b) * (plan.stage / 2);  // staging buffer of this l
      __nv_bfloat16 * sl = sh + size_t(T) * blk;
      const float lf = rsqrtf(float(2 * l + 1));
      const uint32_t tq = tmem + (uint32_t(warp * 32) << 16) + uint32_t(b * kRows);
      for (int tt = t_lo; tt <= t_hi; ++tt) {
        for (int sb = 0; sb < S; ++sb) {
          for (int q = 0; q < n / 4; ++q) {
            float v[4];
            tmem_ld4(tq + uint32_t(tt * Sn + sb * n + 4 * q), v);
            if (row_ok && tt == my_t && sb >= my_a) {
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const int J = sb * n + 4 * q + e;  // column of the centre's Gram block
                if (J < my_i) continue;
                const float x = v[e] * (J > my_i ? lf * kSqrt2 : lf);
                const int jp = J >> 1;  // packed position of (I, J), 2 x 2 tiles
                const int idx = my_t * blk + 4 * (jp * (jp + 1) / 2 + (my_i >> 1)) + (my_i & 1) + 2 * (J & 1);
                const __nv_bfloat16 h = __float2bfloat16_rn(x);
                sh[idx] = h;
                sl[idx] = __float2bfloat16_rn(x - __bfloat162float(h));
                nrm += x * x;
              }
            }
          }
        }
      }
      tc_fence_before();
      __syncthreads();
      // each staged tile (8 bytes of hi, 8 of lo) to its column of the packed row
      for (int e = threadIdx.x; e < 2 * nt * plan.ntile; e += blockDim.x) {
        const int half = e / (nt * plan.ntile), rem = e - half * (nt * plan.ntile);
        const int t = rem / plan.ntile, r = rem - t * plan.ntile;
        const int64_t row = a.row_of_center[c0 + t];
        const int2 te = tab[r];
        const int col = te.y + 4 * (L - l) * int(uint32_t(te.x) >> 16);
        const uint2 * src = reinterpret_cast<const uint2 *>((half ? sl : sh) + t * blk + 4 * r);
        *reinterpret_cast<uint2 *>((half ? Xl : Xh) + size_t(row) * fd.Dg + col) = *src;
      }
    }
    if (!ok) break;
    if (row_ok) atomicAdd(&nrm_s[my_t], nrm);
    __syncthreads();
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
      const int64_t row = a.row_of_center[c0 + t];
      const float nv = sqrtf(nrm_s[t]);
      row_scale[row] = (a.normalize && nv > 0.f) ? 1.f / nv : 1.f;
    }
    // the end of every segment after its tiles, in every row of the tile
    for (int e = threadIdx.x; e < nt * npad; e += blockDim.x) {
      const int t = e / npad, p = e - t * npad;
      int d;
      if (p < nD) {
        const int A = p / padD;
        d = segment_offset(fd, A, A) + 4 * (L + 1) * fd.TD + (p - A * padD);
      } else {
        int k = (p - nD) / padO, A = 0;
        const int r = (p - nD) - k * padO;
        while (k >= fd.G - 1 - A) {
          k -= fd.G - 1 - A;
          ++A;
        }
        d = segment_offset(fd, A, A + 1 + k) + 4 * (L + 1) * fd.TO + r;
      }
      const int64_t row = a.row_of_center[c0 + t];
      Xh[size_t(row) * fd.Dg + d] = __float2bfloat16_rn(0.f);
      Xl[size_t(row) * fd.Dg + d] = __float2bfloat16_rn(0.f);
    }
    __syncthreads();  // nrm_s and the operands are rewritten by the next tile
  }
  // every MMA issued has finished before TMEM is released: the phase of
  // each buffer's last commit completes after all earlier ones
  if (threadIdx.x == 0)
    for (int b = 0; b < 2; ++b)
      if (commits[b] > 0) mbar_drain(&bar[b], (commits[b] - 1u) & 1u, status, 26);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(kTmemCols)));
  }
}

}  // namespace

// Whether the tensor-core forward serves this shape: S n <= 128 rows per
// centre, n a multiple of 4 (the 4-column TMEM reads and 16-byte block
// copies), and the shared memory fits.
bool ps_fwd_tc_supported(const FeatureDims & fd) {
  const int Sn = fd.S * fd.n;
  if (Sn > kRows || fd.n % 4 != 0 || fd.L > kMaxL) return false;
  const int T = kRows / Sn;
  const size_t ops = size_t(op_off(fd.L + 1));
  const size_t ntile = size_t(Sn / 2) * (Sn / 2 + 1) / 2;
  const size_t stage = 2 * size_t(T) * 4 * ntile * 2 * sizeof(__nv_bfloat16);
  return ops + stage + sizeof(int2) * ntile + 256 <= size_t(227 * 1024 - 4096);
}

void launch_ps_fwd_tc(const PsArgs & a, const float * C, __nv_bfloat16 * Xh, __nv_bfloat16 * Xl, float * row_scale,
                      cudaStream_t st) {
  if (a.n_centers == 0) return;
  if (!ps_fwd_tc_supported(a.fd)) throw Error(RGPU_ERR_INVALID_ARGUMENT, "shape not served by the tensor-core forward");
  TcPsPlan plan;
  plan.T = kRows / (a.fd.S * a.fd.n);
  plan.ops = op_off(a.fd.L + 1);
  plan.ntile = (a.fd.Sn / 2) * (a.fd.Sn / 2 + 1) / 2;
  plan.stage = 2 * plan.T * 4 * plan.ntile * int(sizeof(__nv_bfloat16));  // hi + lo of one l
  const size_t smem =
      std::max(kMinSmem, size_t(plan.ops) + 2 * size_t(plan.stage) + sizeof(int2) * plan.ntile + 256);
  int dev = 0, sms = 0;
  RGPU_CUDA(cudaGetDevice(&dev));
  RGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t tiles = (a.n_centers + plan.T - 1) / plan.T;
  const int grid = int(std::min<int64_t>(tiles, int64_t(sms) * 2));
  TcStatus * status = tc_status_word();
#define RGPU_PSTC_CASE(LL)                                                                                      \
  case LL:                                                                                                      \
    RGPU_CUDA(cudaFuncSetAttribute(ps_fwd_tc_kernel<LL>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))); \
    ps_fwd_tc_kernel<LL><<<grid, kThreads, smem, st>>>(a, plan, C, Xh, Xl, row_scale, status);                  \
    break;
  switch (a.fd.L) {
    RGPU_PSTC_CASE(0)
    RGPU_PSTC_CASE(1)
    RGPU_PSTC_CASE(2)
    RGPU_PSTC_CASE(3)
    RGPU_PSTC_CASE(4)
    RGPU_PSTC_CASE(5)
    RGPU_PSTC_CASE(6)
    RGPU_PSTC_CASE(7)
    RGPU_PSTC_CASE(8)
    RGPU_PSTC_CASE(9)
    RGPU_PSTC_CASE(10)
    RGPU_PSTC_CASE(11)
    RGPU_PSTC_CASE(12)
    default:
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_angular above 12 is not supported on the GPU");
  }
#undef RGPU_PSTC_CASE
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

}  // namespace rgpu
