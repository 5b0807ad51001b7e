// tcgen05 (5th-generation tensor core) GEMM for the GAP contractions.
//
//   C[M x N] = A[M x K] B[N x K]^T, A and B K-major (row-major, K fastest),
//   computed as a 3-term BF16 split product with FP32 accumulation in TMEM:
//     A B^T ~= A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T,
//   A_hi = bf16(A), A_lo = bf16(A - A_hi) (same for B), which keeps ~16
//   mantissa bits per product: enough for the 1e-4 force bar that a single
//   TF32 or BF16 pass misses.
//
// One CTA computes one 128 x BN output tile:
//   warp 0   TMA producer: per K block, 4 tiles (A_hi, A_lo, B_hi, B_lo)
//            into a STAGES-deep ring of 128B-swizzled shared buffers;
//   warp 1   MMA issuer: 3 tcgen05.mma (kind::f16, BF16 in, FP32 out) per
//            16-wide K step into a 128 x BN FP32 accumulator in TMEM;
//   warps 2-5 epilogue: tcgen05.ld of their 32-lane TMEM quadrant, then
//            either a plain FP32 store or the fused GAP forward epilogue
//            (k^zeta, per-row energy partial, W = alpha zeta k^(zeta-1)
//            written as a BF16 hi/lo pair for the backward GEMM).
// Every mbarrier wait is bounded; a wait that gives up records an error in
// a device status word and the kernel winds down (TMEM is always freed).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "tcgen05.cuh"

namespace rgpu {
using namespace tc;
namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;  // bf16 elements per K block = 128 bytes (one swizzle row)
constexpr int kThreads = 192;
struct TcArgs {
  int64_t M, N, K;
  int epilogue;        // 0 store FP32 C; 1 GAP forward
  float * C;           // FP32 output (epilogue 0), row stride ldc
  int64_t ldc;
  __nv_bfloat16 * W_hi;  // epilogue 1 outputs, row stride ldw (zero beyond N);
  __nv_bfloat16 * W_lo;  // W_hi == nullptr: energy partials only
  int64_t ldw;
  const float * alpha;  // [N]
  int zeta;
  float * e_part;       // [gridDim.x][M]
  const float * row_scale;  // epilogue 1: k = row_scale[row] * (A B^T) (null: 1)
  TcStatus * status;
  long long mma_wait_limit;  // polls of the MMA warp's operand waits
};

template <int BN, int STAGES, int BK = kBK>
struct Smem {
  static constexpr int A_BYTES = kBM * BK * 2;  // 16 KB at BK = 64
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int TOTAL = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
  // the grouped kernel adds the FP32 epilogue's staging: per epilogue warp
  // two 32 x 32 boxes of 4 KB (128-byte swizzle, 1024-byte aligned)
  static constexpr int STAGING = 4 * 2 * 4096;
  static constexpr int TOTAL_GROUPED = TOTAL + STAGING;
};

__device__ __forceinline__ float powz(float v, int z) {
  float r = 1.f;
  for (int i = 0; i < z; ++i) r *= v;
  return r;
}

template <int BN, int STAGES>
__global__ void __launch_bounds__(kThreads, 1)
gemm_tc_kernel(const __grid_constant__ CUtensorMap mA_hi, const __grid_constant__ CUtensorMap mA_lo,
               const __grid_constant__ CUtensorMap mB_hi, const __grid_constant__ CUtensorMap mB_lo, TcArgs g) {
  using SM = Smem<BN, STAGES>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte alignment for the 128B-swizzle atoms
  unsigned char * base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t * full = reinterpret_cast<uint64_t *>(base + STAGES * SM::STAGE_BYTES);
  uint64_t * empty = full + STAGES;
  uint64_t * accum = empty + STAGES;
  uint32_t * tmem_slot = reinterpret_cast<uint32_t *>(accum + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n0 = int64_t(blockIdx.x) * BN, m0 = int64_t(blockIdx.y) * kBM;
  const int nk = int((g.K + kBK - 1) / kBK);

  if (warp == 0 && lane == 0) {
    prefetch_map(&mA_hi);
    prefetch_map(&mA_lo);
    prefetch_map(&mB_hi);
    prefetch_map(&mB_lo);
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    fence_barrier_init();
  }
  if (warp == 1) {  // TMEM accumulator: BN FP32 columns x 128 lanes
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(uint32_t(BN)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int issued = 0;
      for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % STAGES;
        const uint32_t ph = uint32_t(kb / STAGES) & 1u;
        if (!mbar_wait(&empty[s], ph ^ 1u, g.status, 1)) break;
        unsigned char * st = base + s * SM::STAGE_BYTES;
        mbar_expect_tx(&full[s], SM::STAGE_BYTES);
        const int kx = kb * kBK;
        tma_load_2d(st, &mA_hi, &full[s], kx, int(m0));
        tma_load_2d(st + SM::A_BYTES, &mA_lo, &full[s], kx, int(m0));
        tma_load_2d(st + 2 * SM::A_BYTES, &mB_hi, &full[s], kx, int(n0));
        tma_load_2d(st + 2 * SM::A_BYTES + SM::B_BYTES, &mB_lo, &full[s], kx, int(n0));
        ++issued;
      }
      // drain: the last copies must have landed before the CTA releases its
      // shared memory (they normally have; this matters after a timeout)
      for (int kb = issued > STAGES ? issued - STAGES : 0; kb < issued; ++kb)
        mbar_drain(&full[kb % STAGES], uint32_t(kb / STAGES) & 1u, g.status, 4);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = make_idesc(kBM, BN);
      bool ok = true;
      for (int kb = 0; kb < nk && ok; ++kb) {
        const int s = kb % STAGES;
        const uint32_t ph = uint32_t(kb / STAGES) & 1u;
        if (!mbar_wait(&full[s], ph, g.status, 2, g.mma_wait_limit)) {
          ok = false;
          break;
        }
        tc_fence_after();
        unsigned char * st = base + s * SM::STAGE_BYTES;
        const uint32_t a_hi = smem_u32(st), a_lo = smem_u32(st + SM::A_BYTES);
        const uint32_t b_hi = smem_u32(st + 2 * SM::A_BYTES), b_lo = smem_u32(st + 2 * SM::A_BYTES + SM::B_BYTES);
#pragma unroll
        for (int k = 0; k < kBK / 16; ++k) {
          const uint32_t off = uint32_t(k) * 32u;  // 16 bf16 = 32 bytes along the swizzled row
          const uint32_t acc0 = (kb > 0 || k > 0) ? 1u : 0u;
          mma_bf16(tmem, smem_desc(a_lo + off), smem_desc(b_hi + off), idesc, acc0);
          mma_bf16(tmem, smem_desc(a_hi + off), smem_desc(b_lo + off), idesc, 1u);
          mma_bf16(tmem, smem_desc(a_hi + off), smem_desc(b_hi + off), idesc, 1u);
        }
        mma_commit(&empty[s]);  // frees the stage once these MMAs have read it
      }
      mma_commit(accum);  // accumulator complete (also fires if no MMA was issued)
    }
  } else {
    // epilogue warps 2..5: TMEM lane quadrant = warp % 4
    const int q = warp & 3;
    const int64_t row = m0 + q * 32 + lane;
    const bool ok = __all_sync(0xffffffffu, mbar_wait(accum, 0u, g.status, 3));
    tc_fence_after();
    float e_acc = 0.f;
    if (ok) {
      for (int c0 = 0; c0 < BN; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(c0), v);
        const int64_t col = n0 + c0;
        if (row >= g.M) continue;
        if (g.epilogue == 0) {
          float * out = g.C + row * g.ldc + col;
          if (col + 16 <= g.N) {
#pragma unroll
            for (int i = 0; i < 16; i += 4)
              *reinterpret_cast<float4 *>(out + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
          } else {
            for (int i = 0; i < 16; ++i)
              if (col + i < g.N) out[i] = v[i];
          }
        } else {
          // W_hi == nullptr: energies only, no W output
          if (g.W_hi && col >= g.ldw) continue;
          if (g.row_scale) {
            const float rs = __ldg(g.row_scale + row);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] *= rs;
          }
          __align__(16) __nv_bfloat16 hi[16], lo[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const float al = (col + i < g.N) ? __ldg(g.alpha + col + i) : 0.f;
            e_acc += al * powz(v[i], g.zeta);
            const float w = al * (float(g.zeta) * powz(v[i], g.zeta - 1));
            hi[i] = __float2bfloat16_rn(w);
            lo[i] = __float2bfloat16_rn(w - __bfloat162float(hi[i]));
          }
          if (!g.W_hi) continue;
          uint4 * dh = reinterpret_cast<uint4 *>(g.W_hi + row * g.ldw + col);
          uint4 * dl = reinterpret_cast<uint4 *>(g.W_lo + row * g.ldw + col);
          dh[0] = reinterpret_cast<uint4 *>(hi)[0];
          dh[1] = reinterpret_cast<uint4 *>(hi)[1];
          dl[0] = reinterpret_cast<uint4 *>(lo)[0];
          dl[1] = reinterpret_cast<uint4 *>(lo)[1];
        }
      }
    }
    if (g.epilogue == 1 && row < g.M) g.e_part[int64_t(blockIdx.x) * g.M + row] = e_acc;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    // every MMA issued has finished before TMEM is released (the epilogue
    // waited for this already unless a wait of the launch gave up)
    if (lane == 0) mbar_drain(accum, 0u, g.status, 6);
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(BN)));
  }
}


// ------------------------------------------------------- grouped, persistent
// All species' GEMMs of one direction in one launch: one CTA per SM walks a
// tile list (group, m tile, n tile; n fastest, so CTAs running at the same
// time share A rows in L2). The 128 x BN accumulator is double-buffered in
// TMEM (2 x BN of the 512 columns): the MMA warp fills one buffer while the
// epilogue warps drain the other, and the smem ring runs across tiles.
constexpr int kMaxGroups = 16;

struct TcGroup {
  int64_t M, N, K;
  float * C;
  int64_t ldc;
  __nv_bfloat16 * W_hi;
  __nv_bfloat16 * W_lo;
  int64_t ldw;
  const float * alpha;
  float * e_part;           // [n_tiles][M]
  const float * row_scale;  // may be null
  int64_t tile0;            // first tile of this group in the launch
  int64_t n_tiles;          // tiles along N
  const uint32_t * tile_mask;  // per M-tile: species present in any of its rows (null: all)
};

// Species segments of the packed feature columns (rgpu_internal.h): G groups,
// segment (A, B), A <= B in A-major order, LD (A = B) or LO (A < B) units of
// 32 columns long. A unit is needed by an M-tile when both of its segment's
// groups are in the tile's mask; the other units hold zeros in every row of
// the tile (forward: skipped K blocks add nothing) or are never read for
// them (backward: skipped N tiles are columns of species the rows lack).
struct SegGeom {
  int mode;  // 0: no skipping; 1: K (forward); 2: N (backward)
  int G, LD, LO;
};
struct SegWalk {
  SegGeom sg;
  uint32_t mask;
  int A, B, end;
  bool on;
  __device__ __forceinline__ void start(const SegGeom & g, uint32_t m) {
    sg = g;
    mask = m ? m : 0xFFFFFFFFu;  // a tile always holds its rows' own species
    A = 0;
    B = 0;
    end = g.LD;
    on = mask & 1u;
  }
  // whether unit u is needed; u must not decrease between calls
  __device__ __forceinline__ bool need(int u) {
    while (u >= end && A < sg.G) {
      if (B + 1 < sg.G) {
        ++B;
        end += sg.LO;
      } else {
        ++A;
        B = A;
        end += sg.LD;
      }
      on = ((mask >> A) & 1u) && ((mask >> B) & 1u);
    }
    return A >= sg.G || on;
  }
  // whether any unit of [u0, u0 + n) is needed
  __device__ __forceinline__ bool any(int u0, int n) {
    bool r = false;
    for (int u = u0; u < u0 + n; ++u) r |= need(u);
    return r;
  }
};

struct TcGroupedArgs {
  CUtensorMap a_hi[kMaxGroups], a_lo[kMaxGroups], b_hi[kMaxGroups], b_lo[kMaxGroups];
  CUtensorMap c_map[kMaxGroups];  // FP32 output (epilogue 0): 32 x 32 boxes, 128-byte swizzle
  TcGroup grp[kMaxGroups];
  int n_groups;
  int epilogue;
  int zeta;
  int64_t n_tiles;
  TcStatus * status;
  long long mma_wait_limit;  // polls of the MMA warp's operand waits
  SegGeom seg;
};

// The 32-column units of tile (mt, nt) that are computed: [u0, u0 + nu).
// The tile's BN / 32 units are cut after the last one holding a column the
// epilogue writes (< N; < ldw for the GAP forward, whose W rows are zero up
// to ldw), and under N-mode skipping to the run from its first to its last
// needed unit; nu = 0 drops the tile. The MMA then runs N = 32 nu wide on
// B rows loaded from the span's first column. Every role asks, so all agree.
struct TileSpan {
  int u0, nu;
};
template <int BN>
__device__ __forceinline__ TileSpan tile_span(const TcGroupedArgs & p, const TcGroup & G, int64_t mt, int64_t nt) {
  const int64_t ext = (p.epilogue == 1 && G.ldw > G.N) ? G.ldw : G.N;
  const int64_t ue = (ext + 31) / 32;
  int u0 = int(nt) * (BN / 32);
  int u1 = int(ue < u0 + BN / 32 ? ue : int64_t(u0 + BN / 32));
  if (p.seg.mode == 2 && G.tile_mask) {
    SegWalk w;
    w.start(p.seg, G.tile_mask[mt]);
    int first = u1, last = u0 - 1;
    for (int u = u0; u < u1; ++u)
      if (w.need(u)) {
        first = min(first, u);
        last = u;
      }
    if (last < first) return {u0, 0};
    u0 = first;
    u1 = last + 1;
  }
  return {u0, u1 - u0};
}

__device__ __forceinline__ int find_group(const TcGroupedArgs & p, int64_t t) {
  int g = 0;
  while (g + 1 < p.n_groups && t >= p.grp[g + 1].tile0) ++g;
  return g;
}

template <int BN, int STAGES, int BK>
__global__ void __launch_bounds__(kThreads, 1) gemm_tc_grouped_kernel(const __grid_constant__ TcGroupedArgs p) {
  using SM = Smem<BN, STAGES, BK>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char * base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  float * staging = reinterpret_cast<float *>(base + STAGES * SM::STAGE_BYTES);  // [4 warps][2][32][32]
  uint64_t * full = reinterpret_cast<uint64_t *>(base + STAGES * SM::STAGE_BYTES + SM::STAGING);
  uint64_t * empty = full + STAGES;
  uint64_t * tfull = empty + STAGES;  // [2] accumulator buffer written
  uint64_t * tempty = tfull + 2;      // [2] accumulator buffer read out
  uint64_t * done = tempty + 2;       // every MMA of this CTA finished
  uint32_t * tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  TcStatus * status = p.status;

  if (warp == 0 && lane == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
    }
    mbar_init(done, 1);
    fence_barrier_init();
  }
  if (warp == 1) {  // two accumulators: 2 BN FP32 columns x 128 lanes
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(uint32_t(2 * BN)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;  // K blocks issued by this CTA
      bool ok = true;
      for (int64_t t = blockIdx.x; t < p.n_tiles && ok; t += gridDim.x) {
        const int g = find_group(p, t);
        const TcGroup & G = p.grp[g];
        const int64_t local = t - G.tile0, mt = local / G.n_tiles, nt = local - mt * G.n_tiles;
        const TileSpan sp = tile_span<BN>(p, G, mt, nt);
        if (sp.nu == 0) continue;
        const int m0 = int(mt * kBM), n0 = 32 * sp.u0;
        const int nk = int((G.K + BK - 1) / BK);
        const bool kskip = p.seg.mode == 1 && G.tile_mask;
        SegWalk w;
        if (kskip) w.start(p.seg, G.tile_mask[mt]);
        for (int kb = 0; kb < nk; ++kb) {
          if (kskip && !w.any(kb * (BK / 32), BK / 32)) continue;
          const int s = int(it % STAGES);
          const uint32_t ph = (it / STAGES) & 1u;
          if (!mbar_wait(&empty[s], ph ^ 1u, status, 1)) {
            ok = false;
            break;
          }
          unsigned char * st = base + s * SM::STAGE_BYTES;
          mbar_expect_tx(&full[s], SM::STAGE_BYTES);
          const int kx = kb * BK;
          tma_load_2d(st, &p.a_hi[g], &full[s], kx, m0);
          tma_load_2d(st + SM::A_BYTES, &p.a_lo[g], &full[s], kx, m0);
          // B as one box of BN rows from the span's first column (rows past
          // the span or past N are loaded or zero-filled but not multiplied)
          tma_load_2d(st + 2 * SM::A_BYTES, &p.b_hi[g], &full[s], kx, n0);
          tma_load_2d(st + 2 * SM::A_BYTES + SM::B_BYTES, &p.b_lo[g], &full[s], kx, n0);
          ++it;
        }
      }
      // the last copies must have landed before the CTA releases its shared
      // memory (they normally have; this matters after a timeout)
      for (uint32_t k = it > uint32_t(STAGES) ? it - STAGES : 0u; k < it; ++k)
        mbar_drain(&full[k % STAGES], (k / STAGES) & 1u, status, 4);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t it = 0;
      int i = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < p.n_tiles && ok; t += gridDim.x) {
        const int g = find_group(p, t);
        const TcGroup & G = p.grp[g];
        const int64_t local = t - G.tile0, mt = local / G.n_tiles, nt = local - mt * G.n_tiles;
        const TileSpan sp = tile_span<BN>(p, G, mt, nt);
        if (sp.nu == 0) continue;
        const uint32_t idesc = make_idesc(kBM, 32 * sp.nu);
        const int nk = int((G.K + BK - 1) / BK);
        const int b = i & 1;
        const uint32_t use = uint32_t(i >> 1);
        if (!mbar_wait(&tempty[b], (use & 1u) ^ 1u, status, 5)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + uint32_t(b * BN);
        const bool kskip = p.seg.mode == 1 && G.tile_mask;
        SegWalk w;
        if (kskip) w.start(p.seg, G.tile_mask[mt]);
        bool first = true;  // the tile's first MMA overwrites the accumulator
        for (int kb = 0; kb < nk; ++kb) {
          if (kskip && !w.any(kb * (BK / 32), BK / 32)) continue;
          const int s = int(it % STAGES);
          const uint32_t ph = (it / STAGES) & 1u;
          if (!mbar_wait(&full[s], ph, status, 2, p.mma_wait_limit)) {
            ok = false;
            break;
          }
          tc_fence_after();
          unsigned char * st = base + s * SM::STAGE_BYTES;
          const uint32_t a_hi = smem_u32(st), a_lo = smem_u32(st + SM::A_BYTES);
          const uint32_t b_hi = smem_u32(st + 2 * SM::A_BYTES), b_lo = smem_u32(st + 2 * SM::A_BYTES + SM::B_BYTES);
#pragma unroll
          for (int k = 0; k < BK / 16; ++k) {
            const uint32_t off = uint32_t(k) * 32u;
            const uint32_t acc0 = (first && k == 0) ? 0u : 1u;
            mma_bf16(acc, smem_desc_k<BK>(a_lo + off), smem_desc_k<BK>(b_hi + off), idesc, acc0);
            mma_bf16(acc, smem_desc_k<BK>(a_hi + off), smem_desc_k<BK>(b_lo + off), idesc, 1u);
            mma_bf16(acc, smem_desc_k<BK>(a_hi + off), smem_desc_k<BK>(b_hi + off), idesc, 1u);
          }
          mma_commit(&empty[s]);
          ++it;
          first = false;
        }
        mma_commit(&tfull[b]);  // also after a failed wait, so the epilogue moves on
        ++i;
      }
      mma_commit(done);  // completes when every MMA issued above has finished
      mbar_drain(done, 0u, status, 6);
    }
  } else {
    const int q = warp & 3;  // TMEM lane quadrant of this warp
    float * stg = staging + q * 2048;  // this warp's two 32 x 32 boxes
    int sb = 0;                        // box to fill next
    int i = 0;
    for (int64_t t = blockIdx.x; t < p.n_tiles; t += gridDim.x) {
      const int g = find_group(p, t);
      const TcGroup & G = p.grp[g];
      const int64_t local = t - G.tile0, mt = local / G.n_tiles, nt = local - mt * G.n_tiles;
      const TileSpan sp = tile_span<BN>(p, G, mt, nt);
      if (sp.nu == 0) continue;
      const int64_t m0 = mt * kBM, n0 = 32 * int64_t(sp.u0);
      const int b = i & 1;
      const uint32_t use = uint32_t(i >> 1);
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&tfull[b], use & 1u, status, 3));
      if (!ok) break;
      tc_fence_after();
      const int64_t row = m0 + q * 32 + lane;
      const float rs = (p.epilogue == 1 && G.row_scale && row < G.M) ? __ldg(G.row_scale + row) : 1.f;
      float e_acc = 0.f;
      const float zf = float(p.zeta);
      const int zm1 = p.zeta - 1;
      for (int c0 = 0; c0 < 32 * sp.nu; c0 += 32) {
        float v[32];
        tmem_ld32(tmem + (uint32_t(q * 32) << 16) + uint32_t(b * BN + c0), v);
        const int64_t col = n0 + c0;
        if (p.epilogue == 0) {
          // the warp's 32 rows x 32 columns through shared memory to a TMA
          // store, which clips rows >= M and columns >= N
          if (col >= G.N) continue;  // uniform over the warp
          if (lane == 0) bulk_wait_read<1>();  // the store that read this box last is done with it
          __syncwarp();
          float * box = stg + sb * 1024;
#pragma unroll
          for (int c = 0; c < 8; ++c)  // 16-byte chunk c of row `lane` at chunk c ^ (lane % 8): 128-byte swizzle
            *reinterpret_cast<float4 *>(box + lane * 32 + 4 * (c ^ (lane & 7))) =
                make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
          fence_async_smem();
          __syncwarp();
          if (lane == 0) {
            tma_store_2d(&p.c_map[g], box, int(col), int(m0 + q * 32));
            bulk_commit();
          }
          sb ^= 1;
        } else {
          if (col >= G.ldw) continue;  // uniform over the warp: ldw is a multiple of 32
          // lane j holds alpha of column col + j; every lane takes them all by shuffles
          const float my_al = (col + lane < G.N) ? __ldg(G.alpha + col + lane) : 0.f;
          uint32_t hw[16], lw[16];
#pragma unroll
          for (int k = 0; k < 32; k += 2) {
            const float a0 = __shfl_sync(0xffffffffu, my_al, k), a1 = __shfl_sync(0xffffffffu, my_al, k + 1);
            const float x0 = v[k] * rs, x1 = v[k + 1] * rs;
            float p0 = x0, p1 = x1;  // x^(zeta-1)
            if (zm1 != 1) {
              p0 = 1.f;
              p1 = 1.f;
              for (int z = 0; z < zm1; ++z) {
                p0 *= x0;
                p1 *= x1;
              }
            }
            e_acc += a0 * (p0 * x0) + a1 * (p1 * x1);
            const float w0 = a0 * zf * p0, w1 = a1 * zf * p1;
            const __nv_bfloat162 h = __floats2bfloat162_rn(w0, w1);
            const float2 hf = __bfloat1622float2(h);
            const __nv_bfloat162 l = __floats2bfloat162_rn(w0 - hf.x, w1 - hf.y);
            hw[k / 2] = *reinterpret_cast<const uint32_t *>(&h);
            lw[k / 2] = *reinterpret_cast<const uint32_t *>(&l);
          }
          if (row >= G.M) continue;
          uint4 * dh = reinterpret_cast<uint4 *>(G.W_hi + row * G.ldw + col);
          uint4 * dl = reinterpret_cast<uint4 *>(G.W_lo + row * G.ldw + col);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            dh[k] = make_uint4(hw[4 * k], hw[4 * k + 1], hw[4 * k + 2], hw[4 * k + 3]);
            dl[k] = make_uint4(lw[4 * k], lw[4 * k + 1], lw[4 * k + 2], lw[4 * k + 3]);
          }
        }
      }
      if (p.epilogue == 1 && row < G.M) G.e_part[nt * G.M + row] = e_acc;
      tc_fence_before();  // the TMEM reads above are complete before the buffer is released
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
      ++i;
    }
    if (lane == 0) bulk_wait<0>();  // every TMA store of this warp has completed
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(2 * BN)));
  }
}

// ------------------------------------------------------------------ host side
using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                              const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void * p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cuda_check(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q),
               "cudaGetDriverEntryPoint(cuTensorMapEncodeTiled)");
    if (!p || q != cudaDriverEntryPointSuccess) throw Error(RGPU_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<EncodeFn>(p);
  }
  return fn;
}

// 2D bf16 tensor map over a row-major [rows x cols] matrix with row stride
// ld elements; box = box_rows x 64 columns, 128-byte swizzle, zero fill
// outside the matrix.
// 2D FP32 tensor map for TMA stores of 32 x 32 boxes into a row-major
// [rows x cols] matrix with row stride ld elements (128-byte swizzle: the
// box's 16-byte chunk c of row r sits at chunk c ^ (r % 8) in shared memory).
CUtensorMap make_store_map_f32(const float * ptr, int64_t rows, int64_t cols, int64_t ld) {
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) != 0 || (ld * 4) % 16 != 0)
    throw Error(RGPU_ERR_INVALID_ARGUMENT, "tensor map: base or stride not 16-byte aligned");
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(ld * 4)};
  cuuint32_t box[2] = {32, 32};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(ptr), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(RGPU_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return m;
}

CUtensorMap make_map(const __nv_bfloat16 * ptr, int64_t rows, int64_t cols, int64_t ld, int box_rows,
                     int box_k = kBK) {
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) != 0 || (ld * 2) % 16 != 0)
    throw Error(RGPU_ERR_INVALID_ARGUMENT, "tensor map: base or stride not 16-byte aligned");
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(ld * 2)};
  cuuint32_t box[2] = {cuuint32_t(box_k), cuuint32_t(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(ptr), dims, strides,
                           box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           box_k == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(RGPU_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return m;
}

__global__ void split_bf16_kernel(const float * __restrict__ x, int64_t rows, int64_t cols, int64_t ldx,
                                  __nv_bfloat16 * __restrict__ hi, __nv_bfloat16 * __restrict__ lo, int64_t ldo) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= rows * ldo) return;
  int64_t r = i / ldo, c = i - r * ldo;
  float v = (c < cols) ? x[r * ldx + c] : 0.f;
  __nv_bfloat16 h = __float2bfloat16_rn(v);
  hi[i] = h;
  lo[i] = __float2bfloat16_rn(v - __bfloat162float(h));
}

}  // namespace

void split_bf16(const float * x, int64_t rows, int64_t cols, int64_t ldx, __nv_bfloat16 * hi, __nv_bfloat16 * lo,
                int64_t ldo, cudaStream_t st) {
  if (rows * ldo <= 0) return;
  split_bf16_kernel<<<div_up(rows * ldo, 256), 256, 0, st>>>(x, rows, cols, ldx, hi, lo, ldo);
  RGPU_LAUNCHED();
}

// Polls of the MMA warp's waits for staged operands: kSpinLimit, unless a
// test lowers it to make those waits run out (rgpu_debug_set_gemm_wait_limit).
static std::atomic<long long> g_mma_wait_limit{kSpinLimit};

void set_gemm_wait_limit(long long polls) { g_mma_wait_limit.store(polls < 0 ? kSpinLimit : polls); }

// Status word of the tcgen05 GEMM: one per device, allocated on the current
// device the first time a GEMM runs there.
static PerDevice<TcStatus *> g_tc_status;
static TcStatus * tc_status() {
  return g_tc_status.once(current_device(), [](TcStatus *& p) {
    TcStatus * q = nullptr;
    cuda_check(cudaMalloc(&q, sizeof(TcStatus)), "cudaMalloc(tc status)");
    cuda_check(cudaMemset(q, 0, sizeof(TcStatus)), "cudaMemset(tc status)");
    p = q;
  });
}

TcStatus * tc_status_word() { return tc_status(); }

void gemm_bf16x3(const Bf16x3Gemm & g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0) return;
  constexpr int BN = kTcTileN, STAGES = 2;
  const size_t smem = Smem<BN, STAGES>::TOTAL;
  CUtensorMap a_hi = make_map(g.A_hi, g.M, g.K, g.lda, kBM);
  CUtensorMap a_lo = make_map(g.A_lo, g.M, g.K, g.lda, kBM);
  CUtensorMap b_hi = make_map(g.B_hi, g.N, g.K, g.ldb, BN);
  CUtensorMap b_lo = make_map(g.B_lo, g.N, g.K, g.ldb, BN);
  TcArgs t;
  t.M = g.M;
  t.N = g.N;
  t.K = g.K;
  t.epilogue = g.epilogue;
  t.C = g.C;
  t.ldc = g.ldc;
  t.W_hi = g.W_hi;
  t.W_lo = g.W_lo;
  t.ldw = g.ldw;
  t.alpha = g.alpha;
  t.zeta = g.zeta;
  t.e_part = g.e_part;
  t.row_scale = g.row_scale;
  t.status = tc_status();
  t.mma_wait_limit = g_mma_wait_limit.load();
  cuda_check(cudaFuncSetAttribute(gemm_tc_kernel<BN, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem)),
             "cudaFuncSetAttribute(gemm_tc)");
  dim3 grid(div_up(g.N, BN), div_up(g.M, kBM));
  gemm_tc_kernel<BN, STAGES><<<grid, kThreads, smem, st>>>(a_hi, a_lo, b_hi, b_lo, t);
  RGPU_LAUNCHED();
  cuda_check(cudaGetLastError(), "gemm_tc launch");
}

void gemm_bf16x3_status(const Bf16x3Gemm & g, int * status_dev, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0) return;
  constexpr int BN = kTcTileN, STAGES = 2;
  const size_t smem = Smem<BN, STAGES>::TOTAL;
  CUtensorMap a_hi = make_map(g.A_hi, g.M, g.K, g.lda, kBM);
  CUtensorMap a_lo = make_map(g.A_lo, g.M, g.K, g.lda, kBM);
  CUtensorMap b_hi = make_map(g.B_hi, g.N, g.K, g.ldb, BN);
  CUtensorMap b_lo = make_map(g.B_lo, g.N, g.K, g.ldb, BN);
  TcArgs t;
  t.M = g.M;
  t.N = g.N;
  t.K = g.K;
  t.epilogue = g.epilogue;
  t.C = g.C;
  t.ldc = g.ldc;
  t.W_hi = g.W_hi;
  t.W_lo = g.W_lo;
  t.ldw = g.ldw;
  t.alpha = g.alpha;
  t.zeta = g.zeta;
  t.e_part = g.e_part;
  t.row_scale = g.row_scale;
  t.status = reinterpret_cast<TcStatus *>(status_dev);
  t.mma_wait_limit = g_mma_wait_limit.load();
  cuda_check(cudaFuncSetAttribute(gemm_tc_kernel<BN, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem)),
             "cudaFuncSetAttribute(gemm_tc)");
  dim3 grid(div_up(g.N, BN), div_up(g.M, kBM));
  gemm_tc_kernel<BN, STAGES><<<grid, kThreads, smem, st>>>(a_hi, a_lo, b_hi, b_lo, t);
  RGPU_LAUNCHED();
  cuda_check(cudaGetLastError(), "gemm_tc launch");
}


template <int BN, int STAGES, int BK>
void grouped_launch(const Bf16x3Gemm * gs, int n, cudaStream_t st) {
  TcGroupedArgs p;
  std::memset(&p, 0, sizeof(p));
  int ng = 0;
  int64_t tiles = 0;
  for (int i = 0; i < n; ++i) {
    const Bf16x3Gemm & g = gs[i];
    if (g.M <= 0 || g.N <= 0) continue;
    if (ng == kMaxGroups) throw Error(RGPU_ERR_INVALID_ARGUMENT, "grouped GEMM: more than 16 groups");
    if (ng > 0 && (g.epilogue != p.epilogue || g.zeta != p.zeta))
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "grouped GEMM: groups must share the epilogue");
    p.epilogue = g.epilogue;
    p.zeta = g.zeta;
    if (g.K % BK != 0) throw Error(RGPU_ERR_INVALID_ARGUMENT, "grouped GEMM: K must be a multiple of the K block");
    p.a_hi[ng] = make_map(g.A_hi, g.M, g.K, g.lda, kBM, BK);
    p.a_lo[ng] = make_map(g.A_lo, g.M, g.K, g.lda, kBM, BK);
    p.b_hi[ng] = make_map(g.B_hi, g.N, g.K, g.ldb, BN, BK);
    p.b_lo[ng] = make_map(g.B_lo, g.N, g.K, g.ldb, BN, BK);
    if (g.epilogue == 0) p.c_map[ng] = make_store_map_f32(g.C, g.M, g.N, g.ldc);
    TcGroup & G = p.grp[ng];
    G.M = g.M;
    G.N = g.N;
    G.K = g.K;
    G.C = g.C;
    G.ldc = g.ldc;
    G.W_hi = g.W_hi;
    G.W_lo = g.W_lo;
    G.ldw = g.ldw;
    G.alpha = g.alpha;
    G.e_part = g.e_part;
    G.row_scale = g.row_scale;
    G.n_tiles = (g.N + BN - 1) / BN;
    G.tile0 = tiles;
    G.tile_mask = g.seg_mode ? g.tile_mask : nullptr;
    tiles += G.n_tiles * ((g.M + kBM - 1) / kBM);
    if (ng == 0) {
      p.seg.mode = g.seg_mode;
      p.seg.G = g.seg_G;
      p.seg.LD = g.seg_LD;
      p.seg.LO = g.seg_LO;
    } else if (g.seg_mode != p.seg.mode || g.seg_G != p.seg.G || g.seg_LD != p.seg.LD || g.seg_LO != p.seg.LO) {
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "grouped GEMM: groups must share the species segments");
    }
    if (g.seg_mode) {
      const int64_t units = int64_t(g.seg_G) * g.seg_LD + int64_t(g.seg_G) * (g.seg_G - 1) / 2 * g.seg_LO;
      if (g.seg_mode < 0 || g.seg_mode > 2 || g.seg_G < 1 || g.seg_G > 32 || g.seg_LD < 1 || g.seg_LO < 1 ||
          32 * units != (g.seg_mode == 1 ? g.K : g.N))
        throw Error(RGPU_ERR_INVALID_ARGUMENT, "grouped GEMM: species segments do not tile the feature columns");
    }
    ++ng;
  }
  if (ng == 0) return;
  p.n_groups = ng;
  p.n_tiles = tiles;
  p.status = tc_status();
  p.mma_wait_limit = g_mma_wait_limit.load();
  int dev = 0, sms = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  const size_t smem = Smem<BN, STAGES, BK>::TOTAL_GROUPED;
  cuda_check(cudaFuncSetAttribute(gemm_tc_grouped_kernel<BN, STAGES, BK>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
             "cudaFuncSetAttribute(gemm_tc_grouped)");
  const int grid = int(std::min<int64_t>(tiles, sms));
  gemm_tc_grouped_kernel<BN, STAGES, BK><<<grid, kThreads, smem, st>>>(p);
  RGPU_LAUNCHED();
  cuda_check(cudaGetLastError(), "gemm_tc_grouped launch");
}

// Pipelines of the grouped GEMM (tile 128 x kTcTileN): 0 = 4 stages of K
// blocks of 32 (64-byte swizzle, 192 KB of stages), 1 = 3 stages of 32,
// 2 = 2 stages of K blocks of 64 (128-byte swizzle), used only when every
// group's K is a multiple of 64 (else variant 0 runs).
void gemm_bf16x3_grouped(const Bf16x3Gemm * gs, int n, cudaStream_t st, int variant) {
  if (variant == 2) {
    for (int i = 0; i < n; ++i)
      if (gs[i].M > 0 && gs[i].N > 0 && gs[i].K % 64 != 0) variant = 0;
  }
  switch (variant) {
    case 1:
      grouped_launch<kTcTileN, 3, 32>(gs, n, st);
      break;
    case 2:
      grouped_launch<kTcTileN, 2, 64>(gs, n, st);
      break;
    default:
      grouped_launch<kTcTileN, 4, 32>(gs, n, st);
  }
}

int gemm_tc_timeout(bool reset) {
  TcStatus h{};
  cuda_check(cudaMemcpy(&h, tc_status(), sizeof(h), cudaMemcpyDeviceToHost), "tc status");
  if (reset && h.timeout) cuda_check(cudaMemset(tc_status(), 0, sizeof(TcStatus)), "tc status reset");
  return h.timeout ? h.where : 0;
}

}  // namespace rgpu
