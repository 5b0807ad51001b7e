// Power spectrum, FP32 fast path: forward (the unnormalised p in the packed
// layout of rgpu_internal.h, as a BF16 hi/lo split for the tensor-core
// GEMMs, plus 1/|p| per row, which the GEMM epilogue and the backward apply)
// and the adjoint dE/dx -> dE/dc.
//
// Same contractions as powerspectrum.cu (calculator_spherical_invariants.hh:
// 747-794 forward, 588-652 and 796-921 for the gradient it replaces), laid
// out for the SIMT pipes: the centre's coefficients sit in shared memory as
// [species][n][l-block padded to a multiple of 4], so every length-(2l+1)
// product over m is a few 16-byte loads, and l is a compile-time constant
// in every inner loop. The packed layout keeps one entry per symmetric pair
// of same-species Gram entries, so both kernels touch S n(n-1)/2 (L+1)
// fewer columns than the reference's layout holds.
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

// Sum over the block, one barrier: every warp posts its partial sum, then
// every thread adds the posts. `red` may be written again only after
// another barrier.
__device__ __forceinline__ float block_sum_f(float v, float * red) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float t = 0.f;
  for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w];
  return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void * p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// 16-byte asynchronous copy global -> shared (cp.async, L2 only), and its
// group commit / wait.
__device__ __forceinline__ void cp_async16(void * smem, const void * gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// Bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned) into L2.
__device__ __forceinline__ void prefetch_l2(const void * p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// One task of the forward: tile (i, j), i <= j, of every l-block, i.e. G_l
// over rows 2i, 2i+1 and columns 2j, 2j+1. Row pointers are at column 0 of
// the centre's coefficients; a1 / b1 repeat a0 / b0 when row 2i+1 / 2j+1 is
// beyond S n. Lanes with consecutive i read rows 2i apart; taking row 2i + 1
// first (sw) when bit 2 of i is set spreads the 8 lanes of a 16-byte load
// phase over 8 different bank groups (the row stride is an odd number of
// 16-byte units). A tile of a species pair the centre has no neighbour of
// (live false) holds zeros and reads no coefficients.
struct FwdTask {
  const float * a0;
  const float * a1;
  const float * b0;
  const float * b1;
  int base, T;  // column of the tile at l = L; tiles per l of its segment
  bool sw, diag, i1, j1, live;
};

// Tile k of l-blocks l .. L: scaled by lf (sqrt2 lf off the diagonal), the
// entry below the diagonal of a diagonal tile and rows or columns beyond
// S n zero, stored as 4 consecutive columns at base + 4 (L - l) T (8 bytes
// of BF16 hi, 8 of lo, 16 of FP32 when X is given). Returns the sum of
// squares.
template <int L, int l>
__device__ __forceinline__ float fwd_task(const FwdTask & k, float * __restrict__ X, __nv_bfloat16 * __restrict__ hr,
                                          __nv_bfloat16 * __restrict__ lr) {
  if constexpr (l > L) {
    return 0.f;
  } else {
    constexpr int Q = pad4(2 * l + 1) / 4, O = offp(l);
    const float lf = rsqrtf(float(2 * l + 1)), lf2 = lf * kSqrt2f;
    float u00 = 0.f, u10 = 0.f, u01 = 0.f, u11 = 0.f;  // u_rc: row a_r, column J0 + c
    if (k.live) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const float4 x0 = *reinterpret_cast<const float4 *>(k.a0 + O + 4 * q);
        const float4 x1 = *reinterpret_cast<const float4 *>(k.a1 + O + 4 * q);
        const float4 y0 = *reinterpret_cast<const float4 *>(k.b0 + O + 4 * q);
        const float4 y1 = *reinterpret_cast<const float4 *>(k.b1 + O + 4 * q);
        // chained FMAs into the accumulators (one FFMA per product)
        u00 = fmaf(x0.x, y0.x, fmaf(x0.y, y0.y, fmaf(x0.z, y0.z, fmaf(x0.w, y0.w, u00))));
        u10 = fmaf(x1.x, y0.x, fmaf(x1.y, y0.y, fmaf(x1.z, y0.z, fmaf(x1.w, y0.w, u10))));
        u01 = fmaf(x0.x, y1.x, fmaf(x0.y, y1.y, fmaf(x0.z, y1.z, fmaf(x0.w, y1.w, u01))));
        u11 = fmaf(x1.x, y1.x, fmaf(x1.y, y1.y, fmaf(x1.z, y1.z, fmaf(x1.w, y1.w, u11))));
      }
    }
    // v_rc: row I0 + r, column J0 + c
    float v00 = k.sw ? u10 : u00, v10 = k.sw ? u00 : u10, v01 = k.sw ? u11 : u01, v11 = k.sw ? u01 : u11;
    v00 *= k.diag ? lf : lf2;
    v10 = (k.diag || !k.i1) ? 0.f : v10 * lf2;
    v01 = k.j1 ? v01 * lf2 : 0.f;
    v11 = (k.i1 && k.j1) ? v11 * (k.diag ? lf : lf2) : 0.f;
    const __nv_bfloat162 h0 = __floats2bfloat162_rn(v00, v10), h1 = __floats2bfloat162_rn(v01, v11);
    const float2 f0 = __bfloat1622float2(h0), f1 = __bfloat1622float2(h1);
    const __nv_bfloat162 l0 = __floats2bfloat162_rn(v00 - f0.x, v10 - f0.y);
    const __nv_bfloat162 l1 = __floats2bfloat162_rn(v01 - f1.x, v11 - f1.y);
    uint2 hw, lw;
    hw.x = *reinterpret_cast<const uint32_t *>(&h0);
    hw.y = *reinterpret_cast<const uint32_t *>(&h1);
    lw.x = *reinterpret_cast<const uint32_t *>(&l0);
    lw.y = *reinterpret_cast<const uint32_t *>(&l1);
    const int o = k.base + 4 * (L - l) * k.T;
    *reinterpret_cast<uint2 *>(hr + o) = hw;
    *reinterpret_cast<uint2 *>(lr + o) = lw;
    if (X) *reinterpret_cast<float4 *>(X + o) = make_float4(v00, v10, v01, v11);
    const float ss = v00 * v00 + v10 * v10 + v01 * v01 + v11 * v11;
    return ss + fwd_task<L, l + 1>(k, X, hr, lr);
  }
}

// p of a centre's row in the packed layout as a BF16 hi/lo split (and in
// FP32 when X is given), one 2 x 2 tile of every l-block per task straight
// to HBM, the segments' padding set to zero, and the row's scale 1/|p| (1
// without normalisation); the packed values keep |p|. Consecutive lanes take
// consecutive tiles (mostly of one column pair, whose coefficient rows they
// then read as broadcasts); tiles of species pairs the centre lacks are
// written as zeros. Persistent: each block loops over centres, prefetching
// the next centre's coefficient tile with cp.async while it works on the
// current one.
template <int L>
__global__ void __launch_bounds__(kThreads)
ps_fwd_f32_kernel(PsArgs a, const float * __restrict__ C, float * __restrict__ X,
                  __nv_bfloat16 * __restrict__ Xh, __nv_bfloat16 * __restrict__ Xl,
                  float * __restrict__ row_scale) {
  constexpr int L1 = L + 1, RS = row_stride(L);
  extern __shared__ __align__(16) float smf[];
  const FeatureDims fd = a.fd;
  const int Sn = fd.Sn, tile = Sn * RS;
  float * cbuf = smf;                                          // two coefficient tiles [Sn][RS]
  int2 * tab = reinterpret_cast<int2 *>(smf + 2 * tile);       // task table
  __shared__ float red[32];
  const int np = (Sn + 1) >> 1, nt = np * (np + 1) / 2;
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    int j = int((sqrtf(8.f * float(t) + 1.f) - 1.f) * 0.5f);
    while (j > 0 && j * (j + 1) / 2 > t) --j;
    while ((j + 1) * (j + 2) / 2 <= t) ++j;
    const int i = t - j * (j + 1) / 2;
    int base, lstep;
    tile_column(fd, i, j, base, lstep);
    const uint32_t A = uint32_t(i / fd.npg), B = uint32_t(j / fd.npg);  // species groups
    tab[t] = make_int2(int(uint32_t(i) | (uint32_t(j) << 8) | (A << 16) | (B << 21)), base);
  }
  // zero columns: the end of every segment after its tiles
  const int padD = fd.lenD - 4 * L1 * fd.TD, padO = fd.lenO - 4 * L1 * fd.TO;
  const int nD = fd.G * padD, npad = nD + fd.G * (fd.G - 1) / 2 * padO;
  auto prefetch = [&](int64_t c, float * dst) {
    const float4 * src = reinterpret_cast<const float4 *>(C + size_t(c) * tile);
    for (int e = threadIdx.x; e < tile / 4; e += blockDim.x) cp_async16(dst + 4 * e, src + e);
  };
  int64_t ci = blockIdx.x;
  if (ci < a.n_centers) prefetch(ci, cbuf);
  cp_async_commit();
  for (int buf = 0; ci < a.n_centers; ci += gridDim.x, buf ^= 1) {
    const int64_t next = ci + gridDim.x;
    if (next < a.n_centers) prefetch(next, cbuf + (buf ^ 1) * tile);
    cp_async_commit();
    cp_async_wait<1>();  // this centre's copies (and the task table) are done ...
    __syncthreads();     // ... for every thread
    const float * Cp = cbuf + buf * tile;
    const int64_t row = a.row_of_center[ci];
    const size_t roff = size_t(row) * fd.Dg;
    float * Xr = X ? X + roff : nullptr;
    __nv_bfloat16 * hr = Xh + roff;
    __nv_bfloat16 * lr = Xl + roff;
    const uint32_t pm = (fd.G > 1 && a.present) ? a.present[ci] : 0xFFFFFFFFu;
    float ss = 0.f;
    for (int r = threadIdx.x; r < nt; r += blockDim.x) {
      const int2 e = tab[r];
      const uint32_t x = uint32_t(e.x);
      const int i = int(x & 0xFFu), j = int((x >> 8) & 0xFFu), A = int((x >> 16) & 31u), B = int((x >> 21) & 31u);
      FwdTask k;
      const int I0 = 2 * i, J0 = 2 * j;
      k.i1 = I0 + 1 < Sn;
      k.j1 = J0 + 1 < Sn;
      k.sw = ((i >> 2) & 1) && k.i1;
      k.a0 = Cp + (I0 + int(k.sw)) * RS;
      k.a1 = Cp + (k.i1 ? I0 + 1 - int(k.sw) : I0) * RS;
      k.b0 = Cp + J0 * RS;
      k.b1 = Cp + (k.j1 ? J0 + 1 : J0) * RS;
      k.diag = i == j;
      k.live = ((pm >> A) & (pm >> B) & 1u) != 0u;
      k.base = e.y;
      k.T = A == B ? fd.TD : fd.TO;
      ss += fwd_task<L, 0>(k, Xr, hr, lr);
    }
    for (int e = threadIdx.x; e < npad; e += blockDim.x) {
      int d;
      if (e < nD) {
        const int A = e / padD;
        d = segment_offset(fd, A, A) + 4 * L1 * fd.TD + (e - A * padD);
      } else {
        int k = (e - nD) / padO, A = 0;
        const int r = (e - nD) - k * padO;
        while (k >= fd.G - 1 - A) {
          k -= fd.G - 1 - A;
          ++A;
        }
        d = segment_offset(fd, A, A + 1 + k) + 4 * L1 * fd.TO + r;
      }
      hr[d] = __float2bfloat16_rn(0.f);
      lr[d] = __float2bfloat16_rn(0.f);
      if (Xr) Xr[d] = 0.f;
    }
    ss = block_sum_f(ss, red);  // its barrier follows every tile: this buffer may be refilled
    if (threadIdx.x == 0) {
      const float nrm = sqrtf(ss);
      row_scale[row] = (a.normalize && nrm > 0.f) ? 1.f / nrm : 1.f;
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------- backward
// Every 4-column chunk (one 2 x 2 tile) of a packed row: its slot in the
// per-centre triangle order of the backward's shared memory (tile (i, j) of
// l at l NT + j(j+1)/2 + i, NT tiles per l) in bits 0-23 and its segment's
// groups A, B in bits 24-27 and 28-31; kNoChunk for segment padding.
constexpr uint32_t kNoChunk = 0xFFFFFFFFu;
__global__ void chunk_map_kernel(FeatureDims fd, uint32_t * __restrict__ map) {
  const int c = int(blockIdx.x) * int(blockDim.x) + int(threadIdx.x);
  if (c >= fd.Dg / 4) return;
  const int LD = fd.lenD / 4, LO = fd.lenO / 4, L1 = fd.L + 1;
  const int np = (fd.Sn + 1) / 2, NT = np * (np + 1) / 2;
  int q = c, A = 0;
  while (q >= LD + (fd.G - 1 - A) * LO) {  // segments (A, A..G-1) in turn
    q -= LD + (fd.G - 1 - A) * LO;
    ++A;
  }
  int B, T;
  if (q < LD) {
    B = A;
    T = fd.TD;
  } else {
    q -= LD;
    const int k = q / LO;
    B = A + 1 + k;
    q -= k * LO;
    T = fd.TO;
  }
  const int lr = q / T;  // 0 for l = L (l descends inside a segment)
  if (lr >= L1) {
    map[c] = kNoChunk;
    return;
  }
  const int t = q - lr * T;
  int ii, jj;
  if (A < B) {
    jj = t / fd.npg;
    ii = t - jj * fd.npg;
  } else {
    jj = 0;
    while ((jj + 1) * (jj + 2) / 2 <= t) ++jj;
    ii = t - jj * (jj + 1) / 2;
  }
  const int i = A * fd.npg + ii, j = B * fd.npg + jj;
  map[c] = uint32_t((fd.L - lr) * NT + j * (j + 1) / 2 + i) | (uint32_t(A) << 24) | (uint32_t(B) << 28);
}

// Per centre: the projected gradient G = (g - x (x.g)) / |p| of the packed
// row (x as BF16 hi + lo, g = dE/dx) is formed in shared memory: g arrives
// by cp.async, each 16-byte chunk (one 2 x 2 tile) at its slot of the per-l
// triangles (chunk_map), then two passes over x (L2 reads) reduce x.g and
// project in place. A chunk of a species pair the
// centre has no neighbour of is neither read nor trusted (x is zero there,
// and the GAP backward leaves such columns unwritten when no row of the GEMM
// tile holds the pair): its slot is set to zero. Then dE/dc = lf_l H_l c_l with the
// symmetric
//   H_l[I][J] = sqrt2 G_l(I J)  (I != J),   H_l[I][I] = 2 G_l(I I),
// the derivative of E through the packed entries sqrt2 G_l[I][J] (I < J) and
// G_l[I][I] of the Gram matrix, read straight from the tiles: tile (i, j),
// i <= j, holds rows 2i, 2i+1 and columns 2j, 2j+1.
//
// Contraction tasks are (row pair 2ip, 2ip+1; 4-wide column group g of the
// padded coefficient rows) with g fastest, so the lanes of a half-warp share
// their rows (one broadcast 16-byte load per tile, uniform trip counts and
// the same skips of the species the centre lacks) and
// read consecutive 16-byte chunks of a coefficient row; each task stores its
// two rows of dE/dc as 8-byte pairs. The chunk map is copied into shared
// memory once per block. The next centre's coefficients are copied in with
// cp.async, and its x and dE/dx rows prefetched into L2, while this one is
// worked on.
template <int L>
__global__ void __launch_bounds__(kBwdThreads, 4)
ps_bwd_f32_kernel(PsArgs a, const float * __restrict__ C, const __nv_bfloat16 * __restrict__ Xh,
                  const __nv_bfloat16 * __restrict__ Xl, const float * __restrict__ row_scale,
                  const float * __restrict__ dX, const uint32_t * __restrict__ chunk_map,
                  const uint32_t * __restrict__ present, float * __restrict__ dC) {
  constexpr int L1 = L + 1, RS = row_stride(L), K = L1 * L1;
  extern __shared__ __align__(16) float smf[];
  const FeatureDims fd = a.fd;
  const int Sn = fd.Sn, npg = fd.npg;
  const int NP = (Sn + 1) >> 1, NT = NP * (NP + 1) / 2;
  const int tile = Sn * RS, tileP = (Sn + (Sn & 1)) * RS;  // a coefficient tile; its buffer
  float * Cb = smf;                // two coefficient buffers [Sn rounded up to even][RS]
  float * Ts = Cb + 2 * tileP;     // G: L1 triangles of NT tiles
  const int zslot = L1 * NT;       // a zero tile after the triangles
  uint32_t * smap = reinterpret_cast<uint32_t *>(Ts + 4 * (zslot + 1));  // the chunk map
  __shared__ float red[32];
  // column groups of the contraction: the 4-wide chunks of the padded
  // coefficient row in order (group g covers columns 4g .. 4g+3, of block
  // l = grp_l[g]), so the 8 lanes of a 16-byte load phase read 8 consecutive
  // chunks of one row
  constexpr int kG = offp(L + 1) / 4;
  __shared__ int8_t grp_l[kG];
  for (int t = threadIdx.x; t < kG; t += blockDim.x) {
    int l = 0;
    while (offp_rt(l + 1) <= 4 * t) ++l;
    grp_l[t] = int8_t(l);
  }
  // the row after an odd S n's last row stays zero in both buffers
  for (int e = tile + threadIdx.x; e < tileP; e += blockDim.x) Cb[e] = Cb[tileP + e] = 0.f;
  const int nq = fd.Dg >> 2;  // 4-column chunks of the row (one tile each)
  for (int c = threadIdx.x; c < nq; c += blockDim.x) smap[c] = chunk_map[c];
  float4 * T4 = reinterpret_cast<float4 *>(Ts);
  if (threadIdx.x == 0) T4[zslot] = make_float4(0.f, 0.f, 0.f, 0.f);
  auto prefetch = [&](int64_t c, float * dst) {
    const float4 * src = reinterpret_cast<const float4 *>(C + size_t(c) * tile);
    for (int e = threadIdx.x; e < tile / 4; e += blockDim.x) cp_async16(dst + 4 * e, src + e);
  };
  int64_t ci = blockIdx.x;
  if (ci < a.n_centers) prefetch(ci, Cb);
  cp_async_commit();
  // persistent: the tables above serve every centre of this block
  for (int buf = 0; ci < a.n_centers; ci += gridDim.x, buf ^= 1) {
    const float * Cp = Cb + buf * tileP;
    const int64_t row = a.row_of_center[ci];
    const uint2 * xh = reinterpret_cast<const uint2 *>(Xh + size_t(row) * fd.Dg);
    const uint2 * xl = reinterpret_cast<const uint2 *>(Xl + size_t(row) * fd.Dg);
    const float4 * g4 = reinterpret_cast<const float4 *>(dX + size_t(row) * fd.Dg);
    const float rs = row_scale[row];  // x = rs * p; G = rs * (g - x (x.g))
    const uint32_t pm = fd.G > 1 ? present[ci] : 0xFFFFFFFFu;  // species with neighbours (the groups)
    auto live = [&](uint32_t e) {
      return e != kNoChunk && ((pm >> ((e >> 24) & 15u)) & 1u) && ((pm >> (e >> 28)) & 1u);
    };
    // g into its slots by asynchronous copies (all in flight at once); the
    // slots of absent pairs are zeroed
    for (int c = threadIdx.x; c < nq; c += blockDim.x) {
      const uint32_t e = smap[c];
      if (e == kNoChunk) continue;
      if (live(e))
        cp_async16(T4 + (e & 0xFFFFFFu), g4 + c);
      else
        T4[e & 0xFFFFFFu] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    cp_async_commit();
    const int64_t next = ci + gridDim.x;
    if (next < a.n_centers) {
      prefetch(next, Cb + (buf ^ 1) * tileP);
      if (threadIdx.x == 0) {  // and the next centre's x and dE/dx rows into L2
        const size_t nrow = size_t(a.row_of_center[next]) * fd.Dg;
        prefetch_l2(Xh + nrow, uint32_t(fd.Dg) * 2u);
        prefetch_l2(Xl + nrow, uint32_t(fd.Dg) * 2u);
        prefetch_l2(dX + nrow, uint32_t(fd.Dg) * 4u);
      }
    }
    cp_async_commit();
    cp_async_wait<1>();  // g and this centre's coefficients have landed ...
    __syncthreads();     // ... for every thread
    if (a.normalize) {
      // x.g, then G = rs (g - x (x.g)) in place; x is read twice from L2,
      // by loads that wait on nothing (a chunk without a slot reads the zero
      // tile; the slots of absent pairs hold zero)
      float dot = 0.f;
#pragma unroll 4
      for (int c = threadIdx.x; c < nq; c += blockDim.x) {
        const uint32_t e = smap[c];
        const uint2 hv = xh[c], lv = xl[c];
        const float4 t = T4[e == kNoChunk ? zslot : int(e & 0xFFFFFFu)];
        const __nv_bfloat16 * hb = reinterpret_cast<const __nv_bfloat16 *>(&hv);
        const __nv_bfloat16 * lb = reinterpret_cast<const __nv_bfloat16 *>(&lv);
        dot = fmaf(__bfloat162float(hb[0]) + __bfloat162float(lb[0]), t.x, dot);
        dot = fmaf(__bfloat162float(hb[1]) + __bfloat162float(lb[1]), t.y, dot);
        dot = fmaf(__bfloat162float(hb[2]) + __bfloat162float(lb[2]), t.z, dot);
        dot = fmaf(__bfloat162float(hb[3]) + __bfloat162float(lb[3]), t.w, dot);
      }
      dot = block_sum_f(dot, red) * rs;
      const float k = rs * dot;
      // each thread projects the chunks it read
#pragma unroll 4
      for (int c = threadIdx.x; c < nq; c += blockDim.x) {
        const uint32_t e = smap[c];
        const uint2 hv = __ldcs(xh + c), lv = __ldcs(xl + c);
        if (!live(e)) continue;
        const int d = int(e & 0xFFFFFFu);
        const __nv_bfloat16 * hb = reinterpret_cast<const __nv_bfloat16 *>(&hv);
        const __nv_bfloat16 * lb = reinterpret_cast<const __nv_bfloat16 *>(&lv);
        float4 t = T4[d];
        t.x = (t.x - (__bfloat162float(hb[0]) + __bfloat162float(lb[0])) * k) * rs;
        t.y = (t.y - (__bfloat162float(hb[1]) + __bfloat162float(lb[1])) * k) * rs;
        t.z = (t.z - (__bfloat162float(hb[2]) + __bfloat162float(lb[2])) * k) * rs;
        t.w = (t.w - (__bfloat162float(hb[3]) + __bfloat162float(lb[3])) * k) * rs;
        T4[d] = t;
      }
      __syncthreads();  // G is complete
    }

    // dE/dc_(i l m) = lf_l sqrt2 (sum_j G(i j) c_(j l m) + (sqrt2 - 1) G(i i) c_(i l m)),
    // over the tiles of row pair ip: (j, ip) for j < ip (transposed), the
    // diagonal tile, then (ip, j) for j > ip
    for (int t = threadIdx.x; t < kG * NP; t += blockDim.x) {
      const int ip = t / kG, g = t - ip * kG;
      // rows of a species the centre has no neighbour of: their dE/dc is
      // never read (no pair of that species), so the task is skipped
      const int B = ip / npg;
      if (!((pm >> B) & 1u)) continue;
      const int l = grp_l[g];
      const float4 * Tl = T4 + l * NT;
      const int i0 = 2 * ip;
      float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
      // h_rc = G(i0 + r, 2j + c), cj = row 2j of the coefficients (row S n of
      // an odd S n is the buffer's zero row, and its h are zero)
      auto acc = [&](float h00, float h10, float h01, float h11, const float * cj) {
        const float4 c0 = *reinterpret_cast<const float4 *>(cj);
        const float4 c1 = *reinterpret_cast<const float4 *>(cj + RS);
        a0.x = fmaf(h01, c1.x, fmaf(h00, c0.x, a0.x));
        a0.y = fmaf(h01, c1.y, fmaf(h00, c0.y, a0.y));
        a0.z = fmaf(h01, c1.z, fmaf(h00, c0.z, a0.z));
        a0.w = fmaf(h01, c1.w, fmaf(h00, c0.w, a0.w));
        a1.x = fmaf(h11, c1.x, fmaf(h10, c0.x, a1.x));
        a1.y = fmaf(h11, c1.y, fmaf(h10, c0.y, a1.y));
        a1.z = fmaf(h11, c1.z, fmaf(h10, c0.z, a1.z));
        a1.w = fmaf(h11, c1.w, fmaf(h10, c0.w, a1.w));
      };
      const float * cb = Cp + 4 * g;
      // j < ip: tiles (j, ip), transposed, one run per group A <= B; groups the
      // centre lacks hold zero tiles and zero coefficients and are skipped
      const float4 * tp = Tl + ip * (ip + 1) / 2;  // tile (0, ip)
      for (int A = 0; A <= B; ++A) {
        const int j0 = A * npg, j1 = min(j0 + npg, ip);
        if (j1 <= j0 || !((pm >> A) & 1u)) continue;
        const float * cj = cb + 2 * j0 * RS;
#pragma unroll 2
        for (int j = j0; j < j1; ++j, cj += 2 * RS) {
          const float4 v = tp[j];  // (2j, i0), (2j+1, i0), (2j, i0+1), (2j+1, i0+1)
          acc(v.x, v.z, v.y, v.w, cj);
        }
      }
      {
        const float4 v = tp[ip];  // (i0, i0), zero, (i0, i0+1), (i0+1, i0+1)
        acc(kSqrt2f * v.x, v.z, v.z, kSqrt2f * v.w, cb + i0 * RS);
      }
      // j > ip: tiles (ip, j), one run per group A >= B
      for (int A = B; A < fd.G; ++A) {
        const int j0 = max(A * npg, ip + 1), j1 = min((A + 1) * npg, NP);
        if (j1 <= j0 || !((pm >> A) & 1u)) continue;
        const float4 * tq = Tl + j0 * (j0 + 1) / 2 + ip;  // tile (ip, j0)
        const float * cj = cb + 2 * j0 * RS;
#pragma unroll 2
        for (int j = j0; j < j1; ++j, cj += 2 * RS) {
          const float4 v = *tq;  // (i0, 2j), (i0+1, 2j), (i0, 2j+1), (i0+1, 2j+1)
          acc(v.x, v.y, v.z, v.w, cj);
          tq += j + 1;
        }
      }
      const int M = 2 * l + 1, m0 = 4 * g - offp_rt(l);
      const float sc = rsqrtf(float(M)) * kSqrt2f;
      const float v0[4] = {a0.x, a0.y, a0.z, a0.w}, v1[4] = {a1.x, a1.y, a1.z, a1.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (m0 + e < M) {
          float * o = dC + (size_t(ci) * K + (l * l + m0 + e)) * Sn + i0;
          if (i0 + 1 < Sn) {
            if ((Sn & 1) == 0)  // 8-byte aligned pair
              *reinterpret_cast<float2 *>(o) = make_float2(v0[e] * sc, v1[e] * sc);
            else {
              o[0] = v0[e] * sc;
              o[1] = v1[e] * sc;
            }
          } else {
            o[0] = v0[e] * sc;
          }
        }
      }
    }
    __syncthreads();  // the triangles and this coefficient buffer are read no more
  }
  cp_async_wait<0>();
}

// Shared memory of the forward: two coefficient tiles and the task table.
template <int L>
size_t fwd_smem(const FeatureDims & fd) {
  const size_t np = size_t(fd.Sn + 1) / 2;
  return sizeof(float) * 2 * size_t(fd.Sn) * row_stride(L) + sizeof(int2) * np * (np + 1) / 2 + 16;
}

// Shared memory of the backward: two coefficient buffers, the per-l
// triangles of G and the chunk map.
template <int L>
size_t bwd_smem(const FeatureDims & fd) {
  const size_t Sn = size_t(fd.Sn), np = (Sn + 1) / 2;
  return sizeof(float) * (2 * (Sn + (Sn & 1)) * row_stride(L) + 4 * (size_t(L + 1) * np * (np + 1) / 2 + 1)) +
         sizeof(uint32_t) * size_t(fd.Dg / 4);
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
                        const float * row_scale, const float * dX, uint32_t * chunk_map, const uint32_t * present,
                        float * dC, cudaStream_t st) {
  if (a.n_centers == 0) return;
  if (a.fd.n > kMaxN) throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_radial above 16 is not supported on the fast path");
  const int nchunk = a.fd.Dg / 4;
  chunk_map_kernel<<<div_up(nchunk, 256), 256, 0, st>>>(a.fd, chunk_map);
  RGPU_LAUNCHED();
  constexpr size_t kMaxSmem = 227 * 1024 - 2048;
  const int threads = std::min(tile_config(a.fd.S, a.fd.n, a.fd.L).psb_threads, kBwdThreads);
#define RGPU_PSB_CASE(LL)                                                                                     \
  case LL: {                                                                                                  \
    const size_t smem = bwd_smem<LL>(a.fd);                                                                   \
    if (smem > kMaxSmem)                                                                                      \
      throw Error(RGPU_ERR_INVALID_ARGUMENT,                                                                  \
                  "species x max_radial too large for the FP32 power-spectrum backward; use FP64");           \
    RGPU_CUDA(cudaFuncSetAttribute(ps_bwd_f32_kernel<LL>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                   int(smem)));                                                               \
    ps_bwd_f32_kernel<LL><<<persistent_grid(ps_bwd_f32_kernel<LL>, threads, smem, a.n_centers),               \
                            threads, smem, st>>>(a, C, Xh, Xl, row_scale, dX, chunk_map, present, dC);        \
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
