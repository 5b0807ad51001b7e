// Scans, the stable species sort of centres, fills and small utilities.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "common.cuh"

namespace rgpu {

namespace {
std::atomic<int64_t> g_launches{0};
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int64_t launches(bool reset) {
  return reset ? g_launches.exchange(0) : g_launches.load();
}

void cuda_check(cudaError_t e, const char * what) {
  if (e != cudaSuccess) {
    throw Error(RGPU_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e) + " in " + what);
  }
}

int current_device() {
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    throw Error(RGPU_ERR_CUDA, "device ordinal " + std::to_string(dev) + " beyond the library's table of " +
                                   std::to_string(kMaxDevices) + " devices");
  return dev;
}

namespace {
std::mutex g_tile_mutex;
std::map<std::tuple<int, int, int>, TileConfig> g_tiles;
}  // namespace

TileConfig tile_config(int S, int n, int L) {
  std::lock_guard<std::mutex> lock(g_tile_mutex);
  auto it = g_tiles.find(std::make_tuple(S, n, L));
  return it == g_tiles.end() ? TileConfig{} : it->second;
}

void tile_config_to_array(const TileConfig & c, int32_t * v) {
  v[0] = c.exp_chunk;
  v[1] = c.exp_warps;
  v[2] = c.adj_threads;
  v[3] = c.adj_blocks_per_sm;
  v[4] = c.psf_threads;
  v[5] = c.psb_threads;
  v[6] = c.gemm_variant;
  v[7] = c.psf_tc;
}

TileConfig tile_config_from_array(const int32_t * v) {
  TileConfig c;
  c.exp_chunk = v[0];
  c.exp_warps = v[1];
  c.adj_threads = v[2];
  c.adj_blocks_per_sm = v[3];
  c.psf_threads = v[4];
  c.psb_threads = v[5];
  c.gemm_variant = v[6];
  c.psf_tc = v[7];
  return c;
}

void set_tile_config(int S, int n, int L, const TileConfig * c) {
  if (c) {
    auto bad = [](const char * what) { throw Error(RGPU_ERR_INVALID_ARGUMENT, std::string("tile config: ") + what); };
    if (c->exp_chunk != 8 && c->exp_chunk != 16 && c->exp_chunk != 32) bad("exp_chunk must be 8, 16 or 32");
    if (c->exp_warps < 1 || c->exp_warps > 8) bad("exp_warps must be in [1, 8]");
    if (c->adj_threads < 32 || c->adj_threads > 128 || c->adj_threads % 32) bad("adj_threads must be 32, 64, 96 or 128");
    if (c->adj_blocks_per_sm < 1 || c->adj_blocks_per_sm > 256) bad("adj_blocks_per_sm must be in [1, 256]");
    if (c->psf_threads < 64 || c->psf_threads > 256 || c->psf_threads % 32) bad("psf_threads must be a multiple of 32 in [64, 256]");
    if (c->psb_threads < 64 || c->psb_threads > 320 || c->psb_threads % 32) bad("psb_threads must be a multiple of 32 in [64, 320]");
    if (c->gemm_variant < 0 || c->gemm_variant > 2) bad("gemm_variant must be 0, 1 or 2");
    if (c->psf_tc < 0 || c->psf_tc > 1) bad("psf_tc must be 0 or 1");
  }
  std::lock_guard<std::mutex> lock(g_tile_mutex);
  if (c)
    g_tiles[std::make_tuple(S, n, L)] = *c;
  else
    g_tiles.erase(std::make_tuple(S, n, L));
}

void DevBuf::ensure(size_t bytes) {
  if (bytes <= cap && p) return;
  release();
  size_t want = bytes < 256 ? 256 : bytes;
  // grow geometrically so repeated calls with slowly growing sizes do not
  // reallocate every time
  if (want < cap * 5 / 4) want = cap * 5 / 4;
  cuda_check(cudaMalloc(&p, want), "cudaMalloc");
  cap = want;
}
void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
}

SphConst make_sph_constants() {
  SphConst h{};
  const int S = kMaxL + 2;
  for (int l = 0; l <= kMaxL; ++l) {
    double lsq = double(l) * l, lm1sq = double(l - 1) * (l - 1);
    for (int m = 0; m <= l; ++m) {
      double msq = double(m) * m;
      h.a[l * S + m] = std::sqrt((4 * lsq - 1.0) / (lsq - msq));
      h.b[l * S + m] = -1.0 * std::sqrt((lm1sq - msq) / (4 * lm1sq - 1.0));
      h.plm[l * S + m] = std::sqrt(double((l - m) * (l + m + 1)));
    }
    h.c1[l] = std::sqrt(2 * l + 1);
    h.c2[l] = -std::sqrt(1.0 + 0.5 / l);
  }
  for (int i = 0; i < (kMaxL + 1) * S; ++i) {
    h.af[i] = float(h.a[i]);
    h.bf[i] = float(h.b[i]);
    h.plmf[i] = float(h.plm[i]);
  }
  for (int l = 0; l <= kMaxL; ++l) {
    h.c1f[l] = float(h.c1[l]);
    h.c2f[l] = float(h.c2[l]);
  }
  return h;
}

namespace {

constexpr int kScanBlock = 1024;

template <typename Tin>
__global__ void scan_block_kernel(const Tin * __restrict__ in, int64_t * __restrict__ out, int64_t n,
                                  int64_t * __restrict__ block_sums) {
  __shared__ int64_t warp_tot[32];
  int64_t i = int64_t(blockIdx.x) * kScanBlock + threadIdx.x;
  int64_t v = (i < n) ? int64_t(in[i]) : 0;
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int64_t t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  int64_t excl = x - v + (wid > 0 ? warp_tot[wid - 1] : 0);
  if (i < n) out[i] = excl;
  if (threadIdx.x == kScanBlock - 1) block_sums[blockIdx.x] = excl + v;
}

__global__ void scan_add_kernel(int64_t * __restrict__ out, int64_t n,
                                const int64_t * __restrict__ block_off) {
  int64_t i = int64_t(blockIdx.x) * kScanBlock + threadIdx.x;
  if (i < n) out[i] += block_off[blockIdx.x];
}

__global__ void scan_total_kernel(const int64_t * __restrict__ block_off, int nb,
                                  int64_t * __restrict__ total) {
  *total = block_off[nb];
}

template <typename Tin>
void scan_impl(const Tin * in, int64_t * out, int64_t n, DevBuf & tmp, size_t tmp_off,
               cudaStream_t st) {
  int nb = div_up(n, kScanBlock);
  if (nb == 0) {
    cuda_check(cudaMemsetAsync(out, 0, sizeof(int64_t), st), "memset");
    return;
  }
  int64_t * sums = reinterpret_cast<int64_t *>(static_cast<char *>(tmp.p) + tmp_off);
  int64_t * sums_scan = sums + (nb + 1);
  size_t used = tmp_off + sizeof(int64_t) * 2 * (nb + 1);
  scan_block_kernel<Tin><<<nb, kScanBlock, 0, st>>>(in, out, n, sums);
  RGPU_LAUNCHED();
  if (nb == 1) {
    // total = block sum
    cuda_check(cudaMemcpyAsync(out + n, sums, sizeof(int64_t), cudaMemcpyDeviceToDevice, st), "copy");
    return;
  }
  scan_impl<int64_t>(sums, sums_scan, nb, tmp, used, st);
  scan_add_kernel<<<nb, kScanBlock, 0, st>>>(out, n, sums_scan);
  RGPU_LAUNCHED();
  scan_total_kernel<<<1, 1, 0, st>>>(sums_scan, nb, out + n);
  RGPU_LAUNCHED();
}

size_t scan_tmp_bytes(int64_t n) {
  size_t total = 0;
  while (true) {
    int64_t nb = (n + kScanBlock - 1) / kScanBlock;
    total += sizeof(int64_t) * 2 * (nb + 1);
    if (nb <= 1) break;
    n = nb;
  }
  return total + 64;
}

// ---- stable counting sort of centres by species
constexpr int kSortBlock = 1024;

__global__ void species_count_kernel(int64_t n, const int32_t * __restrict__ types,
                                     const int32_t * __restrict__ center_atom,
                                     const int8_t * __restrict__ lut, int S,
                                     int64_t * __restrict__ block_counts /*[S][nb]*/, int nb) {
  __shared__ int cnt[32];
  if (threadIdx.x < 32) cnt[threadIdx.x] = 0;
  __syncthreads();
  int64_t i = int64_t(blockIdx.x) * kSortBlock + threadIdx.x;
  if (i < n) atomicAdd(&cnt[lut[types[center_atom[i]]]], 1);
  __syncthreads();
  if (threadIdx.x < S) block_counts[int64_t(threadIdx.x) * nb + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void species_rank_kernel(int64_t n, const int32_t * __restrict__ types,
                                    const int32_t * __restrict__ center_atom,
                                    const int8_t * __restrict__ lut, int S,
                                    const int64_t * __restrict__ block_off /*[S][nb] scanned*/, int nb,
                                    int32_t * __restrict__ row_of_center,
                                    int32_t * __restrict__ center_of_row) {
  __shared__ int wcnt[32][32];  // [warp][key]
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = lane; k < 32; k += 32) wcnt[wid][k] = 0;
  __syncthreads();
  int64_t i = int64_t(blockIdx.x) * kSortBlock + threadIdx.x;
  int key = (i < n) ? lut[types[center_atom[i]]] : 31;
  unsigned same = __match_any_sync(0xffffffffu, key);
  int rank_w = __popc(same & lanemask_lt());
  if ((same & lanemask_lt()) == 0) wcnt[wid][key] = __popc(same);
  __syncthreads();
  if (i < n) {
    int before = 0;
    for (int w = 0; w < wid; ++w) before += wcnt[w][key];
    int64_t r = block_off[int64_t(key) * nb + blockIdx.x] + before + rank_w;
    row_of_center[i] = int32_t(r);
    center_of_row[r] = int32_t(i);
  }
}

__global__ void species_total_kernel(const int64_t * __restrict__ counts, int S, int nb,
                                     int64_t * __restrict__ out) {
  int s = threadIdx.x;
  if (s >= S) return;
  int64_t t = 0;
  for (int b = 0; b < nb; ++b) t += counts[int64_t(s) * nb + b];
  out[s] = t;
}

// ---- stable sort of centres by (species, species-presence mask): LSD
// passes of 5 bits over key = species << S | mask
__global__ void mask_key_kernel(int64_t n, const int32_t * __restrict__ types, const int32_t * __restrict__ center_atom,
                                const int8_t * __restrict__ lut, const uint32_t * __restrict__ present, int S,
                                uint32_t * __restrict__ key, int32_t * __restrict__ order) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t m = S >= 32 ? present[i] : present[i] & ((1u << S) - 1u);
  key[i] = (uint32_t(lut[types[center_atom[i]]]) << S) | m;
  order[i] = int32_t(i);
}

__global__ void digit_count_kernel(int64_t n, const int32_t * __restrict__ order, const uint32_t * __restrict__ key,
                                   int shift, int64_t * __restrict__ block_counts /*[32][nb]*/, int nb) {
  __shared__ int cnt[32];
  if (threadIdx.x < 32) cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t k = int64_t(blockIdx.x) * kSortBlock + threadIdx.x;
  if (k < n) atomicAdd(&cnt[(key[order[k]] >> shift) & 31u], 1);
  __syncthreads();
  if (threadIdx.x < 32) block_counts[int64_t(threadIdx.x) * nb + blockIdx.x] = cnt[threadIdx.x];
}

// Stable: positions keep their order within a digit (the tail of the last
// block takes digit 31 and sits after every real position, so it never
// counts before one).
__global__ void digit_rank_kernel(int64_t n, const int32_t * __restrict__ order_in, const uint32_t * __restrict__ key,
                                  int shift, const int64_t * __restrict__ block_off /*[32][nb] scanned*/, int nb,
                                  int32_t * __restrict__ order_out) {
  __shared__ int wcnt[32][32];  // [warp][digit]
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  wcnt[wid][lane] = 0;
  __syncthreads();
  const int64_t k = int64_t(blockIdx.x) * kSortBlock + threadIdx.x;
  const int32_t c = k < n ? order_in[k] : 0;
  const int d = k < n ? int((key[c] >> shift) & 31u) : 31;
  const unsigned same = __match_any_sync(0xffffffffu, d);
  const int rank_w = __popc(same & lanemask_lt());
  if ((same & lanemask_lt()) == 0) wcnt[wid][d] = __popc(same);
  __syncthreads();
  if (k < n) {
    int before = 0;
    for (int w = 0; w < wid; ++w) before += wcnt[w][d];
    order_out[block_off[int64_t(d) * nb + blockIdx.x] + before + rank_w] = c;
  }
}

__global__ void rows_from_order_kernel(int64_t n, const int32_t * __restrict__ order, int32_t * __restrict__ row_of_center,
                                       int32_t * __restrict__ center_of_row) {
  const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int32_t c = order[k];
  row_of_center[c] = int32_t(k);
  center_of_row[k] = c;
}

static_assert(TileMaskArgs::kSpecies >= kMaxSpecies, "tile masks cover every species");

// One warp per 128-row tile of each species' rows: the OR of its rows'
// presence masks.
__global__ void tile_mask_kernel(TileMaskArgs a, const int32_t * __restrict__ center_of_row,
                                 const uint32_t * __restrict__ present, uint32_t * __restrict__ out) {
  const int64_t t = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= a.tile_off[a.S]) return;
  int s = 0;
  while (t >= a.tile_off[s + 1]) ++s;
  const int64_t r0 = a.row0[s] + (t - a.tile_off[s]) * 128, r1 = min(r0 + 128, a.row0[s] + a.rows[s]);
  uint32_t m = 0;
  for (int64_t r = r0 + lane; r < r1; r += 32) m |= present[center_of_row[r]];
  m = __reduce_or_sync(0xffffffffu, m);
  if (lane == 0) out[t] = m;
}

__global__ void round_tf32_kernel(float * x, int64_t n) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) x[i] = to_tf32(x[i]);
}
__global__ void fill_f64_kernel(double * p, int64_t n, double v) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
__global__ void fill_f32_kernel(float * p, int64_t n, float v) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

}  // namespace

void scan_exclusive_i64(const int64_t * in, int64_t * out, int64_t n, DevBuf & tmp, cudaStream_t st) {
  tmp.ensure(scan_tmp_bytes(n));
  scan_impl<int64_t>(in, out, n, tmp, 0, st);
}
void scan_exclusive_i32to64(const int32_t * in, int64_t * out, int64_t n, DevBuf & tmp,
                            cudaStream_t st) {
  tmp.ensure(scan_tmp_bytes(n));
  scan_impl<int32_t>(in, out, n, tmp, 0, st);
}

void launch_mask_sort(int64_t n, const int32_t * types, const int32_t * center_atom, const int8_t * lut,
                      const uint32_t * present, int S, int32_t * row_of_center, int32_t * center_of_row, DevBuf & tmp,
                      cudaStream_t st) {
  if (n <= 0) return;
  const int nb = div_up(n, kSortBlock);
  const size_t cnt = size_t(32) * nb + 1;
  const size_t stmp = scan_tmp_bytes(int64_t(32) * nb);
  const size_t ibytes = (sizeof(int32_t) * size_t(n) + 255) / 256 * 256;
  tmp.ensure(3 * ibytes + 2 * sizeof(int64_t) * cnt + stmp + 256);
  char * base = static_cast<char *>(tmp.p);
  uint32_t * key = reinterpret_cast<uint32_t *>(base);
  int32_t * ord[2] = {reinterpret_cast<int32_t *>(base + ibytes), reinterpret_cast<int32_t *>(base + 2 * ibytes)};
  int64_t * counts = reinterpret_cast<int64_t *>(base + 3 * ibytes);
  int64_t * offs = counts + cnt;
  const size_t scan_off = 3 * ibytes + 2 * sizeof(int64_t) * cnt;
  mask_key_kernel<<<div_up(n, 256), 256, 0, st>>>(n, types, center_atom, lut, present, S, key, ord[0]);
  RGPU_LAUNCHED();
  const int bits = S + 5;  // species index below 32
  int cur = 0;
  for (int shift = 0; shift < bits; shift += 5, cur ^= 1) {
    digit_count_kernel<<<nb, kSortBlock, 0, st>>>(n, ord[cur], key, shift, counts, nb);
    RGPU_LAUNCHED();
    scan_impl<int64_t>(counts, offs, int64_t(32) * nb, tmp, scan_off, st);
    digit_rank_kernel<<<nb, kSortBlock, 0, st>>>(n, ord[cur], key, shift, offs, nb, ord[cur ^ 1]);
    RGPU_LAUNCHED();
  }
  rows_from_order_kernel<<<div_up(n, 256), 256, 0, st>>>(n, ord[cur], row_of_center, center_of_row);
  RGPU_LAUNCHED();
}

void launch_tile_masks(const TileMaskArgs & a, const int32_t * center_of_row, const uint32_t * present, uint32_t * out,
                       cudaStream_t st) {
  const int64_t tiles = a.tile_off[a.S];
  if (tiles <= 0) return;
  tile_mask_kernel<<<div_up(tiles * 32, 256), 256, 0, st>>>(a, center_of_row, present, out);
  RGPU_LAUNCHED();
}

void launch_species_sort(int64_t n, const int32_t * types, const int32_t * center_atom,
                         const int8_t * lut, int S, int64_t * species_count, int32_t * row_of_center,
                         int32_t * center_of_row, DevBuf & tmp, cudaStream_t st) {
  int nb = div_up(n, kSortBlock);
  if (nb == 0) {
    cuda_check(cudaMemsetAsync(species_count, 0, sizeof(int64_t) * S, st), "memset");
    return;
  }
  size_t cbytes = sizeof(int64_t) * (size_t(S) * nb + 1);
  size_t stmp = scan_tmp_bytes(int64_t(S) * nb);
  tmp.ensure(2 * cbytes + stmp + 256);
  int64_t * counts = tmp.as<int64_t>();
  int64_t * offs = counts + (size_t(S) * nb + 1);
  species_count_kernel<<<nb, kSortBlock, 0, st>>>(n, types, center_atom, lut, S, counts, nb);
  RGPU_LAUNCHED();
  species_total_kernel<<<1, 32, 0, st>>>(counts, S, nb, species_count);
  RGPU_LAUNCHED();
  // scan of counts in key-major order gives each (key, block) its first row
  scan_impl<int64_t>(counts, offs, int64_t(S) * nb, tmp, 2 * cbytes, st);
  species_rank_kernel<<<nb, kSortBlock, 0, st>>>(n, types, center_atom, lut, S, offs, nb,
                                                 row_of_center, center_of_row);
  RGPU_LAUNCHED();
}

void launch_round_tf32(float * x, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  round_tf32_kernel<<<div_up(n, 256), 256, 0, st>>>(x, n);
  RGPU_LAUNCHED();
}
void launch_fill_f64(double * p, int64_t n, double v, cudaStream_t st) {
  if (n <= 0) return;
  fill_f64_kernel<<<div_up(n, 256), 256, 0, st>>>(p, n, v);
  RGPU_LAUNCHED();
}
void launch_fill_f32(float * p, int64_t n, float v, cudaStream_t st) {
  if (n <= 0) return;
  fill_f32_kernel<<<div_up(n, 256), 256, 0, st>>>(p, n, v);
  RGPU_LAUNCHED();
}

namespace {
__global__ void add_f64_kernel(const double * __restrict__ a, const double * __restrict__ b,
                               double * __restrict__ out, int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}
__global__ void scale_f64_kernel(const double * __restrict__ x, double a, double * __restrict__ out, int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a * x[i];
}
__global__ void scale_rows_by_group_kernel(float * __restrict__ x, int64_t rows, int64_t cols,
                                           const int32_t * __restrict__ group, const double * __restrict__ scale) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  x[i] *= float(scale[group[i / cols]]);
}
}  // namespace

void launch_add_f64(const double * a, const double * b, double * out, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  add_f64_kernel<<<div_up(n, 256), 256, 0, st>>>(a, b, out, n);
  RGPU_LAUNCHED();
}
void launch_scale_f64(const double * x, double a, double * out, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  scale_f64_kernel<<<div_up(n, 256), 256, 0, st>>>(x, a, out, n);
  RGPU_LAUNCHED();
}
void launch_scale_rows_by_group(float * x, int64_t rows, int64_t cols, const int32_t * group,
                                const double * scale, cudaStream_t st) {
  if (rows * cols <= 0) return;
  scale_rows_by_group_kernel<<<div_up(rows * cols, 256), 256, 0, st>>>(x, rows, cols, group, scale);
  RGPU_LAUNCHED();
}

// ------------------------------------------------------------ packed layout
namespace {
constexpr double kSqrt2 = 1.41421356237309504880;
}

void pack_reference_row(const FeatureDims & fd, const double * ref, double * packed) {
  std::fill(packed, packed + fd.Dg, 0.);
  const int n = fd.n;
  for (int l = 0; l <= fd.L; ++l)
    for (int J = 0; J < fd.Sn; ++J)
      for (int I = 0; I <= J; ++I) {
        const int a = I / n, n1 = I - a * n, b = J / n, n2 = J - b * n;
        double v;
        if (a < b)
          v = ref[reference_column(fd, a, n1, b, n2, l)];
        else if (n1 < n2)  // both orders of a same-species pair, folded
          v = (ref[reference_column(fd, a, n1, a, n2, l)] + ref[reference_column(fd, a, n2, a, n1, l)]) / kSqrt2;
        else
          v = ref[reference_column(fd, a, n1, a, n1, l)];
        packed[packed_column(fd, l, I, J)] = v;
      }
}

void unpack_to_reference(const FeatureDims & fd, const float * packed, float scale, double * ref) {
  const int n = fd.n;
  const float inv_sqrt2 = float(1. / kSqrt2);
  for (int a = 0; a < fd.S; ++a)
    for (int b = a; b < fd.S; ++b)
      for (int n1 = 0; n1 < n; ++n1)
        for (int n2 = 0; n2 < n; ++n2)
          for (int l = 0; l <= fd.L; ++l) {
            float v;
            if (a < b) {
              v = packed[packed_column(fd, l, a * n + n1, b * n + n2)] * scale;
            } else {
              const int lo = std::min(n1, n2), hi = std::max(n1, n2);
              v = packed[packed_column(fd, l, a * n + lo, a * n + hi)] * scale;
              if (n1 != n2) v *= inv_sqrt2;  // the packed entry is sqrt2 p(n1 n2)
            }
            ref[reference_column(fd, a, n1, b, n2, l)] = double(v);
          }
}

}  // namespace rgpu
