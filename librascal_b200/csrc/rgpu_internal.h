// Internal declarations shared by the host orchestration (api.cu) and the
// kernel files. Not part of the C ABI.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rascal_b200.h"
#include "per_device.h"

namespace rgpu {

// Library error carrying an rgpu_status and the reference exception kind.
struct Error : std::runtime_error {
  int code;
  int kind;
  Error(int c, const std::string & m, int k = -1)
      : std::runtime_error(m), code(c),
        kind(k >= 0 ? k
                    : (c == RGPU_ERR_OVERFLOW
                           ? RGPU_EXC_OVERFLOW_ERROR
                           : (c == RGPU_ERR_INVALID_ARGUMENT ? RGPU_EXC_LOGIC_ERROR
                                                             : RGPU_EXC_RUNTIME_ERROR))) {}
};

void cuda_check(cudaError_t e, const char * what);
#define RGPU_CUDA(x) ::rgpu::cuda_check((x), #x)
// Ordinal of the current CUDA device, checked against kMaxDevices (Error
// RGPU_ERR_CUDA outside it).
int current_device();
// Counts launches of this library's kernels (reported by the bench).
void count_launch(int n = 1);
#define RGPU_LAUNCHED() ::rgpu::count_launch(1)

// Parsed calculator hypers (the subset the GPU path supports).
struct Hypers {
  std::string kind;  // "sphericalinvariants" | "sphericalexpansion"
  std::string name;  // registry name: prefix + canonical JSON dump
  std::string soap_type{"PowerSpectrum"};
  int max_radial{0}, max_angular{0};
  double cutoff{0}, smooth_width{0}, sigma{0};
  // cutoff_function "RadialScaling": u(r) = c / (c + (r/r0)^m) times the
  // shifted cosine (rate c, scale r0, exponent m)
  bool radial_scaling{false};
  double rs_rate{0}, rs_scale{1}, rs_exponent{0};
  bool spline{true};
  double spline_accuracy{1e-8};
  bool normalize{true};
  bool compute_gradients{false};
};
void parse_hypers(const std::string & kind, const std::string & json, Hypers & out);

// FP64 natural cubic spline of the orthonormalised GTO radial integral,
// grid_size x width values (width = n_max * (l_max + 1), index n*(l+1)+l).
struct RadialSpline {
  int grid_size{0}, width{0}, search_size{0};
  double x1{0}, h{0}, points_per_unit{0};
  std::vector<double> grid, y, y2h, center;
  void interpolate(double x, double * out) const;
};
void build_radial_spline(const Hypers & hy, RadialSpline & out);

// Launch shapes of the FP32 per-centre and per-pair kernels and of the
// grouped tensor-core GEMM, per feature shape (species S, max_radial n,
// max_angular L). The project's autotuner (librascal_b200/tune.py) times the
// candidates with CUDA events and commits its choices as a table that the
// package loads into the library; shapes without an entry use the defaults.
struct TileConfig {
  int exp_chunk = 16;          // neighbour pairs per chunk of the FP32 expansion: 8, 16 or 32
  int exp_warps = 4;           // centres (one warp each) per block of the FP32 expansion: 1..8
  int adj_threads = 128;       // threads per block of the pair adjoint: 32..128, multiple of 32
  int adj_blocks_per_sm = 64;  // grid cap of the pair adjoint, in blocks per SM: 1..256
  int psf_threads = 256;       // threads per block of the power-spectrum forward: 64..256, multiple of 32
  int psb_threads = 320;       // threads per block of the power-spectrum backward: 64..320, multiple of 32
  int gemm_variant = 0;        // grouped GEMM pipeline: 0 = 4 stages of K 32, 1 = 3 of K 32, 2 = 2 of K 64
  int psf_tc = 0;              // power-spectrum forward: 0 = FP32 pipe, 1 = tcgen05 Gram products
};
constexpr int kTileFields = 8;
TileConfig tile_config(int S, int n, int L);
// Install (c != nullptr, validated) or remove the entry of one shape.
void set_tile_config(int S, int n, int L, const TileConfig * c);
void tile_config_to_array(const TileConfig & c, int32_t * v);
TileConfig tile_config_from_array(const int32_t * v);

// Growable device buffer (reused across calls; never shrinks).
struct DevBuf {
  void * p{nullptr};
  size_t cap{0};
  void ensure(size_t bytes);
  void release();
  template <class T>
  T * as() const {
    return static_cast<T *>(p);
  }
  ~DevBuf() { release(); }
};

// Device view of the radial spline (both precisions).
struct SplineDev {
  const double * grid;
  const double * y;    // [G][W]
  const double * y2h;  // [G][W]
  const float * yf;
  const float * y2hf;
  const float4 * q4f;  // [G-1][W]: (y_k, y2h_k, y_k+1, y2h_k+1) of interval k, FP32
  double x1, h, inv_h, ppu;
  int search_size, W;
};

// Per-structure cell-list geometry (device POD), written by nl_setup.
struct NlGeom {
  double cell[9];  // reference layout: cell[i*3+j] = component i of lattice vector j
  double cinv[9];
  double mesh_min[3], ghost_min[3], ghost_max[3];
  double bound_tol;
  int nboxes[3], pmin[3], reps[3];
  int n_atoms, n_centers;
};

// Status word written by kernels (first error wins).
struct DevStatus {
  int code;
  int where;  // structure or item index
  int detail;
  int pad;
};

// ------------------------------------------------------------------ scans
// Exclusive prefix sum of n int64 values, out[n] = total. `tmp` scratch.
void scan_exclusive_i64(const int64_t * in, int64_t * out, int64_t n, DevBuf & tmp,
                        cudaStream_t st);
void scan_exclusive_i32to64(const int32_t * in, int64_t * out, int64_t n, DevBuf & tmp,
                            cudaStream_t st);

// ------------------------------------------------------------------ NL
struct NlBuffers;  // defined in nl.cu
struct NlInputs {
  int n_struct;
  int64_t n_atoms;
  const int64_t * atom_off;    // [n_struct+1]
  const double * pos;          // [n_atoms*3] original order
  const int32_t * types;       // [n_atoms]
  const double * cells;        // [n_struct*9] ASE rows
  const int32_t * pbc;         // [n_struct*3]
  const int32_t * tag2idx;     // [n_atoms] global original index of each tag, or null
  const int32_t * n_centers;   // [n_struct]
  const int64_t * center_off;  // [n_struct+1]
  const int32_t * atom_struct; // [n_atoms]
  int64_t n_centers_total;     // center_off[n_struct], known on the host
};
struct NlOutputs {
  int64_t n_centers{0}, n_pairs{0};
  int32_t * center_atom{nullptr};   // [n_centers] global original index
  int32_t * center_struct{nullptr}; // [n_centers]
  int64_t * pair_off{nullptr};      // [n_centers+1]
  int32_t * pair_j{nullptr};        // [n_pairs] global original index of the real atom
  int32_t * pair_center{nullptr};   // [n_pairs] centre row of each pair
  int32_t * pair_shift{nullptr};    // [n_pairs*3]
  double * pair_dist{nullptr};      // [n_pairs]
  double * pair_dir{nullptr};       // [n_pairs*3]
};
struct NlWork {
  DevBuf geom, counts64, scan_tmp, ghost_off, site_x, site_type, site_real, site_shift,
      site_box, box_base, box_count, box_ptr, box_fill, sorted, sorted_x, sorted_info,
      pair_count;
  int64_t last_sites{0}, last_boxes{0};
  DevBuf center_atom, center_struct, pair_off, pair_j, pair_shift, pair_dist, pair_dir, pair_center;
};
// Capacities for a neighbour list built without host synchronisation: the
// buffers are sized to them, the kernels stop at them and set status 104
// when a count exceeds its capacity (the results are then unusable).
struct NlCaps {
  int64_t sites, boxes, pairs;
};
// Builds the full list with self pairs and the strict cutoff. Without caps
// it synchronises the stream a few times to size buffers and throws Error on
// invalid input; with caps it enqueues everything and leaves the status word
// for the caller to read.
void build_neighbour_list(const NlInputs & in, double cutoff, NlWork & w, NlOutputs & out,
                          DevStatus * status_dev, DevStatus * status_host, cudaStream_t st,
                          const NlCaps * caps = nullptr);
// Site and box counts of the last list built with synchronisation.
void neighbour_list_counts(const NlWork & w, int64_t & sites, int64_t & boxes);

// ------------------------------------------------------------------ features
struct FeatureDims {
  int S;  // species in the dense layout
  int n, L, K, W;
  int nK;     // n*K
  int P;      // species pairs S(S+1)/2
  int D;      // P*n*n*(L+1)
  int Dpad;   // D rounded up to 32
  // packed layout of the FP32 path (below)
  int Sn;          // S*n: rows of a centre's per-l Gram matrix
  int G, npg;      // groups of row pairs (S when n is even, else 1) and pairs per group
  int TD, TO;      // 2 x 2 tiles per l of a diagonal / off-diagonal block of groups
  int lenD, lenO;  // columns of a diagonal / off-diagonal segment (all l), a multiple of 32
  int Dg;          // row length: G lenD + G(G-1)/2 lenO
};

// RadialScaling cutoff parameters (on = 0: plain shifted cosine).
struct RadialScalingDev {
  int on;
  double rate, exponent, scale;
};
struct ExpansionArgs {
  FeatureDims fd;
  SplineDev sp;
  RadialScalingDev rs;
  const double * center_contrib;  // [n] / sqrt(4 pi) already applied
  const int8_t * species_lut;     // [130] -> species index or -1
  double rc, sw;
  int64_t n_centers;
  const int32_t * center_atom;
  const int64_t * pair_off;
  const int32_t * pair_j;
  const double * pair_dist;
  const double * pair_dir;
  const int32_t * types;
};
// C[i][S][n][K] and the per-centre species presence bitmask.
void launch_expansion_fp64(const ExpansionArgs & a, double * C, uint32_t * present,
                           cudaStream_t st);
// FP32: C[i][S*n][row_stride(L)], each l-block padded to 4 floats (zeros in
// the padding; common.cuh), and the presence bitmask.
void launch_expansion_fp32(const ExpansionArgs & a, float * C, uint32_t * present,
                           cudaStream_t st);
// Plain-path pair gradients for centres [c0,c1): dCp[p - p_base][3][n][K]
// (non-self pairs only; the self slot is left untouched).
void launch_expansion_grad_fp64(const ExpansionArgs & a, int64_t c0, int64_t c1,
                                int64_t p_base, double * dCp, cudaStream_t st);
// Self-pair gradients: dCs[i - c0][S][3][n][K] = -sum_j (j not an image of i).
void launch_expansion_selfgrad_fp64(const ExpansionArgs & a, int64_t c0, int64_t c1,
                                    int64_t p_base, const double * dCp, double * dCs,
                                    cudaStream_t st);

// Packed column layout of the FP32 fast path's feature rows (x and its BF16
// split, dE/dx, and the model's BF16 copies of T).
//
// For each l, a centre's coefficients form an S n x (2l+1) matrix C_l (row
// I = a n + n1 for species a, radial n1), and the reference's features are
// entries of its Gram matrix G_l = lf_l C_l C_l^T (lf_l = (2l+1)^-1/2):
// p_(ab)(n1 n2 l) = s_ab G_l[a n1][b n2] for a <= b, s_ab = sqrt2 for a < b
// (calculator_spherical_invariants.hh:747-794). The packed layout stores the
// upper triangle of each G_l in 2 x 2 tiles: tile (i, j), i <= j, holds rows
// 2i, 2i+1 and columns 2j, 2j+1 as four consecutive columns
// (I & 1) + 2 (J & 1), entries with I < J multiplied by sqrt2, and the one
// entry below the diagonal of a diagonal tile (and any row or column beyond
// S n) zero. For a < b that is the reference's feature itself. For a = b
// the reference keeps both p(n1 n2) and p(n2 n1), which are equal, and the
// packed layout one entry sqrt2 p(n1 n2) (n1 < n2): the sum of squares of a
// packed row is the reference's |p|^2, and its dot product with a sparse
// point packed the same way (the two entries folded into
// (t(n1 n2) + t(n2 n1)) / sqrt2) is the reference's x . t, with
// S n(n-1)/2 (L+1) fewer columns.
//
// Tiles are ordered by the species of their rows: with n even a row pair
// lies in one species, and the pairs form G = S groups of npg = n/2; with n
// odd they form one group. Segment (A, B), A <= B in A-major order, holds
// the tiles of group A's rows and group B's columns for every l (l slowest,
// then the tile's column pair, then its row pair; TD = npg(npg+1)/2 tiles per
// l on the diagonal A = B, TO = npg^2 off it), padded with zero columns to a
// multiple of 32. A centre without a neighbour of species A has zeros in
// every segment of A, so the GEMMs skip those column ranges for tiles of
// rows that all lack A. The reference's dense order, used by the FP64 path
// and by every export, is ((key*n + n1)*n + n2)*(L+1) + l
// (property_block_sparse.hh:911-931).
__host__ __device__ inline int segment_offset(const FeatureDims & fd, int A, int B) {
  // segments before (A, A): A diagonal ones and A(G-1) - A(A-1)/2 off-diagonal ones
  int o = A * fd.lenD + (A * (fd.G - 1) - A * (A - 1) / 2) * fd.lenO;
  if (B > A) o += fd.lenD + (B - A - 1) * fd.lenO;
  return o;
}
// First column of tile (i, j), i <= j (row-pair indices), at l = L, and
// the column step from one l to the next lower one.
__host__ __device__ inline void tile_column(const FeatureDims & fd, int i, int j, int & base, int & lstep) {
  const int A = i / fd.npg, B = j / fd.npg, ii = i - A * fd.npg, jj = j - B * fd.npg;
  const int t = A < B ? jj * fd.npg + ii : jj * (jj + 1) / 2 + ii;
  base = segment_offset(fd, A, B) + 4 * t;
  lstep = 4 * (A < B ? fd.TO : fd.TD);
}
inline int packed_column(const FeatureDims & fd, int l, int I, int J) {
  int base, lstep;
  tile_column(fd, I >> 1, J >> 1, base, lstep);
  return base + (fd.L - l) * lstep + (I & 1) + 2 * (J & 1);
}
// Column of (key(a, b), n1, n2, l), a <= b, in the reference's dense order.
inline int reference_column(const FeatureDims & fd, int a, int n1, int b, int n2, int l) {
  const int key = a * fd.S - a * (a - 1) / 2 + (b - a);
  return ((key * fd.n + n1) * fd.n + n2) * (fd.L + 1) + l;
}
// A row in the reference's dense order (D values) to the packed layout (Dg
// values, zeros in the padding).
void pack_reference_row(const FeatureDims & fd, const double * ref, double * packed);
// A packed row, times `scale`, to the reference's dense order.
void unpack_to_reference(const FeatureDims & fd, const float * packed, float scale, double * ref);

struct PsArgs {
  FeatureDims fd;
  int64_t n_centers;
  bool normalize;
  const int32_t * row_of_center;  // output row for each centre (species-sorted)
  // FP32 forward: the centres' species masks (the FP32 expansion's); tiles of
  // pairs a centre lacks are written as zeros. Null: every pair computed.
  const uint32_t * present = nullptr;
};
// X rows (normalised) and inverse norms.
void launch_ps_fwd_fp64(const PsArgs & a, const double * C, double * X, double * inv_norm,
                        cudaStream_t st);
// FP32 forward: rows (packed layout, Dg columns) of the unnormalised p as a
// BF16 hi/lo split, optionally also in FP32 (X may be null), and
// row_scale[row] = 1/|p| (1 without normalisation); x = row_scale * p.
void launch_ps_fwd_fp32(const PsArgs & a, const float * C, float * X, __nv_bfloat16 * Xh,
                        __nv_bfloat16 * Xl, float * row_scale, cudaStream_t st);
// The same forward (without the FP32 copy) as tcgen05 Gram products of
// the centres' l-blocks, BF16x3 with FP32 accumulation (ps_tc.cu), for
// shapes it supports (S n <= 128, n a multiple of 4).
bool ps_fwd_tc_supported(const FeatureDims & fd);
void launch_ps_fwd_tc(const PsArgs & a, const float * C, __nv_bfloat16 * Xh, __nv_bfloat16 * Xl,
                      float * row_scale, cudaStream_t st);
// Forward used by the FP32 path: the tile configuration picks the tcgen05
// kernel when it supports the shape and no FP32 copy is asked for.
void launch_ps_fwd_fast(const PsArgs & a, const float * C, float * X, __nv_bfloat16 * Xh, __nv_bfloat16 * Xl,
                        float * row_scale, cudaStream_t st);
// Plain-path gradients of the normalised power spectrum for pairs of centres
// [c0,c1): dX[p - p_base][3][D].
void launch_ps_grad_fp64(const PsArgs & a, const ExpansionArgs & e, int64_t c0, int64_t c1,
                         int64_t p_base, const double * C, const double * X,
                         const double * inv_norm, const double * dCp, const double * dCs,
                         double * dX, cudaStream_t st);
// Adjoint: dE/dC from dE/dX rows (species-sorted, packed layout) for all centres, written
// as dC[i][lm][s*n + n'] (lm = l^2 + m; the (species, radial) index is the
// fastest so that the centre's 32 consecutive rows store coalesced).
// x is read back as row_scale * (hi + lo) of the forward's BF16 split.
// chunk_map: scratch of Dg/4 words (the launch fills it with the slot of
// every 4-column chunk of a row in the kernel's per-l triangle order and its
// species pair); present: the centres' species masks (the FP32 expansion's),
// whose absent pairs are taken as zero whatever dX holds there.
void launch_ps_bwd_fp32(const PsArgs & a, const float * C, const __nv_bfloat16 * Xh,
                        const __nv_bfloat16 * Xl, const float * row_scale, const float * dX, uint32_t * chunk_map,
                        const uint32_t * present, float * dC, cudaStream_t st);

// ------------------------------------------------------------------ GAP
struct GapSpecies {
  int64_t row0, rows;  // species segment in the sorted row order
  int m0, M, Mpad;     // sparse points of this species (global index m0..m0+M)
};
// FP64 plain GEMMs: K = X T^T (per species), energies, W, t = W T.
void gemm_nt_fp64(int64_t M, int64_t N, int64_t K, const double * A, int64_t lda,
                  const double * B, int64_t ldb, double * C, int64_t ldc, cudaStream_t st);
void gemm_nn_fp64(int64_t M, int64_t N, int64_t K, const double * A, int64_t lda,
                  const double * B, int64_t ldb, double * C, int64_t ldc, cudaStream_t st);
// k -> (e_row += alpha k^zeta, W = alpha zeta k^(zeta-1)) for FP64.
void launch_gap_pointwise_fp64(int64_t rows, int M, const double * Kmat, int64_t ldk,
                               const double * alpha, int zeta, double * W, int64_t ldw,
                               double * e_row, cudaStream_t st);
// TF32 tensor-core GEMM C = A B^T (both K-major) with optional GAP epilogue.
struct Tf32GemmArgs {
  int64_t M, N, K;  // rows of A, rows of B, reduction length (multiple of 32)
  const float * A;
  int64_t lda;
  const float * B;
  int64_t ldb;
  float * C;  // plain store (epilogue 0) or W (epilogue 1)
  int64_t ldc;
  // GAP epilogue
  int epilogue;          // 0: store C; 1: GAP forward
  const float * alpha;   // [N]
  int zeta;
  float * e_part;        // [n_tiles_N][M] row partial energies
};
void gemm_tf32(const Tf32GemmArgs & g, cudaStream_t st);

// tcgen05 GEMM, C = A B^T as a 3-term BF16 split (A_hi B_hi + A_hi B_lo +
// A_lo B_hi), FP32 accumulation in TMEM. A [M x K] and B [N x K] are
// row-major hi/lo BF16 pairs (row strides lda, ldb; 16-byte aligned).
// epilogue 0: C [M x ldc] FP32; epilogue 1: GAP forward (W_hi/W_lo
// [M x ldw] BF16, zero for columns >= N; e_part [ceil(N/256)][M]) on
// k = row_scale[r] (A B^T)[r] when row_scale is given.
struct Bf16x3Gemm {
  int64_t M, N, K;
  const __nv_bfloat16 * A_hi;
  const __nv_bfloat16 * A_lo;
  int64_t lda;
  const __nv_bfloat16 * B_hi;
  const __nv_bfloat16 * B_lo;
  int64_t ldb;
  int epilogue;
  float * C;
  int64_t ldc;
  __nv_bfloat16 * W_hi;
  __nv_bfloat16 * W_lo;
  int64_t ldw;
  const float * alpha;
  int zeta;
  float * e_part;
  const float * row_scale;
  // Species skipping over the packed feature columns (grouped launches):
  // seg_mode 1 skips the K blocks, 2 the N tiles, whose species pair is
  // absent from every row of an M-tile (tile_mask[mt]: species present in
  // the tile's rows); seg_G, seg_LD, seg_LO: groups and segment lengths in
  // units of 32 columns (FeatureDims G, lenD / 32, lenO / 32).
  const uint32_t * tile_mask = nullptr;
  int seg_mode = 0;
  int seg_G = 0, seg_LD = 0, seg_LO = 0;
};
constexpr int kTcTileN = 256;
void gemm_bf16x3(const Bf16x3Gemm & g, cudaStream_t st);
// Several GEMMs of the same epilogue kind (up to 16; K may differ) in one
// persistent launch with a double-buffered TMEM accumulator.
void gemm_bf16x3_grouped(const Bf16x3Gemm * gs, int n, cudaStream_t st, int variant = 0);
// 0 when no bounded wait of the tcgen05 GEMM gave up, else where it did.
int gemm_tc_timeout(bool reset);
// Polls of the tcgen05 GEMMs' MMA-warp operand waits (negative: the
// default); a test hook that makes those waits run out.
void set_gemm_wait_limit(long long polls);
// gemm_bf16x3 reporting a bounded wait that gave up into the caller's device
// word pair status_dev[0..1] (timeout flag, stage; zero on entry) instead of
// the per-device status word. Allocates nothing. With epilogue 1 and
// W_hi == nullptr only the energy partials are written.
void gemm_bf16x3_status(const Bf16x3Gemm & g, int * status_dev, cudaStream_t st);
// Allocation-free GAP energies e[r] = sum_n alpha_n (A_r . B_n)^zeta (noalloc.cu).
void gap_energies_noalloc(int64_t M, int64_t N, int64_t K, const float * A, const float * B,
                          const float * alpha, int zeta, float * e, cudaStream_t st);
// Measured FMA throughput (TFLOP/s) of the current device's FP32 or FP64
// pipe (peaks.cu).
double measure_fma_peak(int precision);
// hi/lo BF16 split of a row-major FP32 matrix (columns >= cols become 0).
void split_bf16(const float * x, int64_t rows, int64_t cols, int64_t ldx, __nv_bfloat16 * hi,
                __nv_bfloat16 * lo, int64_t ldo, cudaStream_t st);
// energies[structure of centre(center_of_row[row0 + r])] += e(r), where e(r)
// is e_row_fp64[r] or the sum of the n_parts FP32 partials e_part[t*ld + r].
void launch_energy_reduce(int64_t rows, int n_parts, const float * e_part, int64_t ld,
                          const double * e_row_fp64, int64_t row0, const int32_t * center_of_row,
                          const int32_t * center_struct, double * energies, cudaStream_t st);

// Plain force contraction: grad[j] += dX[p] . t_i for pairs of centres [c0,c1).
void launch_force_contract_fp64(const FeatureDims & fd, int64_t c0, int64_t c1, int64_t p_base,
                                const int64_t * pair_off, const int32_t * pair_j,
                                const int32_t * row_of_center, const double * dX,
                                const double * t, int64_t ldt, double * grad, cudaStream_t st,
                                const double * pair_dist = nullptr, const double * pair_dir = nullptr,
                                const int32_t * center_struct = nullptr, double * stress = nullptr);
// ------------------------------------------------------------------ training
// K_NM energy rows from K = X_s T_s^T (rows x M): k^zeta into row
// center_of_row[row0 + r] (atom target) or added into its structure's row.
void launch_knm_rows(int64_t rows, int M, const double * K, int zeta, const int32_t * center_of_row,
                     int64_t row0, const int32_t * center_struct, bool atom_target, const int32_t * ucol,
                     double * out, int64_t ldo, cudaStream_t st);
// K <- zeta K^(zeta-1) (1 for zeta = 1), in place.
void launch_kernel_weight(int64_t n, double * K, int zeta, cudaStream_t st);
// K_MM block of one species: out[ucol[a]][ucol[b]] = K[a][b]^zeta.
void launch_kmm_scatter(int M, const double * K, int zeta, const int32_t * ucol, double * out, int64_t ldo,
                        cudaStream_t st);
// Gradient block of one central species over one chunk of pairs.
struct KnmDerArgs {
  const int32_t * list;  // [n_list][2]: pair index relative to p_base, centre
  int64_t n_list, p_base;
  const double * dX;  // materialised dX/dr of the chunk, [pair][3][D]
  int D;
  const double * T;  // sparse points of the species, M rows of stride ldt
  int64_t ldt;
  int M;
  const double * W;  // zeta k^(zeta-1) of the species' rows, [row - row0][M]
  int64_t row0;
  const int32_t * row_of_center;
  const int32_t * pair_j;
  const int32_t * ucol;  // output column of each sparse point
  double * out;
  int64_t ldo;
};
void launch_knm_derivative(const KnmDerArgs & a, cudaStream_t st);
// Negative-stress rows of one central species over one chunk: 6 virial rows
// per centre into V, contracted with the sparse points.
struct KnmStressArgs {
  const int32_t * centres;  // centres of the species in the chunk
  int64_t n_centres, p_base;
  const int64_t * pair_off;
  const double * pair_dist;
  const double * pair_dir;
  const double * dX;  // chunk [pair][3][D]
  int D;
  double * V;  // [n_centres][6][D] scratch
  const double * T;
  int64_t ldt;
  int M;
  const double * W;
  int64_t row0;
  const int32_t * row_of_center;
  const int32_t * center_struct;
  const int32_t * ucol;
  double * out;
  int64_t ldo, stress_row0;
};
void launch_knm_stress(const KnmStressArgs & a, cudaStream_t st);

// Adjoint pair kernel: forces from dE/dC (FP32, the layout written by
// launch_ps_bwd_fp32) and recomputed dC/dr. With stress, also the unscaled
// negative stress sum_pairs r_ji (x) g_ij per structure (6 Voigt values).
void launch_pair_adjoint_fp32(const ExpansionArgs & a, const int32_t * pair_center, int64_t n_pairs,
                              const float * dC, double * forces,
                              cudaStream_t st, const int32_t * center_struct = nullptr,
                              double * stress = nullptr);

// ------------------------------------------------------------------ helpers
// Stable sort of centres by (species, presence mask): rows of one species
// with the same neighbour species become neighbours, so 128-row GEMM tiles
// share absent species. Replaces row_of_center / center_of_row.
void launch_mask_sort(int64_t n, const int32_t * types, const int32_t * center_atom, const int8_t * lut,
                      const uint32_t * present, int S, int32_t * row_of_center, int32_t * center_of_row, DevBuf & tmp,
                      cudaStream_t st);
// Per 128-row tile of each species' rows (species s: rows row0[s] ..
// row0[s] + rows[s], tiles tile_off[s] .. tile_off[s+1]): the OR of the
// presence masks of its rows.
struct TileMaskArgs {
  static constexpr int kSpecies = 16;  // the largest species count of a dense layout
  int S;
  int64_t row0[kSpecies], rows[kSpecies], tile_off[kSpecies + 1];
};
void launch_tile_masks(const TileMaskArgs & a, const int32_t * center_of_row, const uint32_t * present, uint32_t * out,
                       cudaStream_t st);
void launch_species_sort(int64_t n, const int32_t * types, const int32_t * center_atom,
                         const int8_t * lut, int S, int64_t * species_count /*[S]*/,
                         int32_t * row_of_center, int32_t * center_of_row, DevBuf & tmp,
                         cudaStream_t st);
void launch_round_tf32(float * x, int64_t n, cudaStream_t st);
void launch_fill_f64(double * p, int64_t n, double v, cudaStream_t st);
void launch_fill_f32(float * p, int64_t n, float v, cudaStream_t st);
// out = a + b; out = a x (n doubles, device)
void launch_add_f64(const double * a, const double * b, double * out, int64_t n, cudaStream_t st);
void launch_scale_f64(const double * x, double a, double * out, int64_t n, cudaStream_t st);
// x[r][c] *= scale[group[r]] for a row-major rows x cols FP32 matrix
void launch_scale_rows_by_group(float * x, int64_t rows, int64_t cols, const int32_t * group,
                                const double * scale, cudaStream_t st);

}  // namespace rgpu
