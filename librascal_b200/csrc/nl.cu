// Linked-cell neighbour list with periodic images, self pairs and the strict
// cutoff, for a batch of structures in one set of launches.
//
// Follows src/rascal/structure_managers/adaptor_neighbour_list.hh:903-1118
// (mesh, ghost images, binning, 27-box stencil), adaptor_center_contribution
// .hh:333-406 (self pair first) and adaptor_strict.hh:373-455 (d^2 <= rc^2,
// distance, direction). The pair order is the reference's: for each centre,
// stencil boxes with x slowest and z fastest, ascending tag inside a box.
// Because a box's linear index also has x slowest, the 27 stencil boxes are
// 9 runs of 3 consecutive boxes, i.e. 9 contiguous ranges of the box-sorted
// site array; a warp per centre walks them with coalesced loads, a ballot and
// a popc prefix for compaction.
//
// This file is compiled with --fmad=false: every product and sum of the
// geometry is rounded separately, in the order the CPU oracle uses, so the
// pair sets, distances and directions are bit-identical to it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "common.cuh"

namespace rgpu {
namespace {

constexpr int kThreads = 256;

__device__ void inv3(const double * m, double * r) {
  // m row-major 3x3; adjugate / determinant
  double c00 = m[4] * m[8] - m[5] * m[7];
  double c10 = m[7] * m[2] - m[8] * m[1];
  double c20 = m[1] * m[5] - m[2] * m[4];
  double det = c00 * m[0] + c10 * m[3] + c20 * m[6];
  double inv = 1.0 / det;
  r[0] = c00 * inv;
  r[1] = c10 * inv;
  r[2] = c20 * inv;
  r[3] = (m[5] * m[6] - m[3] * m[8]) * inv;
  r[4] = (m[8] * m[0] - m[6] * m[2]) * inv;
  r[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
  r[6] = (m[3] * m[7] - m[4] * m[6]) * inv;
  r[7] = (m[6] * m[1] - m[7] * m[0]) * inv;
  r[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
}

__global__ void nl_setup_kernel(int n_struct, const int64_t * __restrict__ atom_off,
                                const double * __restrict__ cells, const int32_t * __restrict__ pbc,
                                const int32_t * __restrict__ n_centers, double cutoff,
                                NlGeom * __restrict__ geom, int64_t * __restrict__ nbox,
                                DevStatus * st) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_struct) return;
  NlGeom g;
  bool zero = true;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      g.cell[i * 3 + j] = cells[s * 9 + j * 3 + i];
      if (fabs(g.cell[i * 3 + j]) >= 1e-10) zero = false;
    }
  g.n_atoms = int(atom_off[s + 1] - atom_off[s]);
  g.n_centers = n_centers[s];
  if (zero) {
    set_status(st, 100, s, 0);
    nbox[s] = 1;
    geom[s] = g;
    return;
  }
  inv3(g.cell, g.cinv);
  for (int i = 0; i < 3; ++i) {
    double mn = 0.0, mx = 0.0;
    for (int c = 0; c < 3; ++c) {
      double v = g.cell[i * 3 + c];
      mn += v * static_cast<double>(v < 0.);
      mx += v * static_cast<double>(v > 0.);
    }
    g.mesh_min[i] = mn - 2. * cutoff;
    double lmesh = mx - mn + 4. * cutoff;
    double n = ceil(lmesh / cutoff);
    g.nboxes[i] = static_cast<int>(n);
    g.ghost_min[i] = mn - cutoff;
    double lghost = mx - mn + 2 * cutoff;
    double ngb = ceil(lghost / cutoff);
    g.ghost_max[i] = ngb * cutoff + g.ghost_min[i];
  }
  double mbl = 0.;
  for (int i = 0; i < 3; ++i) mbl = fmax(mbl, g.ghost_max[i] - g.ghost_min[i]);
  g.bound_tol = mbl * 1e-8;
  double xmin[3] = {INFINITY, INFINITY, INFINITY}, xmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int corner = 0; corner < 8; ++corner) {
    double x[3];
    for (int i = 0; i < 3; ++i)
      x[i] = ((corner >> i) & 1) ? g.ghost_max[i] + g.bound_tol : g.ghost_min[i] - g.bound_tol;
    for (int i = 0; i < 3; ++i) {
      double v = g.cinv[i * 3 + 0] * x[0] + g.cinv[i * 3 + 1] * x[1] + g.cinv[i * 3 + 2] * x[2];
      xmin[i] = fmin(xmin[i], v);
      xmax[i] = fmax(xmax[i], v);
    }
  }
  for (int i = 0; i < 3; ++i) {
    int m_min = int(floor(xmin[i]));
    int m_max = int(ceil(xmax[i])) - 1;
    bool per = pbc[s * 3 + i] != 0;
    g.pmin[i] = per ? m_min : 0;
    int pmax = per ? m_max : 0;
    g.reps[i] = -g.pmin[i] + pmax + 1;
  }
  geom[s] = g;
  nbox[s] = int64_t(g.nboxes[0]) * g.nboxes[1] * g.nboxes[2];
}

__global__ void nl_check_kernel(int64_t n_atoms, const int32_t * __restrict__ atom_struct,
                                const double * __restrict__ pos, const int32_t * __restrict__ types,
                                const NlGeom * __restrict__ geom, DevStatus * st) {
  int64_t a = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (a >= n_atoms) return;
  int s = atom_struct[a];
  int t = types[a];
  if (t < 0 || t >= 130) set_status(st, 101, s, t);
  const NlGeom & g = geom[s];
  double x = pos[3 * a], y = pos[3 * a + 1], z = pos[3 * a + 2];
  for (int i = 0; i < 3; ++i) {
    double v = g.cinv[i * 3 + 0] * x + g.cinv[i * 3 + 1] * y + g.cinv[i * 3 + 2] * z;
    if (v < -1e-10 || v > 1. + 1e-10) set_status(st, 102, s, int(a));
  }
}

__device__ __forceinline__ void image_of(const NlGeom & g, int k, int p[3]) {
  p[2] = k % g.reps[2] + g.pmin[2];
  p[1] = (k / g.reps[2]) % g.reps[1] + g.pmin[1];
  p[0] = (k / (g.reps[2] * g.reps[1])) % g.reps[0] + g.pmin[0];
}

__device__ __forceinline__ bool ghost_pos(const NlGeom & g, const double * x0, const int p[3],
                                          double * out) {
  bool inside = true;
  for (int i = 0; i < 3; ++i) {
    double sh = ((g.cell[i * 3 + 0] * double(p[0]) + g.cell[i * 3 + 1] * double(p[1])) +
                 g.cell[i * 3 + 2] * double(p[2]));
    out[i] = x0[i] + sh;
    if (!((out[i] - g.ghost_min[i]) > g.bound_tol)) inside = false;
    if (!((out[i] - g.ghost_max[i]) < -g.bound_tol)) inside = false;
  }
  return inside;
}

__global__ void nl_ghost_count_kernel(int64_t n_atoms, const int32_t * __restrict__ atom_struct,
                                      const int32_t * __restrict__ tag2idx,
                                      const double * __restrict__ pos,
                                      const NlGeom * __restrict__ geom,
                                      int32_t * __restrict__ count) {
  int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n_atoms) return;
  const NlGeom & g = geom[atom_struct[t]];
  int ntot = g.reps[0] * g.reps[1] * g.reps[2];
  int c = 0;
  if (ntot > 1) {
    int64_t a = tag2idx ? tag2idx[t] : t;
    double x0[3] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
    for (int k = 0; k < ntot; ++k) {
      int p[3];
      image_of(g, k, p);
      if (p[0] == 0 && p[1] == 0 && p[2] == 0) continue;
      double gp[3];
      if (ghost_pos(g, x0, p, gp)) ++c;
    }
  }
  count[t] = c;
}

__device__ __forceinline__ bool box_of(const NlGeom & g, const double * x, double cutoff,
                                       int b[3]) {
  bool ok = true;
  for (int i = 0; i < 3; ++i) {
    double d = x[i] - g.mesh_min[i];
    b[i] = max(1, static_cast<int>(floor(d / cutoff)));
    if (b[i] >= g.nboxes[i] - 1) ok = false;
  }
  return ok;
}

// Writes every site (atom or ghost) of the batch and counts sites per box.
__global__ void nl_sites_kernel(int64_t n_atoms, const int64_t * __restrict__ atom_off,
                                const int32_t * __restrict__ atom_struct,
                                const int32_t * __restrict__ tag2idx,
                                const double * __restrict__ pos, const int32_t * __restrict__ types,
                                const NlGeom * __restrict__ geom,
                                const int64_t * __restrict__ ghost_off,
                                const int64_t * __restrict__ box_base, double cutoff,
                                double * __restrict__ site_x, int32_t * __restrict__ site_type,
                                int32_t * __restrict__ site_real, int32_t * __restrict__ site_shift,
                                int64_t * __restrict__ site_box, int32_t * __restrict__ box_count,
                                DevStatus * st, int64_t site_cap, int64_t box_cap) {
  int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n_atoms) return;
  int s = atom_struct[t];
  const NlGeom & g = geom[s];
  int64_t a0 = atom_off[s];
  int64_t gbase = ghost_off[a0];
  int64_t site_base = a0 + gbase;
  int64_t a = tag2idx ? tag2idx[t] : t;
  double x0[3] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
  int typ = types[a];
  auto put = [&](int64_t site, const double * x, const int * p) {
    if (site >= site_cap) {
      set_status(st, 104, s, int(a));  // more sites than the capacity
      return;
    }
    site_x[3 * site + 0] = x[0];
    site_x[3 * site + 1] = x[1];
    site_x[3 * site + 2] = x[2];
    site_type[site] = typ;
    site_real[site] = int32_t(a);
    site_shift[3 * site + 0] = p[0];
    site_shift[3 * site + 1] = p[1];
    site_shift[3 * site + 2] = p[2];
    int b[3];
    if (!box_of(g, x, cutoff, b)) set_status(st, 103, s, int(a));
    b[0] = min(b[0], g.nboxes[0] - 2);
    b[1] = min(b[1], g.nboxes[1] - 2);
    b[2] = min(b[2], g.nboxes[2] - 2);
    int64_t box = box_base[s] + (int64_t(b[0]) * g.nboxes[1] + b[1]) * g.nboxes[2] + b[2];
    if (box >= box_cap) {
      set_status(st, 104, s, int(a));  // more boxes than the capacity
      site_box[site] = -1;
      return;
    }
    site_box[site] = box;
    atomicAdd(&box_count[box], 1);
  };
  int zero[3] = {0, 0, 0};
  put(site_base + (t - a0), x0, zero);
  int ntot = g.reps[0] * g.reps[1] * g.reps[2];
  if (ntot > 1) {
    int64_t slot = site_base + g.n_atoms + (ghost_off[t] - gbase);
    for (int k = 0; k < ntot; ++k) {
      int p[3];
      image_of(g, k, p);
      if (p[0] == 0 && p[1] == 0 && p[2] == 0) continue;
      double gp[3];
      if (ghost_pos(g, x0, p, gp)) put(slot++, gp, p);
    }
  }
}

// n_sites bounds the grid; with ghosts_dev (the device total of ghost
// sites) the count is n_atoms + *ghosts_dev when that is smaller.
__device__ __forceinline__ int64_t site_count(int64_t n_sites, const int64_t * ghosts_dev, int64_t n_atoms) {
  if (!ghosts_dev) return n_sites;
  const int64_t n = n_atoms + *ghosts_dev;
  return n < n_sites ? n : n_sites;
}

__global__ void nl_scatter_kernel(int64_t n_sites, const int64_t * __restrict__ site_box,
                                  const int64_t * __restrict__ box_ptr,
                                  int32_t * __restrict__ box_fill, int64_t * __restrict__ sorted,
                                  const int64_t * __restrict__ ghosts_dev, int64_t n_atoms) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= site_count(n_sites, ghosts_dev, n_atoms)) return;
  int64_t b = site_box[i];
  if (b < 0) return;  // a site past the box capacity
  int64_t slot = box_ptr[b] + atomicAdd(&box_fill[b], 1);
  sorted[slot] = i;
}

// Ascending site (= tag) order inside every box, then pack positions.
__global__ void nl_boxsort_kernel(int64_t n_boxes, const int64_t * __restrict__ box_ptr,
                                  int64_t * __restrict__ sorted) {
  int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= n_boxes) return;  // boxes past the used ones (capacity mode) are empty
  int64_t lo = box_ptr[b], hi = box_ptr[b + 1];
  for (int64_t i = lo + 1; i < hi; ++i) {
    int64_t v = sorted[i];
    int64_t j = i - 1;
    while (j >= lo && sorted[j] > v) {
      sorted[j + 1] = sorted[j];
      --j;
    }
    sorted[j + 1] = v;
  }
}

__global__ void nl_pack_kernel(int64_t n_sites, const int64_t * __restrict__ sorted,
                               const double * __restrict__ site_x, double * __restrict__ sorted_x,
                               const int64_t * __restrict__ box_total) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  // the binned sites (box_ptr's total): all sites unless some overflowed
  if (i >= n_sites || (box_total && i >= *box_total)) return;
  int64_t s = sorted[i];
  sorted_x[3 * i + 0] = site_x[3 * s + 0];
  sorted_x[3 * i + 1] = site_x[3 * s + 1];
  sorted_x[3 * i + 2] = site_x[3 * s + 2];
}

struct GatherCtx {
  const int64_t * atom_off;
  const int64_t * center_off;
  const int32_t * center_struct_in;  // structure of each centre row
  const NlGeom * geom;
  const int64_t * ghost_off;
  const int64_t * box_base;
  const int64_t * box_ptr;
  const int64_t * sorted;
  const double * sorted_x;
  const double * site_x;
  double cutoff, rc2;
  int64_t box_cap, pair_cap;  // capacities (the exact counts when synchronised)
  DevStatus * status;
};

// One warp per centre. MODE 0 counts, MODE 1 writes the pairs.
template <int MODE>
__global__ void nl_gather_kernel(int64_t n_centers, GatherCtx c, int64_t * __restrict__ count,
                                 const int64_t * __restrict__ pair_off,
                                 const int32_t * __restrict__ site_type,
                                 const int32_t * __restrict__ site_real,
                                 const int32_t * __restrict__ site_shift,
                                 int32_t * __restrict__ center_atom,
                                 int32_t * __restrict__ pair_j, int32_t * __restrict__ pair_shift,
                                 double * __restrict__ pair_dist, double * __restrict__ pair_dir,
                                 int32_t * __restrict__ pair_center) {
  const int lane = threadIdx.x & 31;
  int64_t ci = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (ci >= n_centers) return;
  const int s = c.center_struct_in[ci];
  const NlGeom & g = c.geom[s];
  const int64_t a0 = c.atom_off[s];
  const int64_t site = a0 + c.ghost_off[a0] + (ci - c.center_off[s]);
  const double xi[3] = {c.site_x[3 * site], c.site_x[3 * site + 1], c.site_x[3 * site + 2]};
  int b[3];
  box_of(g, xi, c.cutoff, b);
  b[0] = min(b[0], g.nboxes[0] - 2);
  b[1] = min(b[1], g.nboxes[1] - 2);
  b[2] = min(b[2], g.nboxes[2] - 2);
  // a structure whose mesh reaches past the box capacity is skipped (capacity mode)
  if (c.box_base[s] + int64_t(g.nboxes[0]) * g.nboxes[1] * g.nboxes[2] > c.box_cap) {
    if (lane == 0) set_status(c.status, 104, s, 0);
    if (MODE == 0 && lane == 0) count[ci] = 1;
    return;
  }
  int64_t out = 0;
  int64_t base = 0;
  if (MODE == 1) {
    base = pair_off[ci];
    if (base + 1 + 0 > c.pair_cap) {  // not even the self pair fits
      if (lane == 0) set_status(c.status, 104, s, int(ci));
      return;
    }
    if (pair_off[ci + 1] > c.pair_cap && lane == 0) set_status(c.status, 104, s, int(ci));
    if (lane == 0) {
      center_atom[ci] = site_real[site];
      pair_j[base] = site_real[site];
      pair_shift[3 * base] = pair_shift[3 * base + 1] = pair_shift[3 * base + 2] = 0;
      pair_dist[base] = 0.;
      pair_dir[3 * base] = pair_dir[3 * base + 1] = pair_dir[3 * base + 2] = 0.;
    }
    base += 1;
  }
  // The stencil's 9 box rows (dx, dy; 3 boxes along z each) are runs of the
  // box-sorted sites; lanes 0..8 read one run's bounds each, all at once.
  int64_t run_lo = 0, run_len = 0;
  if (lane < 9) {
    const int dx = lane / 3, dy = lane - 3 * (lane / 3);
    const int64_t lin = (int64_t(b[0] + dx - 1) * g.nboxes[1] + (b[1] + dy - 1)) * g.nboxes[2] + (b[2] - 1);
    run_lo = c.box_ptr[c.box_base[s] + lin];
    run_len = c.box_ptr[c.box_base[s] + lin + 3] - run_lo;
  }
  // candidate k (valid: has one) of this lane: its pair, if within the
  // cutoff, takes the next slot in lane order
  auto visit = [&](bool valid, int64_t k) {
    bool ok = false;
    double v[3] = {0., 0., 0.};
    double d2 = 0.;
    int64_t sj = -1;
    if (valid) {
      sj = c.sorted[k];
      v[0] = c.sorted_x[3 * k + 0] - xi[0];
      v[1] = c.sorted_x[3 * k + 1] - xi[1];
      v[2] = c.sorted_x[3 * k + 2] - xi[2];
      d2 = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
      ok = (sj != site) && (d2 <= c.rc2);
    }
    unsigned m = __ballot_sync(0xffffffffu, ok);
    if (MODE == 1 && ok && base + out + __popc(m & lanemask_lt()) < c.pair_cap) {
      int64_t p = base + out + __popc(m & lanemask_lt());
      pair_j[p] = site_real[sj];
      pair_shift[3 * p + 0] = site_shift[3 * sj + 0];
      pair_shift[3 * p + 1] = site_shift[3 * sj + 1];
      pair_shift[3 * p + 2] = site_shift[3 * sj + 2];
      double dist = sqrt(d2);
      pair_dist[p] = dist;
      if (d2 > 0.) {
        pair_dir[3 * p + 0] = v[0] / dist;
        pair_dir[3 * p + 1] = v[1] / dist;
        pair_dir[3 * p + 2] = v[2] / dist;
      } else {
        pair_dir[3 * p + 0] = v[0];
        pair_dir[3 * p + 1] = v[1];
        pair_dir[3 * p + 2] = v[2];
      }
    }
    out += __popc(m);
  };
  int64_t run_end = run_len;  // inclusive scan of the run lengths over lanes 0..8
#pragma unroll
  for (int off = 1; off < 16; off <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, run_end, off);
    if (lane >= off) run_end += t;
  }
  const int64_t total = __shfl_sync(0xffffffffu, run_end, 8);
  if (total <= 32) {
    // one step over the 9 runs concatenated (same order as row by row), so
    // that no candidate load waits on another row's
    const int64_t run_start = run_end - run_len;
    int64_t k = 0;  // this lane's candidate in the sorted sites
#pragma unroll
    for (int r = 0; r < 9; ++r) {
      const int64_t st = __shfl_sync(0xffffffffu, run_start, r), en = __shfl_sync(0xffffffffu, run_end, r),
                    lo = __shfl_sync(0xffffffffu, run_lo, r);
      if (lane >= st && lane < en) k = lo + (lane - st);
    }
    visit(lane < total, k);
  } else {
    for (int r = 0; r < 9; ++r) {  // row by row, 32 candidates per step
      const int64_t lo = __shfl_sync(0xffffffffu, run_lo, r), hi = lo + __shfl_sync(0xffffffffu, run_len, r);
      for (int64_t k0 = lo; k0 < hi; k0 += 32) visit(k0 + lane < hi, k0 + lane);
    }
  }
  if (MODE == 0 && lane == 0) count[ci] = out + 1;
  if (MODE == 1)
    for (int64_t p = base - 1 + lane; p < base + out && p < c.pair_cap; p += 32) pair_center[p] = int32_t(ci);
  (void)site_type;
}

__global__ void center_struct_kernel(int n_struct, const int64_t * __restrict__ center_off,
                                     int32_t * __restrict__ center_struct) {
  // one block per structure
  int s = blockIdx.x;
  if (s >= n_struct) return;
  for (int64_t i = center_off[s] + threadIdx.x; i < center_off[s + 1]; i += blockDim.x)
    center_struct[i] = s;
}

// Capacity mode: offsets past the pair capacity are clamped to it, so that
// every later per-centre loop stays inside the pair buffers even when the
// list overflowed (status 104 then tells the caller to rebuild).
__global__ void nl_clamp_offsets_kernel(int64_t n, int64_t * __restrict__ pair_off, int64_t cap) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n && pair_off[i] > cap) pair_off[i] = cap;
}

}  // namespace

void neighbour_list_counts(const NlWork & w, int64_t & sites, int64_t & boxes) {
  sites = w.last_sites;
  boxes = w.last_boxes;
}

void build_neighbour_list(const NlInputs & in, double cutoff, NlWork & w, NlOutputs & out,
                          DevStatus * status_dev, DevStatus * status_host, cudaStream_t st,
                          const NlCaps * caps) {
  const int S = in.n_struct;
  const int64_t N = in.n_atoms;
  auto check_status = [&](const char * stage) {
    RGPU_CUDA(cudaMemcpyAsync(status_host, status_dev, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
    RGPU_CUDA(cudaStreamSynchronize(st));
    if (status_host->code != 0) {
      int code = status_host->code, where = status_host->where, detail = status_host->detail;
      RGPU_CUDA(cudaMemsetAsync(status_dev, 0, sizeof(DevStatus), st));
      RGPU_CUDA(cudaStreamSynchronize(st));
      char buf[512];
      switch (code) {
        case 100:
          std::snprintf(buf, sizeof buf,
                        "The unit cell should not be filled with zeros but it should contain all "
                        "the atoms even if the structure is not periodic. (structure %d)",
                        where);
          break;
        case 101:
          std::snprintf(buf, sizeof buf,
                        "atom types (or atomic numbers) should be in the range [0, 130]. "
                        "(structure %d, type %d)",
                        where, detail);
          break;
        case 102:
          std::snprintf(buf, sizeof buf,
                        "Some of the atoms in the structure are not inside the unit cell. Please "
                        "wrap them inside it with at least tolerance of 1e-10. (structure %d, "
                        "atom %d)",
                        where, detail);
          break;
        case 103:
          std::snprintf(buf, sizeof buf,
                        "Error: this atom does not fall in one of the linked cell bin. It might "
                        "have not been wrapped properly. (structure %d, atom %d)",
                        where, detail);
          break;
        default:
          std::snprintf(buf, sizeof buf, "neighbour list error %d at %s", code, stage);
      }
      throw Error(RGPU_ERR_STRUCTURE, buf);
    }
  };

  // 1. per-structure geometry and box counts
  w.geom.ensure(sizeof(NlGeom) * S);
  w.counts64.ensure(sizeof(int64_t) * (S + 1));
  w.box_base.ensure(sizeof(int64_t) * (S + 1));
  NlGeom * geom = w.geom.as<NlGeom>();
  nl_setup_kernel<<<div_up(S, 128), 128, 0, st>>>(S, in.atom_off, in.cells, in.pbc, in.n_centers,
                                                  cutoff, geom, w.counts64.as<int64_t>(), status_dev);
  RGPU_LAUNCHED();
  if (!caps) check_status("setup");
  nl_check_kernel<<<div_up(N, kThreads), kThreads, 0, st>>>(N, in.atom_struct, in.pos, in.types,
                                                            geom, status_dev);
  RGPU_LAUNCHED();
  scan_exclusive_i64(w.counts64.as<int64_t>(), w.box_base.as<int64_t>(), S, w.scan_tmp, st);

  // 2. ghost images
  w.pair_count.ensure(sizeof(int32_t) * (N + 1));
  w.ghost_off.ensure(sizeof(int64_t) * (N + 1));
  nl_ghost_count_kernel<<<div_up(N, kThreads), kThreads, 0, st>>>(
      N, in.atom_struct, in.tag2idx, in.pos, geom, w.pair_count.as<int32_t>());
  RGPU_LAUNCHED();
  scan_exclusive_i32to64(w.pair_count.as<int32_t>(), w.ghost_off.as<int64_t>(), N, w.scan_tmp, st);
  int64_t n_sites = 0, n_boxes = 0;
  if (caps) {
    // capacity mode: no host synchronisation; the kernels stop at the
    // capacities and the device counts bound the work
    n_sites = caps->sites;
    n_boxes = caps->boxes;
  } else {
    int64_t totals[2];
    RGPU_CUDA(cudaMemcpyAsync(&totals[0], w.ghost_off.as<int64_t>() + N, sizeof(int64_t),
                              cudaMemcpyDeviceToHost, st));
    RGPU_CUDA(cudaMemcpyAsync(&totals[1], w.box_base.as<int64_t>() + S, sizeof(int64_t),
                              cudaMemcpyDeviceToHost, st));
    check_status("check");
    n_sites = N + totals[0];
    n_boxes = totals[1];
    w.last_sites = n_sites;
    w.last_boxes = n_boxes;
  }
  const int64_t * ghosts_dev = caps ? w.ghost_off.as<int64_t>() + N : nullptr;

  // 3. sites and binning
  w.site_x.ensure(sizeof(double) * 3 * n_sites);
  w.site_type.ensure(sizeof(int32_t) * n_sites);
  w.site_real.ensure(sizeof(int32_t) * n_sites);
  w.site_shift.ensure(sizeof(int32_t) * 3 * n_sites);
  w.site_box.ensure(sizeof(int64_t) * n_sites);
  w.box_count.ensure(sizeof(int32_t) * (n_boxes + 1));
  w.box_fill.ensure(sizeof(int32_t) * (n_boxes + 1));
  w.box_ptr.ensure(sizeof(int64_t) * (n_boxes + 1));
  RGPU_CUDA(cudaMemsetAsync(w.box_count.p, 0, sizeof(int32_t) * (n_boxes + 1), st));
  RGPU_CUDA(cudaMemsetAsync(w.box_fill.p, 0, sizeof(int32_t) * (n_boxes + 1), st));
  nl_sites_kernel<<<div_up(N, kThreads), kThreads, 0, st>>>(
      N, in.atom_off, in.atom_struct, in.tag2idx, in.pos, in.types, geom, w.ghost_off.as<int64_t>(),
      w.box_base.as<int64_t>(), cutoff, w.site_x.as<double>(), w.site_type.as<int32_t>(),
      w.site_real.as<int32_t>(), w.site_shift.as<int32_t>(), w.site_box.as<int64_t>(),
      w.box_count.as<int32_t>(), status_dev, n_sites, n_boxes);
  RGPU_LAUNCHED();
  scan_exclusive_i32to64(w.box_count.as<int32_t>(), w.box_ptr.as<int64_t>(), n_boxes, w.scan_tmp, st);
  w.sorted.ensure(sizeof(int64_t) * n_sites);
  w.sorted_x.ensure(sizeof(double) * 3 * n_sites);
  nl_scatter_kernel<<<div_up(n_sites, kThreads), kThreads, 0, st>>>(
      n_sites, w.site_box.as<int64_t>(), w.box_ptr.as<int64_t>(), w.box_fill.as<int32_t>(),
      w.sorted.as<int64_t>(), ghosts_dev, N);
  RGPU_LAUNCHED();
  nl_boxsort_kernel<<<div_up(n_boxes, kThreads), kThreads, 0, st>>>(n_boxes, w.box_ptr.as<int64_t>(),
                                                                   w.sorted.as<int64_t>());
  RGPU_LAUNCHED();
  nl_pack_kernel<<<div_up(n_sites, kThreads), kThreads, 0, st>>>(
      n_sites, w.sorted.as<int64_t>(), w.site_x.as<double>(), w.sorted_x.as<double>(),
      caps ? w.box_ptr.as<int64_t>() + n_boxes : nullptr);
  RGPU_LAUNCHED();
  // The binning status (an atom outside every bin) is read with the pair
  // count below: the binning kernels clamp their box indices, so everything
  // up to there stays in bounds even when it is set.

  // 4. centres: structure of each centre row
  const int64_t n_centers = in.n_centers_total;
  w.center_struct.ensure(sizeof(int32_t) * (n_centers + 1));
  w.center_atom.ensure(sizeof(int32_t) * (n_centers + 1));
  center_struct_kernel<<<S, 128, 0, st>>>(S, in.center_off, w.center_struct.as<int32_t>());
  RGPU_LAUNCHED();

  // 5. count, scan, fill
  GatherCtx c;
  c.atom_off = in.atom_off;
  c.center_off = in.center_off;
  c.center_struct_in = w.center_struct.as<int32_t>();
  c.geom = geom;
  c.ghost_off = w.ghost_off.as<int64_t>();
  c.box_base = w.box_base.as<int64_t>();
  c.box_ptr = w.box_ptr.as<int64_t>();
  c.sorted = w.sorted.as<int64_t>();
  c.sorted_x = w.sorted_x.as<double>();
  c.site_x = w.site_x.as<double>();
  c.cutoff = cutoff;
  c.rc2 = cutoff * cutoff;
  c.box_cap = n_boxes;
  c.pair_cap = INT64_MAX;  // set below, once the pair count or capacity is known
  c.status = status_dev;
  w.counts64.ensure(sizeof(int64_t) * (n_centers + 1));
  w.pair_off.ensure(sizeof(int64_t) * (n_centers + 1));
  const int warps_per_block = kThreads / 32;
  int grid = div_up(n_centers, warps_per_block);
  if (n_centers > 0) {
    nl_gather_kernel<0><<<grid, kThreads, 0, st>>>(n_centers, c, w.counts64.as<int64_t>(), nullptr,
                                                   nullptr, nullptr, nullptr, nullptr, nullptr,
                                                   nullptr, nullptr, nullptr, nullptr);
    RGPU_LAUNCHED();
  }
  scan_exclusive_i64(w.counts64.as<int64_t>(), w.pair_off.as<int64_t>(), n_centers, w.scan_tmp, st);
  int64_t n_pairs = 0;
  if (caps) {
    n_pairs = caps->pairs;
  } else {
    RGPU_CUDA(cudaMemcpyAsync(&n_pairs, w.pair_off.as<int64_t>() + n_centers, sizeof(int64_t),
                              cudaMemcpyDeviceToHost, st));
    check_status("binning");  // synchronises: n_pairs is on the host after it
  }
  c.pair_cap = n_pairs;
  w.pair_j.ensure(sizeof(int32_t) * (n_pairs + 1));
  w.pair_shift.ensure(sizeof(int32_t) * 3 * (n_pairs + 1));
  w.pair_dist.ensure(sizeof(double) * (n_pairs + 1));
  w.pair_dir.ensure(sizeof(double) * 3 * (n_pairs + 1));
  w.pair_center.ensure(sizeof(int32_t) * (n_pairs + 1));
  if (n_centers > 0) {
    nl_gather_kernel<1><<<grid, kThreads, 0, st>>>(
        n_centers, c, nullptr, w.pair_off.as<int64_t>(), w.site_type.as<int32_t>(),
        w.site_real.as<int32_t>(), w.site_shift.as<int32_t>(), w.center_atom.as<int32_t>(),
        w.pair_j.as<int32_t>(), w.pair_shift.as<int32_t>(), w.pair_dist.as<double>(),
        w.pair_dir.as<double>(), w.pair_center.as<int32_t>());
    RGPU_LAUNCHED();
  }
  if (caps) {
    nl_clamp_offsets_kernel<<<div_up(n_centers + 1, kThreads), kThreads, 0, st>>>(
        n_centers + 1, w.pair_off.as<int64_t>(), n_pairs);
    RGPU_LAUNCHED();
  }
  out.n_centers = n_centers;
  out.n_pairs = n_pairs;
  out.center_atom = w.center_atom.as<int32_t>();
  out.center_struct = w.center_struct.as<int32_t>();
  out.pair_off = w.pair_off.as<int64_t>();
  out.pair_j = w.pair_j.as<int32_t>();
  out.pair_center = w.pair_center.as<int32_t>();
  out.pair_shift = w.pair_shift.as<int32_t>();
  out.pair_dist = w.pair_dist.as<double>();
  out.pair_dir = w.pair_dir.as<double>();
}

}  // namespace rgpu
