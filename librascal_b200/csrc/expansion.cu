// Spherical expansion of the neighbour density: coefficients and (plain path)
// their position gradients.
//
// c^i_{a n lm} = [a == type_i] center_n / sqrt(4 pi) delta_{lm,00}
//              + sum_{j != i, type_j = a} f_c(r_ij) RI_nl(r_ij) Y_lm(r^_ij)
// grad_j c^i   = (dRI f_c + RI df_c) Y dir + RI f_c / r grad Y
// grad_i c^i   = - sum_j grad_j c^i over j that are not images of i
// (src/rascal/representations/calculator_spherical_expansion.hh:2234-2366;
// the orthonormalised RI comes from the cubic spline, :1019-1156).
//
// Work decomposition: one warp per centre. Lanes first evaluate one pair each
// (spline row fetch, spherical harmonics by recurrence) into shared memory,
// then each lane owns output elements (n, lm) and accumulates the pairs of
// each neighbour species in turn.
#include <cuda_runtime.h>

#include "common.cuh"

namespace rgpu {
namespace {

constexpr int kWarps = 4;
constexpr int kPad = 33;  // shared row stride of the per-pair tiles
// The FP32 kernel takes pairs CH at a time (8, 16 or 32; 16 by default, as
// most centres of the molecular benchmark have fewer than 16 pairs, which
// keeps the per-warp tiles small and the resident warps many) with one
// centre per warp and up to kMaxWarpsF warps per block, both chosen per
// feature shape by the tile configuration.
constexpr int kMaxWarpsF = 8;

template <typename T>
struct Tab;
template <>
struct Tab<double> {
  static __device__ __forceinline__ const double * y(const SplineDev & s) { return s.y; }
  static __device__ __forceinline__ const double * d(const SplineDev & s) { return s.y2h; }
};
template <>
struct Tab<float> {
  static __device__ __forceinline__ const float * y(const SplineDev & s) { return s.yf; }
  static __device__ __forceinline__ const float * d(const SplineDev & s) { return s.y2hf; }
};

// cos(x) for x within 0.02 of pi, correctly rounded: -cos(pi - x) by its
// Taylor series in double-double (pi - x is exact by Sterbenz' lemma plus the
// low word of pi). The switching function needs it because 1 + cos(x)
// cancels there: an ulp of difference between two libm's cos becomes a
// relative error of ulp / f_c in f_c.
__device__ __forceinline__ double cos_near_pi(double x) {
  const double pi_hi = 3.141592653589793116, pi_lo = 1.2246467991473532e-16;
  double th = pi_hi - x;
  double s = th + pi_lo;
  double tl = pi_lo - (s - th);
  th = s;
  double u = th * th;
  double ue = fma(th, th, -u) + 2.0 * th * tl;
  double h = u * 0.5, hl = ue * 0.5;
  double c = 1.0 - h;
  double ce = ((1.0 - c) - h) - hl;
  double tail = u * u * (1.0 / 24.0) - u * u * u * (1.0 / 720.0) + u * u * u * u * (1.0 / 40320.0);
  return -(c + (ce + tail));
}

__device__ __forceinline__ double fc_cos(double r, double rc, double sw) {
  if (r <= (rc - sw)) return 1.0;
  if (r > rc) return 0.0;
  double rs = 3.14159265358979323846264338327950288 * (r - rc + sw) / sw;
  double c = (rs > 3.121592653589793) ? cos_near_pi(rs) : cos(rs);
  return 0.5 * (1. + c);
}
__device__ __forceinline__ double dfc_cos(double r, double rc, double sw) {
  if (r <= (rc - sw)) return 0.0;
  if (r > rc) return 0.0;
  double rs = 3.14159265358979323846264338327950288 * (r - rc + sw) / sw;
  return -0.5 * 3.14159265358979323846264338327950288 / sw * sin(rs);
}
// the cutoff function of the calculator: shifted cosine, times the
// RadialScaling factor when that is the cutoff type
__device__ __forceinline__ double cutoff_fc(const ExpansionArgs & a, double r) {
  const double s = fc_cos(r, a.rc, a.sw);
  return a.rs.on ? rs_value(a.rs, r) * s : s;
}
__device__ __forceinline__ void cutoff_fc_dfc(const ExpansionArgs & a, double r, double & fc, double & dfc) {
  const double s = fc_cos(r, a.rc, a.sw), ds = dfc_cos(r, a.rc, a.sw);
  if (a.rs.on) {
    const double u = rs_value(a.rs, r);
    fc = u * s;
    dfc = rs_grad(a.rs, r) * s + u * ds;
  } else {
    fc = s;
    dfc = ds;
  }
}

// Evaluate RI (and optionally dRI) of all W channels at r into smem columns.
template <typename T, bool DER>
__device__ __forceinline__ void spline_eval(const SplineDev & sp, double r, T * RI, T * dRI,
                                            int stride) {
  SplinePos q = spline_pos(sp, r);
  const T a = T(q.a), b = T(q.b);
  const T * y0 = Tab<T>::y(sp) + size_t(q.k) * sp.W;
  const T * d0 = Tab<T>::d(sp) + size_t(q.k) * sp.W;
  const T * y1 = y0 + sp.W;
  const T * d1 = d0 + sp.W;
  const T ca = a * a - T(1), cb = b * b - T(1);
  const T ea = T(3) * a * a - T(1), eb = T(3) * b * b - T(1);
  const T ih = T(sp.inv_h);
  for (int c = 0; c < sp.W; ++c) {
    T yy0 = __ldg(y0 + c), yy1 = __ldg(y1 + c), dd0 = __ldg(d0 + c), dd1 = __ldg(d1 + c);
    RI[c * stride] = a * (yy0 + ca * dd0) + b * (yy1 + cb * dd1);
    if (DER) {
      if (sizeof(T) == 8)
        dRI[c * stride] = (yy1 - yy0 - ea * dd0 + eb * dd1) / T(sp.h);
      else
        dRI[c * stride] = (yy1 - yy0 - ea * dd0 + eb * dd1) * ih;
    }
  }
}

template <typename T, int L>
__global__ void __launch_bounds__(kWarps * 32)
expansion_kernel(ExpansionArgs a, T * __restrict__ C, uint32_t * __restrict__ present) {
  constexpr int K = (L + 1) * (L + 1);
  constexpr int L1 = L + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int W = a.fd.W, nK = a.fd.nK, S = a.fd.S, n = a.fd.n;
  // per-pair values in columns of a row-major [item][kPad] tile: the
  // accumulation reads one pair column across many rows, so the row stride
  // is 33 words to keep those reads on distinct banks
  T * RI = reinterpret_cast<T *>(smem_raw) + size_t(wid) * (W + K + 1) * kPad;
  T * Y = RI + W * kPad;
  T * FC = Y + K * kPad;
  __shared__ int8_t sp_s[kWarps][32];
  __shared__ uint8_t order_s[kWarps][32];
  __shared__ uint8_t lofk[K];
  for (int lm = threadIdx.x; lm < K; lm += blockDim.x) {
    int l = 0;
    while ((l + 1) * (l + 1) <= lm) ++l;
    lofk[lm] = uint8_t(l);
  }
  __syncthreads();
  const int nw = blockDim.x >> 5;  // warps per block (fewer than kWarps for large W + K)
  for (int64_t ci = int64_t(blockIdx.x) * nw + wid; ci < a.n_centers; ci += int64_t(gridDim.x) * nw) {
    T * Ci = C + size_t(ci) * S * nK;
    for (int e = lane; e < S * nK; e += 32) Ci[e] = T(0);
    __syncwarp();
    const int64_t p_lo = a.pair_off[ci] + 1, p_hi = a.pair_off[ci + 1];
    const int ti = a.species_lut[a.types[a.center_atom[ci]]];
    uint32_t mask_all = 1u << ti;
    // centre contribution first, as the reference accumulates
    // (calculator_spherical_expansion.hh:2244-2247)
    for (int nn = lane; nn < n; nn += 32) Ci[size_t(ti) * nK + nn * K] = T(a.center_contrib[nn]);
    __syncwarp();
    for (int64_t p0 = p_lo; p0 < p_hi; p0 += 32) {
      const int np = int(min(int64_t(32), p_hi - p0));
      int my_sp = 31;
      if (lane < np) {
        const int64_t p = p0 + lane;
        const double r = a.pair_dist[p];
        my_sp = a.species_lut[a.types[a.pair_j[p]]];
        FC[lane] = T(cutoff_fc(a, r));
        spline_eval<T, false>(a.sp, r, RI + lane, nullptr, kPad);
        const T dx = T(a.pair_dir[3 * p]), dy = T(a.pair_dir[3 * p + 1]),
                dz = T(a.pair_dir[3 * p + 2]);
        spherical_harmonics<L, false, T>(dx, dy, dz, [&](int lm, T y, T, T, T) {
          Y[lm * kPad + lane] = y;
        });
      }
      // stable order of the chunk's pairs by species
      int before = 0, cnt_sp[kMaxSpecies];
      unsigned my_mask = 0;
      for (int s = 0; s < S; ++s) {
        unsigned m = __ballot_sync(0xffffffffu, my_sp == s);
        cnt_sp[s] = __popc(m);
        if (my_sp == s) my_mask = m;
        if (s < my_sp) before += __popc(m);
        if (m) mask_all |= 1u << s;
      }
      if (lane < np) {
        order_s[wid][before + __popc(my_mask & lanemask_lt())] = uint8_t(lane);
        sp_s[wid][lane] = int8_t(my_sp);
      }
      __syncwarp();
      int start = 0;
      for (int s = 0; s < S; ++s) {
        const int cnt = cnt_sp[s];
        if (cnt == 0) continue;
        T * Cs = Ci + size_t(s) * nK;
        for (int e = lane; e < nK; e += 32) {
          const int nn = e / K, lm = e - nn * K;
          const int l = lofk[lm];
          const T * ri = RI + (nn * L1 + l) * kPad;
          const T * yy = Y + lm * kPad;
          T acc = Cs[e];  // pairs added in neighbour-list order
          for (int q = 0; q < cnt; ++q) {
            const int pl = order_s[wid][start + q];
            acc += (ri[pl] * yy[pl]) * FC[pl];
          }
          Cs[e] = acc;
        }
        start += cnt;
      }
      __syncwarp();
    }
    if (lane == 0) present[ci] = mask_all;
    __syncwarp();
  }
}


#ifndef RGPU_PART_FP64
// FP32 fast path. The same sums, organised for throughput instead of the
// reference's accumulation order (the FP64 kernel above keeps that order):
//   (a) lanes = pairs: f_c, the spline interval and Y_lm of one pair each;
//   (b) lanes = radial channels: f_c RI_c(r_p) for the chunk's pairs one
//       after the other, one 16-byte load of the interval table per channel;
//   (c) lanes = (l, four columns m of the padded l-block, four radial
//       channels): 16 accumulators per lane; per pair of a species one
//       16-byte load of Y and four loads of f_c RI feed 16 products; the
//       sums are written once, as 16-byte stores, into the padded row
//       layout [S*n][row_stride(L)] (Y is zero in the padding columns, so
//       the padding of every l-block is written as zero).
template <int L, int CH>
__global__ void __launch_bounds__(kMaxWarpsF * 32)
expansion_f32_kernel(ExpansionArgs a, float * __restrict__ C, uint32_t * __restrict__ present) {
  constexpr int K = (L + 1) * (L + 1);
  constexpr int L1 = L + 1;
  constexpr int RS = row_stride(L), OL = offp(L + 1), NG = OL / 4;
  constexpr int kChunkF = CH, kPadF = CH + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;  // centres per block
  const int W = a.fd.W, S = a.fd.S, n = a.fd.n;
  const int wpad = (W * kPadF + 3) & ~3;  // keeps Yp 16-byte aligned
  float * RIf = reinterpret_cast<float *>(smem_raw) + size_t(wid) * (wpad + CH * RS);  // [W][kPadF]
  float * Yp = RIf + wpad;  // [CH][RS]: Y_lm of each pair in the padded column layout
  __shared__ float pa_s[kMaxWarpsF][32], pb_s[kMaxWarpsF][32], fc_s[kMaxWarpsF][32];
  __shared__ int pk_s[kMaxWarpsF][32];
  __shared__ uint8_t order_s[kMaxWarpsF][32];
  __shared__ int16_t colk[K];  // padded column of lm: offp(l) + m
  __shared__ uint8_t grp_l[NG];
  for (int lm = threadIdx.x; lm < K; lm += blockDim.x) {
    int l = 0;
    while ((l + 1) * (l + 1) <= lm) ++l;
    colk[lm] = int16_t(offp_rt(l) + (lm - l * l));
  }
  for (int g = threadIdx.x; g < NG; g += blockDim.x) {
    int l = 0;
    while (4 * g >= offp_rt(l + 1)) ++l;
    grp_l[g] = uint8_t(l);
  }
  for (int e = lane; e < CH * RS; e += 32) Yp[e] = 0.f;  // padding columns stay zero
  __syncthreads();
  const int nblk = (n + 3) >> 2;  // blocks of four radial channels
  for (int64_t ci = int64_t(blockIdx.x) * nw + wid; ci < a.n_centers; ci += int64_t(gridDim.x) * nw) {
    float * Ci = C + size_t(ci) * S * n * RS;
    const int64_t p_lo = a.pair_off[ci] + 1, p_hi = a.pair_off[ci + 1];
    const int ti = a.species_lut[a.types[a.center_atom[ci]]];
    uint32_t mask_all = 1u << ti;
    // the columns after the last l-block
    for (int j = lane; j < S * n * (RS - OL); j += 32) {
      const int row = j / (RS - OL), c = OL + (j - row * (RS - OL));
      Ci[row * RS + c] = 0.f;
    }
    bool first = true;
    for (int64_t p0 = p_lo; p0 < p_hi || first; p0 += kChunkF) {
      const int np = int(max(int64_t(0), min(int64_t(kChunkF), p_hi - p0)));
      int my_sp = 31;
      if (lane < np) {
        const int64_t p = p0 + lane;
        const double r = a.pair_dist[p];
        my_sp = a.species_lut[a.types[a.pair_j[p]]];
        const SplinePos q = spline_pos(a.sp, r);
        pk_s[wid][lane] = q.k;
        pa_s[wid][lane] = float(q.a);
        pb_s[wid][lane] = float(q.b);
        fc_s[wid][lane] = float(cutoff_fc(a, r));
        const float dx = float(a.pair_dir[3 * p]), dy = float(a.pair_dir[3 * p + 1]),
                    dz = float(a.pair_dir[3 * p + 2]);
        float * yrow = Yp + lane * RS;
        spherical_harmonics<L, false, float>(dx, dy, dz, [&](int lm, float y, float, float, float) {
          yrow[colk[lm]] = y;
        });
      }
      // stable order of the chunk's pairs by species
      int before = 0;
      unsigned my_mask = 0;
      for (int s = 0; s < S; ++s) {
        unsigned m = __ballot_sync(0xffffffffu, my_sp == s);
        if (my_sp == s) my_mask = m;
        if (s < my_sp) before += __popc(m);
        if (m) mask_all |= 1u << s;
      }
      if (lane < np) order_s[wid][before + __popc(my_mask & lanemask_lt())] = uint8_t(lane);
      __syncwarp();
      // lanes = radial channels c and c + 32 (then c + 64, ... when W is
      // larger); four pairs per step, so that their table loads are in
      // flight together
      const bool c1_ok = lane + 32 < W, c0_ok = lane < W;
#pragma unroll 4
      for (int q = 0; q < np; ++q) {
        const float fa = pa_s[wid][q], fb = pb_s[wid][q], f = fc_s[wid][q];
        const float ca = fa * fa - 1.f, cb = fb * fb - 1.f;
        const float4 * row = a.sp.q4f + size_t(pk_s[wid][q]) * W;
        if (c0_ok) {
          const float4 t = __ldg(row + lane);
          RIf[lane * kPadF + q] = f * (fa * (t.x + ca * t.y) + fb * (t.z + cb * t.w));
        }
        if (c1_ok) {
          const float4 t = __ldg(row + lane + 32);
          RIf[(lane + 32) * kPadF + q] = f * (fa * (t.x + ca * t.y) + fb * (t.z + cb * t.w));
        }
        for (int c = lane + 64; c < W; c += 32) {
          const float4 t = __ldg(row + c);
          RIf[c * kPadF + q] = f * (fa * (t.x + ca * t.y) + fb * (t.z + cb * t.w));
        }
      }
      __syncwarp();
      int start = 0;
      for (int s = 0; s < S; ++s) {
        const int cnt = __popc(__ballot_sync(0xffffffffu, my_sp == s));
        if (cnt > 0 || first) {
          float * Cs = Ci + size_t(s) * n * RS;
          for (int t = lane; t < NG * nblk; t += 32) {
            const int g = t % NG, n0 = 4 * (t / NG);
            const int l = grp_l[g], col = 4 * g;
            const float * ri = RIf + (n0 * L1 + l) * kPadF;  // channel (n0 + k) L1 + l at + k L1 kPadF
            float acc[4][4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
              for (int e = 0; e < 4; ++e) acc[k][e] = 0.f;
            for (int q = 0; q < cnt; ++q) {
              const int pl = order_s[wid][start + q];
              const float4 y = *reinterpret_cast<const float4 *>(Yp + pl * RS + col);
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                if (n0 + k < n) {
                  const float rv = ri[k * L1 * kPadF + pl];
                  acc[k][0] += rv * y.x;
                  acc[k][1] += rv * y.y;
                  acc[k][2] += rv * y.z;
                  acc[k][3] += rv * y.w;
                }
              }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const int nn = n0 + k;
              if (nn < n) {
                float4 * dst = reinterpret_cast<float4 *>(Cs + nn * RS + col);
                if (first) {
                  // centre contribution (calculator_spherical_expansion.hh:2244-2247)
                  if (s == ti && col == 0) acc[k][0] += float(a.center_contrib[nn]);
                  *dst = make_float4(acc[k][0], acc[k][1], acc[k][2], acc[k][3]);
                } else {
                  float4 o = *dst;
                  o.x += acc[k][0];
                  o.y += acc[k][1];
                  o.z += acc[k][2];
                  o.w += acc[k][3];
                  *dst = o;
                }
              }
            }
          }
        }
        start += cnt;
      }
      __syncwarp();
      first = false;
    }
    if (lane == 0) present[ci] = mask_all;
    __syncwarp();
  }
}
#endif

// Plain path: grad_j c^i for every non-self pair of centres [c0, c1); each
// lane streams its pair's 3 x n x K block.
template <int L>
__global__ void __launch_bounds__(kWarps * 32)
expansion_grad_kernel(ExpansionArgs a, int64_t c0, int64_t c1, int64_t p_base,
                      double * __restrict__ dCp) {
  constexpr int K = (L + 1) * (L + 1);
  constexpr int L1 = L + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int W = a.fd.W, n = a.fd.n, nK = a.fd.nK;
  double * RI = reinterpret_cast<double *>(smem_raw) + size_t(wid) * 2 * W * 32;
  double * P1 = RI + W * 32;
  const int nw = blockDim.x >> 5;  // warps per block (fewer than kWarps for large W)
  for (int64_t ci = c0 + int64_t(blockIdx.x) * nw + wid; ci < c1; ci += int64_t(gridDim.x) * nw) {
    const int64_t p_lo = a.pair_off[ci] + 1, p_hi = a.pair_off[ci + 1];
    for (int64_t p = p_lo + lane; p < p_hi; p += 32) {
      const double r = a.pair_dist[p];
      double fc, dfc;
      cutoff_fc_dfc(a, r, fc, dfc);
      spline_eval<double, true>(a.sp, r, RI + lane, P1 + lane, 32);
      for (int c = 0; c < W; ++c) {
        // p1 = dRI f_c + RI df_c
        P1[c * 32 + lane] = (P1[c * 32 + lane] * fc) + (RI[c * 32 + lane] * dfc);
      }
      const double dir[3] = {a.pair_dir[3 * p], a.pair_dir[3 * p + 1], a.pair_dir[3 * p + 2]};
      double * out = dCp + size_t(p - p_base) * 3 * nK;
      spherical_harmonics<L, true, double>(dir[0], dir[1], dir[2],
                                           [&](int lm, double y, double gx, double gy, double gz) {
        int l = 0;
#pragma unroll
        for (int ll = 1; ll <= L; ++ll) l += (lm >= ll * ll);
        const double g[3] = {gx, gy, gz};
        for (int nn = 0; nn < n; ++nn) {
          const double p1 = P1[(nn * L1 + l) * 32 + lane];
          const double ri = RI[(nn * L1 + l) * 32 + lane];
#pragma unroll
          for (int cc = 0; cc < 3; ++cc)
            out[cc * nK + nn * K + lm] = (p1 * y) * dir[cc] + ((ri * g[cc]) * fc) / r;
        }
      });
    }
  }
}

// Plain path: grad_i c^i = - sum over non-image neighbours, per species block.
__global__ void expansion_selfgrad_kernel(ExpansionArgs a, int64_t c0, int64_t p_base,
                                          const double * __restrict__ dCp,
                                          double * __restrict__ dCs) {
  const int64_t ci = c0 + blockIdx.x;
  const int nK3 = 3 * a.fd.nK, S = a.fd.S;
  const int64_t p_lo = a.pair_off[ci] + 1, p_hi = a.pair_off[ci + 1];
  const int32_t self_atom = a.center_atom[ci];
  double * out = dCs + size_t(blockIdx.x) * S * nK3;
  for (int s = 0; s < S; ++s) {
    for (int e = threadIdx.x; e < nK3; e += blockDim.x) {
      double acc = 0.;
      for (int64_t p = p_lo; p < p_hi; ++p) {
        const int32_t j = a.pair_j[p];
        if (j == self_atom) continue;  // periodic image of the centre
        if (a.species_lut[a.types[j]] != s) continue;
        acc -= dCp[size_t(p - p_base) * nK3 + e];
      }
      out[size_t(s) * nK3 + e] = acc;
    }
  }
}

// Warps per block of a kernel whose warps each need `per_warp` bytes of
// shared memory: kWarps, or as many as the device's per-block limit allows
// (the FP64 tiles of large n (l+1) + (l+1)^2 do not fit four times).
int warps_for(size_t per_warp, const char * what) {
  int dev = 0, optin = 0;
  RGPU_CUDA(cudaGetDevice(&dev));
  RGPU_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const int w = int(std::min<size_t>(kWarps, size_t(optin) / per_warp));
  if (w < 1)
    throw Error(RGPU_ERR_INVALID_ARGUMENT, std::string(what) + ": max_radial x (max_angular + 1) too large for "
                                                               "shared memory");
  return w;
}

template <typename T>
size_t exp_smem_per_warp(const FeatureDims & fd) {
  return size_t(fd.W + fd.K + 1) * kPad * sizeof(T);
}

template <typename T>
void launch_exp(const ExpansionArgs & a, T * C, uint32_t * present, cudaStream_t st) {
  if (a.n_centers == 0) return;
  sph_constants_tu();
  const int warps = warps_for(exp_smem_per_warp<T>(a.fd), "spherical expansion");
  const size_t smem = size_t(warps) * exp_smem_per_warp<T>(a.fd);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int grid = int(std::min<int64_t>((a.n_centers + warps - 1) / warps, int64_t(sms) * 16));
#define RGPU_EXP_CASE(LL)                                                                   \
  case LL:                                                                                  \
    RGPU_CUDA(cudaFuncSetAttribute(expansion_kernel<T, LL>,                                 \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))); \
    expansion_kernel<T, LL><<<grid, warps * 32, smem, st>>>(a, C, present);                 \
    break;
  switch (a.fd.L) {
    RGPU_EXP_CASE(0)
    RGPU_EXP_CASE(1)
    RGPU_EXP_CASE(2)
    RGPU_EXP_CASE(3)
    RGPU_EXP_CASE(4)
    RGPU_EXP_CASE(5)
    RGPU_EXP_CASE(6)
    RGPU_EXP_CASE(7)
    RGPU_EXP_CASE(8)
    RGPU_EXP_CASE(9)
    RGPU_EXP_CASE(10)
    RGPU_EXP_CASE(11)
    RGPU_EXP_CASE(12)
    default:
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_angular above 12 is not supported on the GPU");
  }
#undef RGPU_EXP_CASE
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

#ifndef RGPU_PART_FP64
void launch_exp_f32(const ExpansionArgs & a, float * C, uint32_t * present, cudaStream_t st) {
  if (a.n_centers == 0) return;
  if (a.fd.n > 16) throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_radial above 16 is not supported on the fast path");
  sph_constants_tu();
  const TileConfig cfg = tile_config(a.fd.S, a.fd.n, a.fd.L);
  const int CH = cfg.exp_chunk;
  int dev = 0, sms = 148, optin = 0;
  RGPU_CUDA(cudaGetDevice(&dev));
  RGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RGPU_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t per_warp =
      ((size_t(a.fd.W) * (CH + 1) + 3) / 4 * 4 + size_t(CH) * row_stride(a.fd.L)) * sizeof(float);
  const int warps = int(std::max<size_t>(1, std::min<size_t>(size_t(cfg.exp_warps), (size_t(optin) - 8192) / per_warp)));
  const size_t smem = size_t(warps) * per_warp;
  int grid = int(std::min<int64_t>((a.n_centers + warps - 1) / warps, int64_t(sms) * 16 * (4 / std::min(warps, 4))));
#define RGPU_EXPF_NV(LL, CHH)                                                                       \
  {                                                                                                 \
    RGPU_CUDA(cudaFuncSetAttribute(expansion_f32_kernel<LL, CHH>,                                   \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));        \
    expansion_f32_kernel<LL, CHH><<<grid, warps * 32, smem, st>>>(a, C, present);                   \
  }
#define RGPU_EXP_CASE(LL)              \
  case LL:                             \
    if (CH == 8) {                     \
      RGPU_EXPF_NV(LL, 8)              \
    } else if (CH == 32) {             \
      RGPU_EXPF_NV(LL, 32)             \
    } else {                           \
      RGPU_EXPF_NV(LL, 16)             \
    }                                  \
    break;
  switch (a.fd.L) {
    RGPU_EXP_CASE(0)
    RGPU_EXP_CASE(1)
    RGPU_EXP_CASE(2)
    RGPU_EXP_CASE(3)
    RGPU_EXP_CASE(4)
    RGPU_EXP_CASE(5)
    RGPU_EXP_CASE(6)
    RGPU_EXP_CASE(7)
    RGPU_EXP_CASE(8)
    RGPU_EXP_CASE(9)
    RGPU_EXP_CASE(10)
    RGPU_EXP_CASE(11)
    RGPU_EXP_CASE(12)
    default:
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_angular above 12 is not supported on the GPU");
  }
#undef RGPU_EXP_CASE
#undef RGPU_EXPF_NV
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}
#endif

}  // namespace

// The library compiles this file twice: RGPU_PART_FP64 (with --fmad=false, so
// the FP64 arithmetic rounds like the CPU restatement) and RGPU_PART_FP32.
#ifndef RGPU_PART_FP32
void launch_expansion_fp64(const ExpansionArgs & a, double * C, uint32_t * present,
                           cudaStream_t st) {
  launch_exp<double>(a, C, present, st);
}
#endif
#ifndef RGPU_PART_FP64
void launch_expansion_fp32(const ExpansionArgs & a, float * C, uint32_t * present,
                           cudaStream_t st) {
  launch_exp_f32(a, C, present, st);
}
#endif

#ifndef RGPU_PART_FP32
void launch_expansion_grad_fp64(const ExpansionArgs & a, int64_t c0, int64_t c1, int64_t p_base,
                                double * dCp, cudaStream_t st) {
  if (c1 <= c0) return;
  sph_constants_tu();
  const size_t per_warp = size_t(2) * a.fd.W * 32 * sizeof(double);
  const int warps = warps_for(per_warp, "spherical expansion gradients");
  const size_t smem = size_t(warps) * per_warp;
  int grid = int(std::min<int64_t>((c1 - c0 + warps - 1) / warps, 148 * 16));
#define RGPU_GRAD_CASE(LL)                                                                  \
  case LL:                                                                                  \
    RGPU_CUDA(cudaFuncSetAttribute(expansion_grad_kernel<LL>,                               \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))); \
    expansion_grad_kernel<LL><<<grid, warps * 32, smem, st>>>(a, c0, c1, p_base, dCp);      \
    break;
  switch (a.fd.L) {
    RGPU_GRAD_CASE(0)
    RGPU_GRAD_CASE(1)
    RGPU_GRAD_CASE(2)
    RGPU_GRAD_CASE(3)
    RGPU_GRAD_CASE(4)
    RGPU_GRAD_CASE(5)
    RGPU_GRAD_CASE(6)
    RGPU_GRAD_CASE(7)
    RGPU_GRAD_CASE(8)
    RGPU_GRAD_CASE(9)
    RGPU_GRAD_CASE(10)
    RGPU_GRAD_CASE(11)
    RGPU_GRAD_CASE(12)
    default:
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_angular above 12 is not supported on the GPU");
  }
#undef RGPU_GRAD_CASE
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}

void launch_expansion_selfgrad_fp64(const ExpansionArgs & a, int64_t c0, int64_t c1,
                                    int64_t p_base, const double * dCp, double * dCs,
                                    cudaStream_t st) {
  if (c1 <= c0) return;
  expansion_selfgrad_kernel<<<int(c1 - c0), 256, 0, st>>>(a, c0, p_base, dCp, dCs);
  RGPU_LAUNCHED();
  RGPU_CUDA(cudaGetLastError());
}
#endif

}  // namespace rgpu
