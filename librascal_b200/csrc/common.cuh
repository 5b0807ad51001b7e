// Device helpers shared by the kernel files.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rgpu_internal.h"

namespace rgpu {

constexpr int kMaxL = 12;        // largest max_angular the GPU kernels support
constexpr int kMaxSpecies = 16;  // largest species count of a dense layout

__device__ __forceinline__ void set_status(DevStatus * st, int code, int where, int detail) {
  if (atomicCAS(&st->code, 0, code) == 0) {
    st->where = where;
    st->detail = detail;
  }
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

inline int div_up(int64_t a, int64_t b) { return int((a + b - 1) / b); }

// Radial factor u(r) of the RadialScaling cutoff and its derivative
// (representations/cutoff_functions.hh:178-280): c / (c + (r/r0)^m), or
// (r/r0)^-m when c is zero (|c| <= 100 eps, the reference's test), or 1 when
// m is zero. It multiplies the shifted cosine; the products below follow the
// reference's order: f_c = u * s, df_c = u' * s + u * s'.
__device__ __forceinline__ double rs_value(const RadialScalingDev & p, double r) {
  if (fabs(p.rate) <= 100.0 * 2.220446049250313e-16) return 1.0 / pow(r / p.scale, p.exponent);
  if (p.exponent == 0.0) return 1.0;
  return p.rate / (p.rate + pow(r / p.scale, p.exponent));
}
__device__ __forceinline__ double rs_grad(const RadialScalingDev & p, double r) {
  if (fabs(p.rate) <= 100.0 * 2.220446049250313e-16) return -p.exponent / r / pow(r / p.scale, p.exponent);
  if (p.exponent == 0.0) return 0.0;
  const double ff = pow(r / p.scale, p.exponent);
  const double d = p.rate + ff;
  return -p.rate * p.exponent * ff / r / (d * d);
}

// v^zeta of the GAP kernel (models/kernels.hh:48-61)
__device__ __forceinline__ double pow_zeta_d(double v, int z) {
  if (z == 0) return 1.;
  if (z == 1) return v;
  if (z == 2) return v * v;
  if (z == 3) return v * v * v;
  double r = 1., x = v;
  int n = z;
  do {
    if (n & 1) r *= x;
    n >>= 1;
    x *= x;
  } while (n);
  return r;
}

// Spherical-harmonics constants per (l, m), double and float copies:
// coeff_a, coeff_b (math/spherical_harmonics.cc:54-64), sqrt(2l+1) and
// -sqrt(1 + 1/(2l)) (:67-71), and the ladder factors sqrt((l-m)(l+m+1))
// (:86-91). Index l*(kMaxL+2)+m.
struct SphConst {
  double a[(kMaxL + 1) * (kMaxL + 2)];
  double b[(kMaxL + 1) * (kMaxL + 2)];
  double plm[(kMaxL + 1) * (kMaxL + 2)];
  double c1[kMaxL + 1];
  double c2[kMaxL + 1];
  float af[(kMaxL + 1) * (kMaxL + 2)];
  float bf[(kMaxL + 1) * (kMaxL + 2)];
  float plmf[(kMaxL + 1) * (kMaxL + 2)];
  float c1f[kMaxL + 1];
  float c2f[kMaxL + 1];
};
// Each translation unit that evaluates spherical harmonics holds its own copy
// (no relocatable device code), and every device has its own instance of
// it: sph_constants_tu() fills the current device's copy the first time a
// kernel of this translation unit is launched there.
static __constant__ SphConst c_sph;
SphConst make_sph_constants();
static PerDevice<char> g_sph_filled;
static inline void sph_constants_tu() {
  g_sph_filled.once(current_device(), [](char &) {
    SphConst h = make_sph_constants();
    cuda_check(cudaMemcpyToSymbol(c_sph, &h, sizeof(h)), "cudaMemcpyToSymbol(c_sph)");
  });
}

template <typename T>
struct SphC;
template <>
struct SphC<double> {
  static __device__ __forceinline__ double a(int i) { return c_sph.a[i]; }
  static __device__ __forceinline__ double b(int i) { return c_sph.b[i]; }
  static __device__ __forceinline__ double plm(int i) { return c_sph.plm[i]; }
  static __device__ __forceinline__ double c1(int l) { return c_sph.c1[l]; }
  static __device__ __forceinline__ double c2(int l) { return c_sph.c2[l]; }
};
template <>
struct SphC<float> {
  static __device__ __forceinline__ float a(int i) { return c_sph.af[i]; }
  static __device__ __forceinline__ float b(int i) { return c_sph.bf[i]; }
  static __device__ __forceinline__ float plm(int i) { return c_sph.plmf[i]; }
  static __device__ __forceinline__ float c1(int l) { return c_sph.c1f[l]; }
  static __device__ __forceinline__ float c2(int l) { return c_sph.c2f[l]; }
};

// Real spherical harmonics of a unit vector and (optionally) their Cartesian
// gradients, following math/spherical_harmonics.cc:97-363: associated
// Legendre functions by the l-recurrence, cos/sin(m phi) by the Chebyshev
// recurrence, storage order (l, m = -l..l), pole branch at sin(theta) <= 0.1.
// The callback receives (lm, Y, dY/dx, dY/dy, dY/dz) for every lm in order.
struct NoBeginL {
  __device__ __forceinline__ void operator()(int) const {}
};

// `begin_l(l)` runs before the first emit of every l (compile-time l after
// unrolling), so a caller can stage per-l data in registers.
template <int L, bool DER, typename T, typename Emit, typename BeginL = NoBeginL>
__device__ __forceinline__ void spherical_harmonics(T x, T y, T z, Emit && emit, BeginL && begin_l = BeginL()) {
  constexpr int S = kMaxL + 2;
  const T nrm2 = x * x + y * y + z * z;
  if (fabs(double(nrm2) - 1.0) > (sizeof(T) == 8 ? 100.0 * 2.220446049250313e-16 : 1e-5)) {
    T inv = T(1) / sqrt(nrm2);
    x *= inv;
    y *= inv;
    z *= inv;
  }
  const T cos_t = z;
  const T sxy = hypot(x, y);
  T cos_p = T(1), sin_p = T(0);
  if (sxy >= T(100.0 * 2.220446049250313e-16)) {
    cos_p = x / sxy;
    sin_p = y / sxy;
  }
  const T sin_t = sqrt(T(1) - cos_t * cos_t);
  const T sin_td = sxy;  // sin(theta) used by the derivative formulas
  T cm[L + 2], sm[L + 2];
#pragma unroll
  for (int m = 0; m < L + 2; ++m) {
    if (m == 0) {
      cm[0] = T(1);
      sm[0] = T(0);
    } else if (m == 1) {
      cm[1] = cos_p;
      sm[1] = sin_p;
    } else {
      cm[m] = T(2) * cos_p * cm[m - 1] - cm[m - 2];
      sm[m] = T(2) * cos_p * sm[m - 1] - sm[m - 2];
    }
  }
  const T inv_sqrt2 = T(0.707106781186547524400844362104849039);
  const T sqrt_inv_2pi = T(0.398942280401432677939946059934381868);  // sqrt(1/(2 pi))
  T p2[L + 2], p1[L + 2], p0[L + 2];  // rows l-2, l-1, l
#pragma unroll
  for (int m = 0; m < L + 2; ++m) p2[m] = p1[m] = p0[m] = T(0);
  T l_accum = sqrt_inv_2pi;
#pragma unroll
  for (int l = 0; l <= L; ++l) {
    if (l == 0) {
      p0[0] = sqrt_inv_2pi;
    } else if (l == 1) {
      p0[0] = cos_t * T(1.7320508075688772935274463415058723) * sqrt_inv_2pi;
      l_accum = l_accum * -T(1.2247448713915890491) * sin_t;  // -sqrt(3/2)
      p0[1] = l_accum;
    } else {
#pragma unroll
      for (int m = 0; m < l - 1; ++m) {
        T v = cos_t * p1[m];
        v += SphC<T>::b(l * S + m) * p2[m];
        v *= SphC<T>::a(l * S + m);
        p0[m] = v;
      }
      p0[l - 1] = l_accum * cos_t * SphC<T>::c1(l);
      l_accum = l_accum * sin_t * SphC<T>::c2(l);
      p0[l] = l_accum;
    }
#pragma unroll
    for (int m = l + 1; m < L + 2; ++m) p0[m] = T(0);
    const int base = l * l + l;
    begin_l(l);
    // Y values
    T Yv[2 * L + 1];
#pragma unroll
    for (int m = 0; m <= l; ++m) {
      Yv[l + m] = p0[m] * cm[m];
      Yv[l - m] = p0[m] * sm[m];
    }
    Yv[l] = p0[0] * inv_sqrt2;
    if (!DER || l == 0) {
#pragma unroll
      for (int k = 0; k < 2 * l + 1; ++k) emit(base - l + k, Yv[k], T(0), T(0), T(0));
    } else {
      const T pl0 = SphC<T>::plm(l * S + 0);
      emit(base, Yv[l], cos_t * cos_p * pl0 * inv_sqrt2 * p0[1],
           cos_t * sin_p * pl0 * inv_sqrt2 * p0[1], T(-1) * sin_td * pl0 * inv_sqrt2 * p0[1]);
#pragma unroll
      for (int k = 0; k < l; ++k) {
        const int m = k + 1;
        const T pk = SphC<T>::plm(l * S + k), pk1 = SphC<T>::plm(l * S + k + 1);
        const T lpd = pk * p0[k] - pk1 * p0[k + 2];
        T pdf;
        if (sin_td > T(0.1))
          pdf = T(k + 1) / sin_td * p0[k + 1];
        else
          pdf = T(-0.5) / cos_t * (pk * p0[k] + pk1 * p0[k + 2]);
        T dxp = sin_p * pdf * sm[m];
        dxp += T(-0.5) * cos_t * cos_p * cm[m] * lpd;
        T dxn = T(-1) * sin_p * pdf * cm[m];
        dxn += T(-0.5) * cos_t * cos_p * sm[m] * lpd;
        T dyp = T(-1) * cos_p * pdf * sm[m];
        dyp += T(-0.5) * cos_t * sin_p * cm[m] * lpd;
        T dyn = cos_p * pdf * cm[m];
        dyn += T(-0.5) * cos_t * sin_p * sm[m] * lpd;
        T dzp = T(0.5) * sin_td * cm[m] * lpd;
        T dzn = T(0.5) * sin_td * sm[m] * lpd;
        emit(base + m, Yv[l + m], dxp, dyp, dzp);
        emit(base - m, Yv[l - m], dxn, dyn, dzn);
      }
    }
#pragma unroll
    for (int m = 0; m < L + 2; ++m) {
      p2[m] = p1[m];
      p1[m] = p0[m];
    }
  }
}

// Cubic-spline evaluation of the radial table at r: index search with the
// reference's points-per-unit quirk (math/interpolator.cc:214-230), value and
// derivative formulas of math/interpolator.cc:177-212.
// Padded coefficient layout of the FP32 path: each l-block of 2l+1 values
// is padded to a multiple of 4 floats, so every product over m is a few
// 16-byte loads. Rows ((species, n) pairs) are row_stride(L) floats apart.
__host__ __device__ constexpr int pad4(int x) { return (x + 3) & ~3; }
// padded offset of block l: sum_{l' < l} pad4(2l'+1)
__host__ __device__ constexpr int offp(int l) {
  int o = 0;
  for (int i = 0; i < l; ++i) o += pad4(2 * i + 1);
  return o;
}
// the same sum in closed form for a runtime l: blocks of l' = 2k and 2k+1
// pad to 4(k+1) each
__host__ __device__ __forceinline__ int offp_rt(int l) {
  const int k = l >> 1;
  return 4 * k * (k + 1) + ((l & 1) ? 4 * (k + 1) : 0);
}
// row stride of the padded layout: the block sum rounded so that stride/4
// is odd (conflict-free 16-byte loads across 8 consecutive rows)
__host__ __device__ constexpr int row_stride(int L) {
  int s = offp(L + 1);
  return ((s / 4) % 2 == 1) ? s : s + 4;
}

struct SplinePos {
  int k;
  double a, b;
};
__device__ __forceinline__ SplinePos spline_pos(const SplineDev & s, double r) {
  SplinePos p;
  int k = static_cast<int>((r - s.x1) * s.ppu) - 1;
  k = max(0, min(s.search_size, k));
  p.k = k;
  p.a = (s.grid[k + 1] - r) / s.h;
  p.b = 1 - p.a;
  return p;
}

}  // namespace rgpu
