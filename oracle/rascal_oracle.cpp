// CPU FP64 oracle for the librascal descriptor hot path.
//
// TEST INFRASTRUCTURE ONLY: this file is a plain restatement of the
// reference algorithms, used by tests/ (parity checks), by
// __graft_entry__.smoke() (as the checker) and by bench.py's CPU-baseline
// leg. The product library never links or calls it.
//
// Every function names the reference file:line it follows (paths relative to
// the librascal source tree). Floating point is evaluated in the order the
// reference writes it, and the file is compiled with -ffp-contract=off so no
// FMA contraction changes the rounding of the neighbour-list geometry.
//
// Conventions
//   * Cells are given ASE-style: 3x3 row-major, rows = lattice vectors. The
//     reference stores the transpose (columns = lattice vectors,
//     atomic_structure.hh:400-449); `cell_t(i,j)` below is that transpose.
//   * Dense species layout: the caller passes a sorted species list; dense
//     expansion rows are [species][n][lm] and power-spectrum rows are
//     [(a<=b) pair][n1][n2][l], zero where a key is absent. Absent keys hold
//     zeros in the reference's dense export too
//     (property_block_sparse.hh:911-987), so the numbers are identical.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double SQRT_TWO = 1.41421356237309504880168872420969808;
constexpr double INV_SQRT_TWO = 0.707106781186547524400844362104849039;
constexpr double SQRT_THREE = 1.7320508075688772935274463415058723;
constexpr double DBL_FTOL = 100.0 * std::numeric_limits<double>::epsilon();
constexpr double DOVERFLOW = std::numeric_limits<double>::infinity();
constexpr int MAX_CHEM_ELEMENTS = 130;  // utils.hh:399

// math/utils.hh:83-122 -- repeated-squaring integer powers.
static double pow_u(double x, size_t n) {
  double value{1};
  do {
    if (n & 1) value *= x;
    n >>= 1;
    x *= x;
  } while (n);
  return value;
}
static double pow_i(double x, int n) {
  size_t un{0};
  double value{x};
  if (n < 0) {
    value = 1.0 / x;
    un = static_cast<size_t>(-n);
  } else {
    un = static_cast<size_t>(n);
  }
  return pow_u(value, un);
}

// Eigen-3.3 style LinSpaced (low + i*step, last point pinned to high).
static std::vector<double> linspaced(int num, double low, double high) {
  std::vector<double> v(num);
  if (num == 1) {
    v[0] = high;
    return v;
  }
  double step = (high - low) / double(num - 1);
  bool flip = std::fabs(high) < std::fabs(low);
  int size1 = num - 1;
  for (int i = 0; i < num; ++i) {
    if (flip)
      v[i] = (i == 0) ? low : (high - double(size1 - i) * step);
    else
      v[i] = (i == size1) ? high : (low + double(i) * step);
  }
  return v;
}

/* ------------------------------------------------------------------------ */
// math/hyp1f1.cc:51-195 -- power series of 1F1(a,b,z).
struct Hyp1f1Series {
  double a, b;
  size_t mmax;
  double prefac, tolerance;
  bool is_exp{false};
  std::vector<double> coeff, coeff_der;
  Hyp1f1Series(double a_, double b_, size_t mmax_, double tol)
      : a{a_}, b{b_}, mmax{mmax_}, prefac{std::tgamma(a_) / std::tgamma(b_)},
        tolerance{tol} {
    if (std::fabs(1 - b / a) < DBL_FTOL) {
      is_exp = true;
    } else {
      coeff.resize(mmax);
      coeff_der.resize(mmax);
      double u{0.};
      coeff[0] = a / b;
      coeff_der[0] = (a + 1) / (b + 1);
      for (size_t i{1}; i < mmax; ++i) {
        u = (a + i) / ((i + 1) * (b + i));
        coeff[i] = coeff[i - 1] * u;
        u = (a + i + 1) / ((i + 1) * (b + i + 1));
        coeff_der[i] = coeff_der[i - 1] * u;
      }
    }
  }
  double sum(double z, const std::vector<double> & c) const {
    double res{1.0}, a1{1.0}, zpow{z}, z4{z * z};
    z4 *= z4;
    for (size_t i{0}; i < mmax - 3; i += 4) {
      a1 = zpow * (c[i] + z * (c[i + 1] + z * (c[i + 2] + z * c[i + 3])));
      if (a1 < tolerance * res) {
        res += a1;
        break;
      }
      zpow *= z4;
      res += a1;
    }
    if (res > DOVERFLOW) throw std::overflow_error("Hyp1f1Series overflow");
    return res;
  }
  double hyp1f1(double z, bool der) const {
    if (!der) return sum(z, coeff);
    return sum(z, coeff_der) * a / b;
  }
  double calc(double z, bool der) const {
    if (!is_exp) return hyp1f1(z, der);
    return std::exp(z);
  }
  double calc(double z, double z2, double ez2, bool der) const {
    if (!is_exp) return prefac * calc(z, der) * ez2;
    return prefac * std::exp(z + z2);
  }
};

// math/hyp1f1.cc:197-271 -- asymptotic expansion (2F0) of 1F1(a,b,z).
struct Hyp1f1Asymptotic {
  double a, b, prefac;
  bool is_n_and_l{false}, is_exp{false};
  double tolerance;
  size_t mmax;
  std::vector<double> coeff, coeff_der;
  Hyp1f1Asymptotic(double a_, double b_, size_t mmax_, double tol)
      : a{a_}, b{b_}, prefac{std::tgamma(b_) / std::tgamma(a_)}, tolerance{tol},
        mmax{mmax_} {
    double intpart;
    double f2{std::modf(2 * (a - b), &intpart)};
    if (std::fabs(f2) < 1e-14) is_n_and_l = true;
    if (std::fabs(1 - b / a) < DBL_FTOL) {
      is_exp = true;
    } else {
      coeff.resize(mmax);
      coeff_der.resize(mmax);
      double bma{b - a}, oma{1 - a}, u{0.}, oma1{1 - a - 1};
      coeff[0] = bma * oma;
      coeff_der[0] = bma * oma1;
      for (size_t i{1}; i < mmax; ++i) {
        u = (bma + i) * (oma + i) / (i + 1);
        coeff[i] = coeff[i - 1] * u;
        u = (bma + i) * (oma1 + i) / (i + 1);
        coeff_der[i] = coeff_der[i - 1] * u;
      }
    }
  }
  double z_power_a_b(double z) const {
    if (is_n_and_l) return std::sqrt(pow_i(z, static_cast<int>(2 * (a - b))));
    return std::pow(z, a - b);
  }
  double sum(double z, const std::vector<double> & c) const {
    double iz{1.0 / z};
    double res{1.}, izpow{1.}, s_i{1.};
    for (size_t i{0}; i < mmax; ++i) {
      izpow *= iz;
      s_i = c[i] * izpow;
      if (res > 0 and std::fabs(s_i) < tolerance * res) break;
      res += s_i;
    }
    if (res > DOVERFLOW) throw std::overflow_error("Hyp1f1Asymptotic overflow");
    return res;
  }
  double hyp2f0(double z, bool der) const {
    return der ? sum(z, coeff_der) : sum(z, coeff);
  }
  double calc(double z, double z2, bool der) const {
    if (!is_exp) {
      double fac{z_power_a_b(z)};
      return hyp2f0(z, der) * std::exp(z + z2) * fac;
    }
    return std::exp(z + z2) / prefac;
  }
  double calc(double z, bool der) const {
    if (!is_exp) {
      double fac{z_power_a_b(z)};
      double result{prefac * std::exp(z) * fac * hyp2f0(z, der)};
      if (std::isnan(result)) result = DOVERFLOW;
      return result;
    }
    return std::exp(z);
  }
};

// math/hyp1f1.cc:273-356 -- switch between series and asymptotic forms.
struct Hyp1f1 {
  Hyp1f1Series series;
  Hyp1f1Asymptotic asym;
  double a, b, tolerance;
  double z_asympt{1.}, h1f1_a{0}, h1f1_s{0}, z_above{0.}, z_below{0.};
  Hyp1f1(double a_, double b_, size_t mmax, double tol)
      : series{a_, b_, mmax, tol}, asym{a_, b_, mmax, tol}, a{a_}, b{b_},
        tolerance{tol} {
    if (std::fabs(1 - b / a) > DBL_FTOL) {
      find_switching_point();
      update_switching_point();
    }
  }
  void update_switching_point() {
    h1f1_s = series.calc(z_asympt, false);
    h1f1_a = asym.calc(z_asympt, false);
  }
  void find_switching_point() {
    int max_it{100};
    int i_it{0};
    update_switching_point();
    z_below = z_above = z_asympt;
    if (std::fabs(1 - h1f1_s / h1f1_a) > tolerance) {
      i_it = 0;
      while (std::fabs(1 - h1f1_s / h1f1_a) > 100 * tolerance and
             i_it < max_it) {
        z_asympt *= 1.5;
        update_switching_point();
        i_it++;
      }
      z_above = z_asympt;
    } else {
      i_it = 0;
      while (std::fabs(1 - h1f1_s / h1f1_a) < 100 * tolerance and
             i_it < max_it) {
        z_asympt *= 0.5;
        update_switching_point();
        i_it++;
      }
      z_below = z_asympt;
    }
    z_asympt = (z_above + z_below) * 0.5;
    update_switching_point();
    i_it = 0;
    while (z_above - z_below > tolerance and i_it < max_it) {
      if (std::fabs(1 - h1f1_s / h1f1_a) > tolerance) {
        z_below = z_asympt;
      } else {
        z_above = z_asympt;
      }
      z_asympt = (z_above + z_below) * 0.5;
      update_switching_point();
      i_it++;
    }
  }
  double calc(double z, bool der) const {
    if (z > z_asympt) return asym.calc(z, der);
    return series.calc(z, der);
  }
  double calc(double z, double z2, double ez2, bool der) const {
    if (z > z_asympt) return asym.calc(z, z2, der);
    return series.calc(z, z2, ez2, der);
  }
};

// math/hyp1f1.cc:376-490 -- the (n, l) table of modified 1F1 values G and
// their radial derivatives, direct or by downward recursion in l.
struct Hyp1f1SphericalExpansion {
  size_t max_angular{0}, max_radial{0};
  std::vector<Hyp1f1> h;
  double tolerance;
  size_t precomputation_size;
  bool recursion;
  std::vector<double> values, derivatives, z, dz_dr;  // row-major n x (L+1)
  Hyp1f1SphericalExpansion(bool rec, double tol, size_t pre)
      : tolerance{tol}, precomputation_size{pre}, recursion{rec} {}
  int pos(int n, int l) const { return l + (int(max_angular) + 1) * n; }
  static double get_a(int n, int l) { return 0.5 * (n + l + 3); }
  static double get_b(int l) { return l + 1.5; }
  void precompute(size_t nmax, size_t lmax) {
    max_angular = lmax;
    max_radial = nmax;
    values.assign(nmax * (lmax + 1), 0.);
    derivatives.assign(nmax * (lmax + 1), 0.);
    z.assign(nmax, 0.);
    dz_dr.assign(nmax, 0.);
    h.clear();
    for (size_t n{0}; n < nmax; n++)
      for (size_t l{0}; l < lmax + 1; l++)
        h.emplace_back(get_a(int(n), int(l)), get_b(int(l)),
                       precomputation_size, tolerance);
  }
  double & val(int n, int l) { return values[pos(n, l)]; }
  double & der(int n, int l) { return derivatives[pos(n, l)]; }
  static double rec_val(double a, double b, double z, double M1p2p,
                        double M1p1p) {
    return (z * (a - b) * M1p2p + M1p1p * b) / a;
  }
  static double rec_der(double, double b, double z, double M2p3p,
                        double M1p2p) {
    return z * M2p3p + M1p2p * (b + 1);
  }
  void prepare_z(double r_ij, double alpha, const std::vector<double> & fac_b,
                 double & z2, double & ez2) {
    double alpha_rij{alpha * r_ij};
    z2 = -r_ij * alpha_rij;
    ez2 = std::exp(z2);
    for (size_t n{0}; n < max_radial; ++n) {
      z[n] = (alpha_rij * alpha) * (1.0 / (alpha + fac_b[n]));
      dz_dr[n] = z[n];
      z[n] *= r_ij;
      dz_dr[n] *= 2;
    }
  }
  void calc(double r_ij, double alpha, const std::vector<double> & fac_b,
            bool derivative) {
    if (not recursion or max_angular < 3)
      calc_direct(r_ij, alpha, fac_b, derivative);
    else
      calc_recursion(r_ij, alpha, fac_b);
  }
  void calc_recursion(double r_ij, double alpha,
                      const std::vector<double> & fac_b) {
    double M1p2p{0.}, M2p3p{0.}, MP1p2p{0.}, MP2p3p{0.}, M1p1p{0.}, Moo{0.},
        MP1p1p{0.}, MPoo{0.};
    double z2, ez2;
    double alpha_rij{alpha * r_ij};
    prepare_z(r_ij, alpha, fac_b, z2, ez2);
    for (int n{0}; n < int(max_radial); ++n) {
      double zz{z[n]};
      int l{static_cast<int>(max_angular)};
      int ip{pos(n, l)};
      M1p2p = h[ip].calc(zz, z2, ez2, false);
      val(n, l) = M1p2p;
      M2p3p = h[ip].calc(zz, z2, ez2, true);
      der(n, l) = M2p3p;
      ip = pos(n, l - 1);
      MP1p2p = h[ip].calc(zz, z2, ez2, false);
      val(n, l - 1) = MP1p2p;
      MP2p3p = h[ip].calc(zz, z2, ez2, true);
      der(n, l - 1) = MP2p3p;
      l -= 2;
      for (; l > 0; l -= 2) {
        double a{get_a(n, l)}, b{get_b(l)};
        M1p1p = rec_der(a, b, zz, M2p3p, M1p2p);
        Moo = rec_val(a, b, zz, M1p2p, M1p1p);
        val(n, l) = Moo;
        der(n, l) = M1p1p;
        M2p3p = M1p1p;
        M1p2p = Moo;
        a = get_a(n, l - 1);
        b = get_b(l - 1);
        MP1p1p = rec_der(a, b, zz, MP2p3p, MP1p2p);
        MPoo = rec_val(a, b, zz, MP1p2p, MP1p1p);
        val(n, l - 1) = MPoo;
        der(n, l - 1) = MP1p1p;
        MP2p3p = MP1p1p;
        MP1p2p = MPoo;
      }
      if (max_angular % 2 == 0) {
        double a{get_a(n, 0)}, b{get_b(0)};
        M1p1p = rec_der(a, b, zz, M2p3p, M1p2p);
        Moo = rec_val(a, b, zz, M1p2p, M1p1p);
        val(n, 0) = Moo;
        der(n, 0) = M1p1p;
      }
      for (size_t l2{0}; l2 < max_angular + 1; ++l2) der(n, l2) *= dz_dr[n];
    }
    for (size_t i{0}; i < derivatives.size(); ++i)
      derivatives[i] -= (2 * alpha_rij) * values[i];
  }
  void calc_direct(double r_ij, double alpha, const std::vector<double> & fac_b,
                   bool derivative) {
    double z2, ez2;
    prepare_z(r_ij, alpha, fac_b, z2, ez2);
    for (int n{0}; n < int(max_radial); n++)
      for (int l{0}; l < int(max_angular) + 1; l++)
        val(n, l) = h[pos(n, l)].calc(z[n], z2, ez2, false);
    if (derivative) {
      for (int n{0}; n < int(max_radial); n++) {
        for (int l{0}; l < int(max_angular) + 1; l++)
          der(n, l) = h[pos(n, l)].calc(z[n], z2, ez2, true);
        for (int l{0}; l < int(max_angular) + 1; l++) der(n, l) *= dz_dr[n];
      }
      for (size_t i{0}; i < derivatives.size(); ++i)
        derivatives[i] -= (2 * alpha * r_ij) * values[i];
    }
  }
};

/* ------------------------------------------------------------------------ */
// Cyclic Jacobi eigen-decomposition of a small symmetric matrix. Stands in
// for Eigen::SelfAdjointEigenSolver used by
// representations/calculator_spherical_expansion.hh:670-679.
static void jacobi_eigen(int n, std::vector<double> A, std::vector<double> & w,
                         std::vector<double> & V) {
  V.assign(n * n, 0.);
  for (int i = 0; i < n; ++i) V[i * n + i] = 1.;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[p * n + q] * A[p * n + q];
    if (off < 1e-300) break;
    for (int p = 0; p < n; ++p) {
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p * n + q];
        if (apq == 0.) continue;
        double app = A[p * n + p], aqq = A[q * n + q];
        double theta = (aqq - app) / (2. * apq);
        double t = (theta >= 0 ? 1. : -1.) /
                   (std::fabs(theta) + std::sqrt(theta * theta + 1.));
        double c = 1. / std::sqrt(t * t + 1.), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
      }
    }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = A[i * n + i];
}

/* ------------------------------------------------------------------------ */
// GTO radial contribution, representations/calculator_spherical_expansion.hh:
// 351-384 (hypers), 404-411 (precompute), 478-501 (centre), 518-584
// (neighbour value and derivative), 588-618 (orthonormalisation), 621-680
// (sigmas, norms, overlap and S^-1/2).
struct GTO {
  int nmax, lmax;
  double rc, fac_a;
  std::vector<double> sigmas, fac_b, norm, n_factors;
  std::vector<double> ortho;       // S^-1/2, n x n row-major
  std::vector<double> ortho_norm;  // diag(norm) * S^-1/2
  std::vector<double> center;      // n, raw (not orthonormalised)
  Hyp1f1SphericalExpansion hyp{true, 1e-13, 200};
  std::vector<double> dfal, abln, RI, dRI;  // scratch

  GTO(int n, int l, double rc_, double sigma) : nmax{n}, lmax{l}, rc{rc_} {
    fac_a = 0.5 * pow_i(sigma, -2);
    sigmas.resize(n);
    fac_b.resize(n);
    norm.resize(n);
    n_factors.resize(n);
    for (int i = 0; i < n; ++i) {
      sigmas[i] = std::max(std::sqrt(static_cast<double>(i)), 1.0) * rc /
                  static_cast<double>(n);
      fac_b[i] = 0.5 * pow_i(sigmas[i], -2);
      norm[i] = 0.25 * std::sqrt(2.0 / (std::tgamma(1.5 + i) *
                                        pow_u(sigmas[i], 3 + 2 * size_t(i))));
      n_factors[i] = std::tgamma(0.5 * (3.0 + i)) / std::tgamma(1.5);
    }
    std::vector<double> S(n * n);
    for (int n1 = 0; n1 < n; ++n1)
      for (int n2 = 0; n2 < n; ++n2) {
        double s1 = sigmas[n1], s2 = sigmas[n2];
        S[n1 * n + n2] =
            std::pow(0.5 / pow_i(s1, 2) + 0.5 / pow_i(s2, 2),
                     -0.5 * (3.0 + n1 + n2)) /
            (pow_u(s1, size_t(n1)) * pow_u(s2, size_t(n2))) *
            std::tgamma(0.5 * (3.0 + n1 + n2)) /
            (std::pow(s1 * s2, 1.5) *
             std::sqrt(std::tgamma(1.5 + n1) * std::tgamma(1.5 + n2)));
      }
    std::vector<double> w, V;
    jacobi_eigen(n, S, w, V);
    ortho.assign(n * n, 0.);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double s = 0.;
        for (int k = 0; k < n; ++k)
          s += V[i * n + k] * (1. / std::sqrt(w[k])) * V[j * n + k];
        ortho[i * n + j] = s;
      }
    ortho_norm.assign(n * n, 0.);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) ortho_norm[i * n + j] = norm[i] * ortho[i * n + j];
    hyp.precompute(n, l);
    center.resize(n);
    for (int i = 0; i < n; ++i) {
      double abln0{0};
      if (i % 2 == 0)
        abln0 = std::sqrt(pow_i(fac_a + fac_b[i], -1 * static_cast<int>(3 + i)));
      else
        abln0 = pow_i(fac_a + fac_b[i], -1 * static_cast<int>(3 + i) / 2);
      center[i] = n_factors[i] * abln0;
    }
    dfal.resize(l + 1);
    abln.resize(n * (l + 1));
    RI.resize(n * (l + 1));
    dRI.resize(n * (l + 1));
  }
  // Raw (non-orthonormalised) radial integral and optionally its derivative.
  void neighbour(double distance, bool with_der) {
    int L1 = lmax + 1;
    dfal[0] = 1.;
    double dfa{distance * fac_a};
    for (int l = 1; l < L1; ++l) dfal[l] = dfal[l - 1] * dfa;
    std::vector<double> abl(nmax);
    for (int n = 0; n < nmax; ++n) abl[n] = 1.0 / std::sqrt(fac_a + fac_b[n]);
    for (int n = 0; n < nmax; ++n) abln[n * L1] = pow_u(abl[n], 3 + size_t(n));
    for (int l = 1; l < L1; ++l)
      for (int n = 0; n < nmax; ++n)
        abln[n * L1 + l] = abln[n * L1 + l - 1] * abl[n];
    hyp.calc(distance, fac_a, fac_b, with_der);
    for (int n = 0; n < nmax; ++n)
      for (int l = 0; l < L1; ++l)
        RI[n * L1 + l] = (abln[n * L1 + l] * hyp.values[n * L1 + l]) * dfal[l];
    if (with_der) {
      for (int n = 0; n < nmax; ++n)
        for (int l = 0; l < L1; ++l) {
          double pf = double(l) / distance;
          dRI[n * L1 + l] =
              (abln[n * L1 + l] * hyp.derivatives[n * L1 + l]) * dfal[l] +
              RI[n * L1 + l] * pf;
        }
    }
  }
  // out = ortho_norm^T * in (n x cols), row-major.
  void lhs(const double * in, double * out, int cols) const {
    for (int i = 0; i < nmax; ++i)
      for (int c = 0; c < cols; ++c) {
        double s = 0.;
        for (int k = 0; k < nmax; ++k) s += ortho_norm[k * nmax + i] * in[k * cols + c];
        out[i * cols + c] = s;
      }
  }
};

/* ------------------------------------------------------------------------ */
// Natural cubic spline on a uniform grid over a vector-valued function,
// math/interpolator.hh:167-185 (grid), 502-543 (absolute error),
// 705-712 (refinement), 976-1287 (matrix interpolator) and
// math/interpolator.cc:148-230 (second derivatives, evaluation, search).
struct Spline {
  double x1, x2, h{0}, h_sq_6{0}, ppu{0};
  int G{0}, width{0}, search_size{0}, dof{5};
  std::vector<double> grid, y, y2h;  // y and y''*h^2/6: G x width row-major

  template <class F>
  Spline(F && func, double x1_, double x2_, double accuracy, int width_,
         int max_grid_points = 100000)
      : x1{x1_}, x2{x2_}, width{width_} {
    bool below = grid_error(func, accuracy);
    while (!below && int(grid.size()) < max_grid_points) {
      dof++;
      below = grid_error(func, accuracy);
    }
  }
  template <class F>
  bool grid_error(F && func, double accuracy) {
    int npts = 2 << dof;
    grid = linspaced(npts, x1, x2);
    G = npts;
    y.assign(size_t(G) * width, 0.);
    for (int i = 0; i < G; ++i) func(grid[i], &y[size_t(i) * width]);
    init_second_derivative();
    ppu = G / (grid[G - 1] - grid[0]);
    search_size = G - 2;
    int tdof = std::max(dof, 5);
    int tn = 2 << tdof;
    double offset = (x2 - x1) / (2 * (tn - 1));
    std::vector<double> test = linspaced(tn - 1, x1 + offset, x2 - offset);
    std::vector<double> vi(width), ve(width);
    double err = 0.;
    for (size_t t = 0; t < test.size(); ++t) {
      interpolate(test[t], vi.data());
      func(test[t], ve.data());
      for (int c = 0; c < width; ++c) err += std::fabs(vi[c] - ve[c]);
    }
    err /= double(test.size() * size_t(width));
    return err < accuracy;
  }
  void init_second_derivative() {
    h = grid[1] - grid[0];
    h_sq_6 = h * h / 6.0;
    int n = G;
    std::vector<double> y2(size_t(n) * width, 0.), u(size_t(n) * width, 0.);
    double sig = 0.5;
    for (int i = 1; i < n - 1; i++) {
      for (int c = 0; c < width; ++c) {
        double p = sig * y2[size_t(i - 1) * width + c] + 2.0;
        y2[size_t(i) * width + c] = (sig - 1.0) / p;
        double uu = (3. * (y[size_t(i + 1) * width + c] -
                           2 * y[size_t(i) * width + c] +
                           y[size_t(i - 1) * width + c])) /
                    (h * h);
        uu -= sig * u[size_t(i - 1) * width + c];
        uu /= p;
        u[size_t(i) * width + c] = uu;
      }
    }
    for (int c = 0; c < width; ++c) y2[size_t(n - 1) * width + c] = 0.;
    for (int k = n - 2; k > 0; k--)
      for (int c = 0; c < width; ++c)
        y2[size_t(k) * width + c] =
            y2[size_t(k) * width + c] * y2[size_t(k + 1) * width + c] +
            u[size_t(k) * width + c];
    for (int c = 0; c < width; ++c) y2[c] = 0.;
    y2h.resize(y2.size());
    for (size_t i = 0; i < y2.size(); ++i) y2h[i] = y2[i] * h_sq_6;
  }
  int search(double x) const {
    return std::max(0, std::min(search_size,
                                static_cast<int>((x - x1) * ppu) - 1));
  }
  void interpolate(double x, double * out) const {
    int klo = search(x), khi = klo + 1;
    double a{(grid[khi] - x) / h};
    double b{1 - a};
    const double *ylo = &y[size_t(klo) * width], *yhi = &y[size_t(khi) * width];
    const double *dlo = &y2h[size_t(klo) * width], *dhi = &y2h[size_t(khi) * width];
    for (int c = 0; c < width; ++c)
      out[c] = a * (ylo[c] + (a * a - 1) * dlo[c]) +
               b * (yhi[c] + (b * b - 1) * dhi[c]);
  }
  void derivative(double x, double * out) const {
    int klo = search(x), khi = klo + 1;
    double a{(grid[khi] - x) / h};
    double b{1 - a};
    const double *ylo = &y[size_t(klo) * width], *yhi = &y[size_t(khi) * width];
    const double *dlo = &y2h[size_t(klo) * width], *dhi = &y2h[size_t(khi) * width];
    for (int c = 0; c < width; ++c)
      out[c] = (yhi[c] - ylo[c] - (3 * a * a - 1) * dlo[c] +
                (3 * b * b - 1) * dhi[c]) /
               h;
  }
};

/* ------------------------------------------------------------------------ */
// Real spherical harmonics and their Cartesian gradients,
// math/spherical_harmonics.cc:36-363.
struct SphericalHarmonics {
  int L;
  std::vector<double> P;                 // (L+1) x (L+2)
  std::vector<double> coeff_a, coeff_b;  // (L+1) x (2L+1)
  std::vector<double> ac1, ac2, plm;     // plm: (L+1) x (L+1)
  std::vector<double> cosm, sinm;        // L+1
  std::vector<double> Y, dY;             // K, 3 x K
  std::vector<double> lpd, pdf;
  explicit SphericalHarmonics(int lmax) : L{lmax} {
    int K = (L + 1) * (L + 1);
    P.assign((L + 1) * (L + 2), 0.);
    coeff_a.assign((L + 1) * (2 * L + 1), 0.);
    coeff_b.assign((L + 1) * (2 * L + 1), 0.);
    for (int l = 0; l < L + 1; l++) {
      double lsq = double(l) * double(l);
      double lm1sq = double(l - 1) * double(l - 1);
      for (int m = 0; m < l + 1; m++) {
        double msq = double(m) * double(m);
        coeff_a[l * (2 * L + 1) + m] = std::sqrt((4 * lsq - 1.0) / (lsq - msq));
        coeff_b[l * (2 * L + 1) + m] =
            -1.0 * std::sqrt((lm1sq - msq) / (4 * lm1sq - 1.0));
      }
    }
    ac1.assign(L + 1, 0.);
    ac2.assign(L + 1, 0.);
    for (int l = 0; l < L + 1; l++) {
      ac1[l] = std::sqrt(2 * l + 1);
      ac2[l] = -std::sqrt(1.0 + 0.5 / l);
    }
    plm.assign((L + 1) * (L + 1), 0.);
    for (int l = 0; l < L + 1; l++)
      for (int m = 0; m < l + 1; m++)
        plm[l * (L + 1) + m] = std::sqrt(double((l - m) * (l + m + 1)));
    cosm.assign(L + 1, 0.);
    sinm.assign(L + 1, 0.);
    Y.assign(K, 0.);
    dY.assign(3 * K, 0.);
    lpd.assign(L + 1, 0.);
    pdf.assign(L + 1, 0.);
  }
  double & p(int l, int m) { return P[l * (L + 2) + m]; }
  void alp(double cos_theta) {
    double sin_theta = std::sqrt(1.0 - pow_i(cos_theta, 2));
    const double SQRT_INV_2PI = std::sqrt(0.5 / PI);
    double l_accum{SQRT_INV_2PI};
    p(0, 0) = SQRT_INV_2PI;
    if (L > 0) {
      p(1, 0) = cos_theta * SQRT_THREE * SQRT_INV_2PI;
      l_accum = l_accum * -std::sqrt(3.0 / 2.0) * sin_theta;
      p(1, 1) = l_accum;
    }
    for (int l = 2; l < L + 1; l++) {
      for (int m = 0; m < l - 1; ++m) {
        double v = cos_theta * p(l - 1, m);
        v += coeff_b[l * (2 * L + 1) + m] * p(l - 2, m);
        v *= coeff_a[l * (2 * L + 1) + m];
        p(l, m) = v;
      }
      p(l, l - 1) = l_accum * cos_theta * ac1[l];
      l_accum = l_accum * sin_theta * ac2[l];
      p(l, l) = l_accum;
    }
  }
  void calc(const double * direction, bool with_der) {
    double d[3] = {direction[0], direction[1], direction[2]};
    if (std::fabs((d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) - 1.0) > DBL_FTOL) {
      double nrm = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      for (int c = 0; c < 3; ++c) d[c] = direction[c] / nrm;
    }
    double cos_theta = d[2];
    double sqrt_xy = std::hypot(d[0], d[1]);
    double cos_phi{1.0}, sin_phi{0.0};
    if (sqrt_xy >= DBL_FTOL) {
      cos_phi = d[0] / sqrt_xy;
      sin_phi = d[1] / sqrt_xy;
    }
    alp(cos_theta);
    for (int m = 0; m < L + 1; m++) {
      if (m == 0) {
        cosm[0] = 1.0;
        sinm[0] = 0.0;
      } else if (m == 1) {
        cosm[1] = cos_phi;
        sinm[1] = sin_phi;
      } else {
        cosm[m] = 2.0 * cos_phi * cosm[m - 1] - cosm[m - 2];
        sinm[m] = 2.0 * cos_phi * sinm[m - 1] - sinm[m - 2];
      }
    }
    int lm_base = 0;
    for (int l = 0; l < L + 1; l++) {
      for (int m = 0; m < l + 1; ++m) Y[lm_base + l + m] = p(l, m) * cosm[m];
      for (int m = 0; m < l + 1; ++m) Y[lm_base + l - m] = p(l, m) * sinm[m];
      Y[lm_base + l] = p(l, 0) * INV_SQRT_TWO;
      lm_base += 2 * l + 1;
    }
    if (with_der) derivatives(sqrt_xy, cos_theta, sin_phi, cos_phi);
  }
  void derivatives(double sin_theta, double cos_theta, double sin_phi,
                   double cos_phi) {
    int K = (L + 1) * (L + 1);
    double * dx = &dY[0];
    double * dy = &dY[K];
    double * dz = &dY[2 * K];
    dx[0] = dy[0] = dz[0] = 0.;
    int lb = 1;
    for (int l = 1; l < L + 1; l++) {
      const double * pl = &plm[l * (L + 1)];
      for (int k = 0; k < l; ++k)
        lpd[k] = pl[k] * p(l, k) - pl[k + 1] * p(l, k + 2);
      if (sin_theta > 0.1) {
        for (int k = 0; k < l; ++k) pdf[k] = double(k + 1) / sin_theta * p(l, k + 1);
      } else {
        for (int k = 0; k < l; ++k)
          pdf[k] = -0.5 / cos_theta * (pl[k] * p(l, k) + pl[k + 1] * p(l, k + 2));
      }
      dx[lb + l] = cos_theta * cos_phi * pl[0] * INV_SQRT_TWO * p(l, 1);
      dy[lb + l] = cos_theta * sin_phi * pl[0] * INV_SQRT_TWO * p(l, 1);
      dz[lb + l] = -1.0 * sin_theta * pl[0] * INV_SQRT_TWO * p(l, 1);
      for (int k = 0; k < l; ++k) {
        int m = k + 1;
        double v;
        v = sin_phi * pdf[k] * sinm[m];
        v += -0.5 * cos_theta * cos_phi * cosm[m] * lpd[k];
        dx[lb + l + m] = v;
        v = -1.0 * sin_phi * pdf[k] * cosm[m];
        v += -0.5 * cos_theta * cos_phi * sinm[m] * lpd[k];
        dx[lb + l - m] = v;
        v = -1.0 * cos_phi * pdf[k] * sinm[m];
        v += -0.5 * cos_theta * sin_phi * cosm[m] * lpd[k];
        dy[lb + l + m] = v;
        v = cos_phi * pdf[k] * cosm[m];
        v += -0.5 * cos_theta * sin_phi * sinm[m] * lpd[k];
        dy[lb + l - m] = v;
        dz[lb + l + m] = 0.5 * sin_theta * cosm[m] * lpd[k];
        dz[lb + l - m] = 0.5 * sin_theta * sinm[m] * lpd[k];
      }
      lb += 2 * l + 1;
    }
  }
};

// cos(x) for x within 0.02 of pi, correctly rounded: -cos(pi - x) from its
// Taylor series in double-double. In f_c = (1 + cos x)/2 the sum cancels
// near the cutoff, so the last bit of cos decides the relative accuracy of
// f_c there; a libm's cos may be off by an ulp in near-tie cases, and the
// GPU and this oracle both use this correctly rounded value instead.
static double cos_near_pi(double x) {
  const double pi_hi = 3.141592653589793116, pi_lo = 1.2246467991473532e-16;
  double th = pi_hi - x;
  double s = th + pi_lo;
  double tl = pi_lo - (s - th);
  th = s;
  double u = th * th;
  double ue = std::fma(th, th, -u) + 2.0 * th * tl;
  double h = u * 0.5, hl = ue * 0.5;
  double c = 1.0 - h;
  double ce = ((1.0 - c) - h) - hl;
  double tail = u * u * (1.0 / 24.0) - u * u * u * (1.0 / 720.0) + u * u * u * u * (1.0 / 40320.0);
  return -(c + (ce + tail));
}

// representations/cutoff_functions.hh:69-107
static double fc_cos(double r, double rc, double sw) {
  if (r <= (rc - sw)) return 1.0;
  if (r > rc) return 0.0;
  double rs{PI * (r - rc + sw) / sw};
  double c = (rs > 3.121592653589793) ? cos_near_pi(rs) : std::cos(rs);
  return (0.5 * (1. + c));
}
static double dfc_cos(double r, double rc, double sw) {
  if (r <= (rc - sw)) return 0.0;
  if (r > rc) return 0.0;
  double rs{PI * (r - rc + sw) / sw};
  return (-0.5 * PI / sw * std::sin(rs));
}

/* ------------------------------------------------------------------------ */
// Calculator: GTO radial basis (direct or splined), ShiftedCosine cutoff,
// constant Gaussian smearing.
struct Calculator {
  double rc, sw, sigma, accuracy;
  int nmax, lmax;
  bool use_spline, normalize;
  // RadialScaling cutoff (representations/cutoff_functions.hh:178-280):
  // f_c(r) = u(r) * shifted cosine, u = c / (c + (r/r0)^m)
  bool radial_scaling{false};
  double rs_rate{0.}, rs_scale{1.}, rs_exponent{0.};
  double rs_value(double r) const {
    if (std::abs(rs_rate) <= DBL_FTOL) return 1. / std::pow(r / rs_scale, rs_exponent);
    if (rs_exponent == 0) return 1.;
    return rs_rate / (rs_rate + std::pow(r / rs_scale, rs_exponent));
  }
  double rs_grad(double r) const {
    if (std::abs(rs_rate) <= DBL_FTOL) return -rs_exponent / r / std::pow(r / rs_scale, rs_exponent);
    if (rs_exponent == 0) return 0.;
    double ff = std::pow(r / rs_scale, rs_exponent);
    return -rs_rate * rs_exponent * ff / r / pow_u(rs_rate + ff, 2);
  }
  // the calculator's cutoff function and its derivative (:258-272)
  double f_c(double r) const {
    return radial_scaling ? rs_value(r) * fc_cos(r, rc, sw) : fc_cos(r, rc, sw);
  }
  double df_c(double r) const {
    if (!radial_scaling) return dfc_cos(r, rc, sw);
    return rs_grad(r) * fc_cos(r, rc, sw) + rs_value(r) * dfc_cos(r, rc, sw);
  }
  GTO gto;
  Spline * spline{nullptr};
  std::vector<double> center_final;  // ortho_norm^T * center (spline mode)
  Calculator(double rc_, double sw_, double sigma_, int n, int l, bool spl,
             double acc, bool norm)
      : rc{rc_}, sw{sw_}, sigma{sigma_}, accuracy{acc}, nmax{n}, lmax{l},
        use_spline{spl}, normalize{norm}, gto{n, l, rc_, sigma_} {
    center_final.assign(n, 0.);
    for (int i = 0; i < n; ++i) {
      double s = 0.;
      for (int k = 0; k < n; ++k) s += gto.ortho_norm[k * n + i] * gto.center[k];
      center_final[i] = s;
    }
    if (use_spline) {
      // calculator_spherical_expansion.hh:1107-1135; range starts at
      // SPHERICAL_BESSEL_FUNCTION_FTOL = 1e-5 (math/bessel.hh:42).
      int W = n * (l + 1);
      std::vector<double> tmp(W);
      auto func = [this, W, &tmp](double r, double * out) {
        gto.neighbour(r, false);
        gto.lhs(gto.RI.data(), out, lmax + 1);
        (void)W;
        (void)tmp;
      };
      spline = new Spline(func, 1e-5, rc, accuracy, W);
    }
  }
  ~Calculator() { delete spline; }
  // Orthonormalised radial integral (and derivative) at distance r.
  // Spline mode returns the final coefficients; direct mode returns raw
  // values (orthonormalised later, calculator_spherical_expansion.hh:
  // 1078-1087 vs 588-618).
  void radial(double r, double * RI, double * dRI) {
    int W = nmax * (lmax + 1);
    if (use_spline) {
      spline->interpolate(r, RI);
      if (dRI) spline->derivative(r, dRI);
    } else {
      gto.neighbour(r, dRI != nullptr);
      std::copy(gto.RI.begin(), gto.RI.end(), RI);
      if (dRI) std::copy(gto.dRI.begin(), gto.dRI.end(), dRI);
    }
    (void)W;
  }
};

/* ------------------------------------------------------------------------ */
// Neighbour list: structure_manager_centers.cc:39-94,
// adaptor_neighbour_list.hh:92-437,903-1118, adaptor_center_contribution.hh:
// 333-406, adaptor_strict.hh:373-455.
struct Pair {
  int center;      // centre row within the structure (tag order)
  int j_real;      // original index of the neighbour atom in the structure
  int shift[3];    // periodic image of the neighbour (0 for in-cell atoms)
  double dist;
  double dir[3];
  int j_type;
  bool self;
};

struct StructureNL {
  std::vector<int> center_atoms;  // original index per centre row
  std::vector<Pair> pairs;        // grouped by centre, self pair first
  std::vector<int> pair_offsets;  // n_centers + 1
};

static void inv3(const double m[3][3], double r[3][3]) {
  double c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
  double c10 = m[2][1] * m[0][2] - m[2][2] * m[0][1];
  double c20 = m[0][1] * m[1][2] - m[0][2] * m[1][1];
  double det = c00 * m[0][0] + c10 * m[1][0] + c20 * m[2][0];
  double inv = 1.0 / det;
  r[0][0] = c00 * inv;
  r[0][1] = c10 * inv;
  r[0][2] = c20 * inv;
  r[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * inv;
  r[1][1] = (m[2][2] * m[0][0] - m[2][0] * m[0][2]) * inv;
  r[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv;
  r[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * inv;
  r[2][1] = (m[2][0] * m[0][1] - m[2][1] * m[0][0]) * inv;
  r[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv;
}

static StructureNL build_nl(int N, const double * pos, const int * types,
                            const double * cell_ase, const int * pbc,
                            const unsigned char * mask, double cutoff) {
  // reference cell: columns are lattice vectors
  double cell[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) cell[i][j] = cell_ase[j * 3 + i];
  bool all_zero = true;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (std::fabs(cell[i][j]) >= 1e-10) all_zero = false;
  if (all_zero)
    throw std::runtime_error(
        "The unit cell should not be filled with zeros but it should contain "
        "all the atoms even if the structure is not periodic.");
  for (int a = 0; a < N; ++a)
    if (types[a] >= MAX_CHEM_ELEMENTS || types[a] < 0)
      throw std::runtime_error(
          "atom types (or atomic numbers) should be in the range [0, 130].");
  double cinv[3][3];
  inv3(cell, cinv);
  const double tol_in = 1e-10;
  for (int a = 0; a < N; ++a)
    for (int i = 0; i < 3; ++i) {
      double s = cinv[i][0] * pos[a * 3 + 0] + cinv[i][1] * pos[a * 3 + 1] +
                 cinv[i][2] * pos[a * 3 + 2];
      if (s < -tol_in || s > 1. + tol_in)
        throw std::runtime_error(
            "Some of the atoms in the structure are not inside the unit cell. "
            "Please wrap them inside it with at least tolerance of 1e-10.");
    }
  // tags: centres first, then masked atoms (structure_manager_centers.cc:
  // 50-62); tag -> original index.
  std::vector<int> tag2idx;
  for (int a = 0; a < N; ++a)
    if (!mask || mask[a]) tag2idx.push_back(a);
  int n_centers = int(tag2idx.size());
  for (int a = 0; a < N; ++a)
    if (mask && !mask[a]) tag2idx.push_back(a);

  // mesh and ghost bounds (adaptor_neighbour_list.hh:920-975)
  double mesh_min[3], ghost_min[3], ghost_max[3];
  int nboxes[3];
  for (int i = 0; i < 3; ++i) {
    double min_coord{0.0}, max_coord{0.0};
    for (int col = 0; col < 3; ++col) {
      min_coord += cell[i][col] * static_cast<double>(cell[i][col] < 0.);
      max_coord += cell[i][col] * static_cast<double>(cell[i][col] > 0.);
    }
    mesh_min[i] = min_coord - 2. * cutoff;
    double lmesh{max_coord - min_coord + 4. * cutoff};
    double n{std::ceil(lmesh / cutoff)};
    nboxes[i] = static_cast<int>(n);
    ghost_min[i] = min_coord - cutoff;
    double lghost{max_coord - min_coord + 2 * cutoff};
    double n_ghost_boxes{std::ceil(lghost / cutoff)};
    ghost_max[i] = n_ghost_boxes * cutoff + ghost_min[i];
  }
  double max_box_length = 0.;
  for (int i = 0; i < 3; ++i)
    max_box_length = std::max(max_box_length, ghost_max[i] - ghost_min[i]);
  double bound_tol{max_box_length * 1e-8};
  // multipliers from the 8 corners (adaptor_neighbour_list.hh:981-1010)
  double xmin[3], xmax[3];
  for (int i = 0; i < 3; ++i) {
    xmin[i] = std::numeric_limits<double>::infinity();
    xmax[i] = -std::numeric_limits<double>::infinity();
  }
  for (int corner = 0; corner < 8; ++corner) {
    double x[3];
    for (int i = 0; i < 3; ++i) {
      int hi = (corner >> i) & 1;
      x[i] = hi ? ghost_max[i] + bound_tol : ghost_min[i] - bound_tol;
    }
    for (int i = 0; i < 3; ++i) {
      double s = cinv[i][0] * x[0] + cinv[i][1] * x[1] + cinv[i][2] * x[2];
      xmin[i] = std::min(xmin[i], s);
      xmax[i] = std::max(xmax[i], s);
    }
  }
  int pmin[3], reps[3];
  for (int i = 0; i < 3; ++i) {
    int m_min = int(std::floor(xmin[i]));
    int m_max = int(std::ceil(xmax[i])) - 1;
    int pmax = pbc[i] ? m_max : 0;
    pmin[i] = pbc[i] ? m_min : 0;
    reps[i] = -pmin[i] + pmax + 1;
  }
  int ntot = reps[0] * reps[1] * reps[2];

  // all atoms and ghosts: position, type, original index, shift
  struct Site {
    double x[3];
    int type, idx, shift[3];
  };
  std::vector<Site> sites;
  for (int t = 0; t < N; ++t) {
    int a = tag2idx[t];
    Site s;
    for (int c = 0; c < 3; ++c) s.x[c] = pos[a * 3 + c];
    s.type = types[a];
    s.idx = a;
    s.shift[0] = s.shift[1] = s.shift[2] = 0;
    sites.push_back(s);
  }
  for (int t = 0; t < N; ++t) {
    int a = tag2idx[t];
    for (int k = 0; k < ntot; ++k) {
      int p[3];
      int factor = 1;
      for (int i = 2; i >= 0; --i) {
        p[i] = k / factor % reps[i] + pmin[i];
        if (i != 0) factor *= reps[i];
      }
      if (p[0] == 0 && p[1] == 0 && p[2] == 0) continue;
      double g[3];
      for (int i = 0; i < 3; ++i) {
        double sh = ((cell[i][0] * double(p[0]) + cell[i][1] * double(p[1])) +
                     cell[i][2] * double(p[2]));
        g[i] = pos[a * 3 + i] + sh;
      }
      bool inside = true;
      for (int i = 0; i < 3; ++i) {
        if (!((g[i] - ghost_min[i]) > bound_tol)) inside = false;
        if (!((g[i] - ghost_max[i]) < -bound_tol)) inside = false;
      }
      if (inside) {
        Site s;
        for (int c = 0; c < 3; ++c) s.x[c] = g[c];
        s.type = types[a];
        s.idx = a;
        for (int c = 0; c < 3; ++c) s.shift[c] = p[c];
        sites.push_back(s);
      }
    }
  }
  // binning (adaptor_neighbour_list.hh:1067-1073, 325-336, 398-419)
  size_t nb_total = size_t(nboxes[0]) * nboxes[1] * nboxes[2];
  std::vector<std::vector<int>> boxes(nb_total);
  std::vector<std::array<int, 3>> site_box(sites.size());
  for (size_t s = 0; s < sites.size(); ++s) {
    int b[3];
    for (int i = 0; i < 3; ++i) {
      double d = sites[s].x[i] - mesh_min[i];
      b[i] = std::max(1, static_cast<int>(std::floor(d / cutoff)));
      if (b[i] >= nboxes[i] - 1 || b[i] <= 0)
        throw std::runtime_error(
            "Error: this atom does not fall in one of the linked cell bin. It "
            "might have not been wrapped properly.");
    }
    site_box[s] = {b[0], b[1], b[2]};
    boxes[(size_t(b[0]) * nboxes[1] + b[1]) * nboxes[2] + b[2]].push_back(int(s));
  }
  StructureNL out;
  out.center_atoms.assign(tag2idx.begin(), tag2idx.begin() + n_centers);
  out.pair_offsets.push_back(0);
  double rc2 = cutoff * cutoff;
  for (int ci = 0; ci < n_centers; ++ci) {
    const Site & si = sites[ci];
    // self pair first (adaptor_center_contribution.hh:372-381), then the
    // stencil gather filtered by d^2 <= rc^2 (adaptor_strict.hh:408-437)
    Pair sp;
    sp.center = ci;
    sp.j_real = si.idx;
    sp.shift[0] = sp.shift[1] = sp.shift[2] = 0;
    sp.dist = 0.;
    sp.dir[0] = sp.dir[1] = sp.dir[2] = 0.;
    sp.j_type = si.type;
    sp.self = true;
    out.pairs.push_back(sp);
    auto bi = site_box[ci];
    for (int k = 0; k < 27; ++k) {
      int s0 = k / 9 % 3 + bi[0] - 1;
      int s1 = k / 3 % 3 + bi[1] - 1;
      int s2 = k % 3 + bi[2] - 1;
      const auto & box = boxes[(size_t(s0) * nboxes[1] + s1) * nboxes[2] + s2];
      for (int sj : box) {
        if (sj == ci) continue;
        const Site & so = sites[sj];
        double v[3];
        for (int c = 0; c < 3; ++c) v[c] = so.x[c] - si.x[c];
        double d2 = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
        if (d2 <= rc2) {
          Pair p;
          p.center = ci;
          p.j_real = so.idx;
          for (int c = 0; c < 3; ++c) p.shift[c] = so.shift[c];
          p.dist = std::sqrt(d2);
          if (d2 > 0.) {
            for (int c = 0; c < 3; ++c) p.dir[c] = v[c] / p.dist;
          } else {
            for (int c = 0; c < 3; ++c) p.dir[c] = v[c];
          }
          p.j_type = so.type;
          p.self = false;
          out.pairs.push_back(p);
        }
      }
    }
    out.pair_offsets.push_back(int(out.pairs.size()));
  }
  return out;
}

/* ------------------------------------------------------------------------ */
// A computed batch: neighbour list, expansion, power spectrum and (optional)
// gradients, all dense over the given species list.
struct Run {
  int S{0}, n{0}, L{0}, K{0}, D{0}, n_struct{0};
  std::vector<int> species;
  std::vector<long> atom_off;        // n_struct + 1
  std::vector<int> center_atom;      // global atom index per centre row
  std::vector<int> center_struct;    // structure of each centre row
  std::vector<int> center_type;
  std::vector<long> pair_off;        // n_centers + 1 (global pair rows)
  std::vector<Pair> pairs;           // global; center field = global row
  std::vector<int> pair_jglobal;     // global atom index of the neighbour
  std::vector<double> C, dC;         // expansion: rows x S*n*K; pairs x S*3*n*K
  std::vector<double> X, dX;         // PS: rows x D; pairs x 3*D
  std::vector<double> volume;        // cell volume of each structure
  bool grads{false};
};

// Cell volume as the reference computes it, from the lattice vector lengths
// and the cosines of the angles between them
// (structure_managers/atomic_structure.hh:137-155). `cell` holds the lattice
// vectors as rows.
static double cell_volume(const double * cell) {
  double len[3], v[3][3];
  for (int i = 0; i < 3; ++i) {
    for (int k = 0; k < 3; ++k) v[i][k] = cell[3 * i + k];
    len[i] = std::sqrt(v[i][0] * v[i][0] + v[i][1] * v[i][1] + v[i][2] * v[i][2]);
  }
  auto dot = [&](int a, int b) { return v[a][0] * v[b][0] + v[a][1] * v[b][1] + v[a][2] * v[b][2]; };
  const double al = std::acos(dot(1, 2) / len[1] / len[2]);
  const double be = std::acos(dot(0, 2) / len[0] / len[2]);
  const double ga = std::acos(dot(1, 0) / len[1] / len[0]);
  const double c0 = std::cos(al), c1 = std::cos(be), c2 = std::cos(ga);
  return len[0] * len[1] * len[2] * std::sqrt(1 - c0 * c0 - c1 * c1 - c2 * c2 + 2 * c0 * c1 * c2);
}

static int species_index(const std::vector<int> & sp, int t) {
  auto it = std::lower_bound(sp.begin(), sp.end(), t);
  if (it == sp.end() || *it != t)
    throw std::runtime_error("atom type missing from the species list");
  return int(it - sp.begin());
}

static void compute_run(Calculator & calc, Run & R, const double * pos,
                        const int * types, const double * cells,
                        const int * pbc, const unsigned char * mask) {
  const int n = calc.nmax, L = calc.lmax, K = (L + 1) * (L + 1);
  const int S = int(R.species.size());
  R.S = S;
  R.n = n;
  R.L = L;
  R.K = K;
  R.D = S * (S + 1) / 2 * n * n * (L + 1);
  const int L1 = L + 1, W = n * L1;
  const int nK = n * K;
  SphericalHarmonics sph(L);
  std::vector<double> RI(W), dRI(W), tmp(W);
  R.pair_off.assign(1, 0);
  R.volume.assign(R.n_struct, 0.);
  for (int s = 0; s < R.n_struct; ++s) {
    long a0 = R.atom_off[s], N = R.atom_off[s + 1] - a0;
    R.volume[s] = cell_volume(cells + 9 * s);
    StructureNL nl = build_nl(int(N), pos + a0 * 3, types + a0, cells + 9 * s,
                              pbc + 3 * s, mask ? mask + a0 : nullptr, calc.rc);
    long row0 = long(R.center_atom.size());
    for (size_t c = 0; c < nl.center_atoms.size(); ++c) {
      R.center_atom.push_back(int(a0 + nl.center_atoms[c]));
      R.center_struct.push_back(s);
      R.center_type.push_back(types[a0 + nl.center_atoms[c]]);
      long base = long(R.pairs.size());
      for (int p = nl.pair_offsets[c]; p < nl.pair_offsets[c + 1]; ++p) {
        Pair q = nl.pairs[p];
        q.center = int(row0 + c);
        R.pairs.push_back(q);
        R.pair_jglobal.push_back(int(a0 + q.j_real));
      }
      (void)base;
      R.pair_off.push_back(long(R.pairs.size()));
    }
    if (R.grads && mask) {
      for (long a = 0; a < N; ++a)
        if (!mask[a0 + a])
          throw std::logic_error(
              "Can't compute spherical expansion gradients with masked center "
              "atoms");
    }
  }
  const long NC = long(R.center_atom.size());
  const long NP = long(R.pairs.size());
  R.C.assign(size_t(NC) * S * nK, 0.);
  if (R.grads) R.dC.assign(size_t(NP) * S * 3 * nK, 0.);
  const double inv_sqrt_4pi = 1.0 / std::sqrt(4.0 * PI);
  // expansion, calculator_spherical_expansion.hh:2234-2366
  for (long i = 0; i < NC; ++i) {
    double * Ci = &R.C[size_t(i) * S * nK];
    int ti = species_index(R.species, R.center_type[i]);
    const std::vector<double> & cen = calc.use_spline ? calc.center_final : calc.gto.center;
    for (int nn = 0; nn < n; ++nn) Ci[ti * nK + nn * K + 0] += cen[nn] / std::sqrt(4.0 * PI);
    (void)inv_sqrt_4pi;
    long pself = R.pair_off[i];
    double * dCself = R.grads ? &R.dC[size_t(pself) * S * 3 * nK] : nullptr;
    int center_real = R.center_atom[i];
    for (long p = R.pair_off[i] + 1; p < R.pair_off[i + 1]; ++p) {
      const Pair & pr = R.pairs[p];
      int tj = species_index(R.species, pr.j_type);
      sph.calc(pr.dir, R.grads);
      calc.radial(pr.dist, RI.data(), R.grads ? dRI.data() : nullptr);
      double f_c = calc.f_c(pr.dist);
      double * Cij = Ci + tj * nK;
      int lb = 0;
      for (int l = 0; l < L1; ++l) {
        for (int m = 0; m < 2 * l + 1; ++m)
          for (int nn = 0; nn < n; ++nn)
            Cij[nn * K + lb + m] += (RI[nn * L1 + l] * sph.Y[lb + m]) * f_c;
        lb += 2 * l + 1;
      }
      if (R.grads) {
        double df_c = calc.df_c(pr.dist);
        double * dCp = &R.dC[size_t(p) * S * 3 * nK] + size_t(tj) * 3 * nK;
        double * dCs = dCself + size_t(tj) * 3 * nK;
        bool not_image_of_center = R.pair_jglobal[p] != center_real;
        for (int c = 0; c < 3; ++c) {
          lb = 0;
          for (int l = 0; l < L1; ++l) {
            for (int nn = 0; nn < n; ++nn) {
              double p1 = (dRI[nn * L1 + l] * f_c) + (RI[nn * L1 + l] * df_c);
              for (int m = 0; m < 2 * l + 1; ++m) {
                double g = (p1 * sph.Y[lb + m]) * pr.dir[c] +
                           ((RI[nn * L1 + l] * sph.dY[c * K + lb + m]) * f_c) / pr.dist;
                if (not_image_of_center) dCs[c * nK + nn * K + lb + m] -= g;
                dCp[c * nK + nn * K + lb + m] = g;
              }
            }
            lb += 2 * l + 1;
          }
        }
      }
    }
    if (!calc.use_spline) {
      // finalize_coefficients: C = ortho_norm^T C for every key
      for (int a = 0; a < S; ++a) {
        std::vector<double> blk(Ci + a * nK, Ci + (a + 1) * nK);
        calc.gto.lhs(blk.data(), Ci + a * nK, K);
      }
      if (R.grads) {
        for (long p = R.pair_off[i]; p < R.pair_off[i + 1]; ++p)
          for (int a = 0; a < S; ++a)
            for (int c = 0; c < 3; ++c) {
              double * blk = &R.dC[size_t(p) * S * 3 * nK + size_t(a) * 3 * nK + c * nK];
              std::vector<double> cp(blk, blk + nK);
              calc.gto.lhs(cp.data(), blk, K);
            }
      }
    }
  }
  // power spectrum, calculator_spherical_invariants.hh:747-931
  const int nn2 = n * n;
  const int blk = nn2 * L1;
  std::vector<int> pair_a, pair_b;
  std::vector<std::vector<int>> pair_id(S, std::vector<int>(S, -1));
  for (int a = 0; a < S; ++a)
    for (int b = a; b < S; ++b) {
      pair_id[a][b] = int(pair_a.size());
      pair_a.push_back(a);
      pair_b.push_back(b);
    }
  std::vector<double> lf(L1);
  for (int l = 0; l < L1; ++l) lf[l] = pow_i(std::sqrt(2 * l + 1), -1);
  R.X.assign(size_t(NC) * R.D, 0.);
  if (R.grads) R.dX.assign(size_t(NP) * 3 * R.D, 0.);
  std::vector<double> inv_norm(NC, 1.);
  for (long i = 0; i < NC; ++i) {
    const double * Ci = &R.C[size_t(i) * S * nK];
    double * Xi = &R.X[size_t(i) * R.D];
    // keys of the centre: species with a nonzero block (environment wise)
    std::vector<bool> present(S, false);
    present[species_index(R.species, R.center_type[i])] = true;
    for (long p = R.pair_off[i] + 1; p < R.pair_off[i + 1]; ++p)
      present[species_index(R.species, R.pairs[p].j_type)] = true;
    for (int a = 0; a < S; ++a) {
      if (!present[a]) continue;
      for (int b = a; b < S; ++b) {
        if (!present[b]) continue;
        double * P = Xi + pair_id[a][b] * blk;
        for (int n1 = 0; n1 < n; ++n1)
          for (int n2 = 0; n2 < n; ++n2) {
            int lb = 0;
            for (int l = 0; l < L1; ++l) {
              double s = 0.;
              for (int m = 0; m < 2 * l + 1; ++m)
                s += Ci[a * nK + n1 * K + lb + m] * Ci[b * nK + n2 * K + lb + m];
              double v = s * lf[l];
              if (a < b) v *= SQRT_TWO;
              P[(n1 * n + n2) * L1 + l] = v;
              lb += 2 * l + 1;
            }
          }
      }
    }
    if (calc.normalize) {
      double s = 0.;
      for (int d = 0; d < R.D; ++d) s += Xi[d] * Xi[d];
      double nrm = std::sqrt(s);
      if (std::fabs(nrm) > 0.)
        for (int d = 0; d < R.D; ++d) Xi[d] /= nrm;
      inv_norm[i] = 1. / nrm;
    }
    if (R.grads) {
      for (long p = R.pair_off[i]; p < R.pair_off[i + 1]; ++p) {
        const double * dCp = &R.dC[size_t(p) * S * 3 * nK];
        double * dXp = &R.dX[size_t(p) * 3 * R.D];
        bool self = R.pairs[p].self;
        int tj = species_index(R.species, R.pairs[p].j_type);
        for (int a = 0; a < S; ++a) {  // gradient key
          if (self ? !present[a] : a != tj) continue;
          for (int b = 0; b < S; ++b) {  // centre key
            if (!present[b]) continue;
            int lo = std::min(a, b), hi = std::max(a, b);
            double * G = dXp + pair_id[lo][hi] * blk;
            for (int c = 0; c < 3; ++c) {
              const double * g1 = dCp + size_t(a) * 3 * nK + c * nK;
              const double * c2 = Ci + b * nK;
              for (int n1 = 0; n1 < n; ++n1)
                for (int n2 = 0; n2 < n; ++n2) {
                  int lb = 0;
                  for (int l = 0; l < L1; ++l) {
                    double v = 0.;
                    if (a <= b) {  // grad c^a_{n1} c^b_{n2}
                      double s = 0.;
                      for (int m = 0; m < 2 * l + 1; ++m)
                        s += g1[n1 * K + lb + m] * c2[n2 * K + lb + m];
                      v += s * lf[l];
                    }
                    if (a >= b) {  // c^b_{n1} grad c^a_{n2}
                      double s = 0.;
                      for (int m = 0; m < 2 * l + 1; ++m)
                        s += g1[n2 * K + lb + m] * c2[n1 * K + lb + m];
                      v += s * lf[l];
                    }
                    G[c * R.D + (n1 * n + n2) * L1 + l] += v;
                    lb += 2 * l + 1;
                  }
                }
            }
          }
        }
        for (int k = 0; k < int(pair_a.size()); ++k)
          if (pair_a[k] != pair_b[k])
            for (int c = 0; c < 3; ++c)
              for (int e = 0; e < blk; ++e) dXp[c * R.D + k * blk + e] *= SQRT_TWO;
        if (calc.normalize) {
          // calculator_spherical_invariants.hh:588-652
          for (int e = 0; e < 3 * R.D; ++e) dXp[e] *= inv_norm[i];
          for (int c = 0; c < 3; ++c) {
            double dot = 0.;
            for (int d = 0; d < R.D; ++d) dot += dXp[c * R.D + d] * Xi[d];
            for (int d = 0; d < R.D; ++d) dXp[c * R.D + d] -= dot * Xi[d];
          }
        }
      }
    }
  }
}

// GAP energies and forces, the reference's own algorithm:
// models/sparse_kernels.hh:104-131 (K_NM), models/krr.py:92-121 (energy),
// models/sparse_kernel_predict.hh:70-266 (forces), models/krr.py:123-166.
static double pow_zeta(double v, int zeta) {
  if (zeta == 1) return v;
  if (zeta == 2) return v * v;
  if (zeta == 3) return v * v * v;
  return pow_u(v, size_t(zeta));
}

// The negative stress (Voigt xx, yy, zz, yz, xz, xy) per structure follows
// compute_sparse_kernel_neg_stress (models/sparse_kernel_predict.hh:291-377):
// sum over pairs of r_ji (x) the pair's partial gradient dE_i/dr_j, with the
// off-diagonals taken as yz <- r_y g_z, xz <- r_z g_x, xy <- r_x g_y, divided
// by the cell volume.
static void gap_predict(const Run & R, int M, const int * sp_species,
                        const double * T, const double * alpha, int zeta,
                        double * energies, double * forces, double * neg_stress = nullptr) {
  long NC = long(R.center_atom.size());
  long NA = R.atom_off[R.n_struct];
  for (int s = 0; s < R.n_struct; ++s) energies[s] = 0.;
  if (forces)
    for (long a = 0; a < 3 * NA; ++a) forces[a] = 0.;
  if (neg_stress)
    for (int s = 0; s < 6 * R.n_struct; ++s) neg_stress[s] = 0.;
  std::vector<double> k(M), t(R.D);
  for (long i = 0; i < NC; ++i) {
    const double * Xi = &R.X[size_t(i) * R.D];
    int ti = R.center_type[i];
    double e = 0.;
    std::fill(t.begin(), t.end(), 0.);
    for (int m = 0; m < M; ++m) {
      if (sp_species[m] != ti) continue;
      const double * Tm = T + size_t(m) * R.D;
      double dot = 0.;
      for (int d = 0; d < R.D; ++d) dot += Xi[d] * Tm[d];
      e += alpha[m] * pow_zeta(dot, zeta);
      if (forces) {
        double w = alpha[m] * (zeta * pow_zeta(dot, zeta - 1));
        for (int d = 0; d < R.D; ++d) t[d] += w * Tm[d];
      }
    }
    energies[R.center_struct[i]] += e;
    if (forces) {
      for (long p = R.pair_off[i]; p < R.pair_off[i + 1]; ++p) {
        const double * dXp = &R.dX[size_t(p) * 3 * R.D];
        long j = R.pair_jglobal[p];
        double g[3];
        for (int c = 0; c < 3; ++c) {
          g[c] = 0.;
          for (int d = 0; d < R.D; ++d) g[c] += dXp[c * R.D + d] * t[d];
          forces[3 * j + c] -= g[c];
        }
        if (neg_stress) {
          const Pair & q = R.pairs[p];
          double * ns = neg_stress + 6 * R.center_struct[i];
          const double rji[3] = {-q.dist * q.dir[0], -q.dist * q.dir[1], -q.dist * q.dir[2]};
          ns[0] += rji[0] * g[0];
          ns[4] += rji[2] * g[0];
          ns[1] += rji[1] * g[1];
          ns[5] += rji[0] * g[1];
          ns[2] += rji[2] * g[2];
          ns[3] += rji[1] * g[2];
        }
      }
    }
  }
  if (neg_stress)
    for (int s = 0; s < R.n_struct; ++s)
      for (int k = 0; k < 6; ++k) neg_stress[6 * s + k] /= R.volume[s];
}

// Sparse kernel matrices for training.
//
// K_NM energy rows (models/sparse_kernels.hh:104-131 for target "Structure",
// :165-191 for target "Atom"): k(X_i, T_m) = (X_i . T_m)^zeta for the sparse
// points of the centre's species and 0 for the others, summed over the
// centres of each structure or kept per centre.
static void kernel_nm(const Run & R, int M, const int * sp_species, const double * T, int zeta,
                      bool atom_target, double * out) {
  const long NC = long(R.center_atom.size());
  const long rows = atom_target ? NC : long(R.n_struct);
  std::fill(out, out + size_t(rows) * M, 0.);
  for (long i = 0; i < NC; ++i) {
    const double * Xi = &R.X[size_t(i) * R.D];
    double * row = out + size_t(atom_target ? i : R.center_struct[i]) * M;
    for (int m = 0; m < M; ++m) {
      if (sp_species[m] != R.center_type[i]) continue;
      const double * Tm = T + size_t(m) * R.D;
      double dot = 0.;
      for (int d = 0; d < R.D; ++d) dot += Xi[d] * Tm[d];
      row[m] += pow_zeta(dot, zeta);
    }
  }
}

// K_NM gradient rows (models/sparse_kernels.hh:258-499): three rows (x, y, z)
// per centre, row 3a+c = d/dr_a[c] of sum_i k(X_i, T_m) over the centres i of
// a's structure, accumulated pair by pair as
//   dk[j][c][m] += (dX_i/dr_j[c] . T_m) * zeta (X_i . T_m)^(zeta-1)
// with j the neighbour's real atom. With `neg_stress`, six rows per structure
// follow all centre rows: sum over pairs of r_ji[a] times the pair term for
// component b, in the Voigt order xx, yy, zz, yz (r_y, z), xz (r_z, x),
// xy (r_x, y), divided by the cell volume (:405-425, :470-482).
// A structure none of whose centre species has sparse points ends the loop
// over structures, as the early return at :347-349 does: its rows and those
// of every later structure stay zero.
static void kernel_nm_derivative(const Run & R, int M, const int * sp_species, const double * T,
                                 int zeta, bool neg_stress, double * out) {
  const long NC = long(R.center_atom.size());
  const long rows = 3 * NC + (neg_stress ? 6L * R.n_struct : 0L);
  std::fill(out, out + size_t(rows) * M, 0.);
  const long NA = R.atom_off[R.n_struct];
  std::vector<long> row_of_atom(size_t(NA), -1);
  for (long i = 0; i < NC; ++i) row_of_atom[size_t(R.center_atom[i])] = i;
  std::set<int> sparse_sp(sp_species, sp_species + M);
  std::vector<double> w(static_cast<size_t>(M), 0.);
  long i = 0;
  for (int s = 0; s < R.n_struct; ++s) {
    long i_end = i;
    bool shared = false;
    while (i_end < NC && R.center_struct[i_end] == s) {
      if (sparse_sp.count(R.center_type[i_end])) shared = true;
      ++i_end;
    }
    if (!shared) break;
    double * st = neg_stress ? out + size_t(3 * NC + 6L * s) * M : nullptr;
    for (; i < i_end; ++i) {
      const double * Xi = &R.X[size_t(i) * R.D];
      for (int m = 0; m < M; ++m) {
        w[m] = 0.;
        if (sp_species[m] != R.center_type[i]) continue;
        if (zeta > 1) {
          const double * Tm = T + size_t(m) * R.D;
          double dot = 0.;
          for (int d = 0; d < R.D; ++d) dot += Xi[d] * Tm[d];
          w[m] = double(zeta) * pow_zeta(dot, zeta - 1);
        } else {
          w[m] = 1.;
        }
      }
      for (long p = R.pair_off[i]; p < R.pair_off[i + 1]; ++p) {
        const double * dXp = &R.dX[size_t(p) * 3 * R.D];
        const long rj = row_of_atom[size_t(R.pair_jglobal[p])];
        const Pair & q = R.pairs[p];
        const double rji[3] = {-q.dist * q.dir[0], -q.dist * q.dir[1], -q.dist * q.dir[2]};
        for (int m = 0; m < M; ++m) {
          if (sp_species[m] != R.center_type[i]) continue;
          const double * Tm = T + size_t(m) * R.D;
          for (int c = 0; c < 3; ++c) {
            double v = 0.;
            for (int d = 0; d < R.D; ++d) v += dXp[c * R.D + d] * Tm[d];
            v *= w[m];
            if (rj >= 0) out[size_t(3 * rj + c) * M + m] += v;
            if (st) {
              // xx yy zz from r_ji[c]; then xz (c = x, r_z), xy (c = y, r_x), yz (c = z, r_y)
              static const int voigt_row[3] = {4, 5, 3}, voigt_dim[3] = {2, 0, 1};
              st[size_t(c) * M + m] += rji[c] * v;
              st[size_t(voigt_row[c]) * M + m] += rji[voigt_dim[c]] * v;
            }
          }
        }
      }
    }
    if (st)
      for (int k = 0; k < 6 * M; ++k) st[k] /= R.volume[s];
  }
}

// K_MM (models/sparse_kernels.hh:141-156 with sparse_points.hh:144-170):
// (T_a . T_b)^zeta for two sparse points of one species, 0 across species.
static void kernel_mm(int M, int D, const int * sp_species, const double * T, int zeta, double * out) {
  for (int a = 0; a < M; ++a)
    for (int b = 0; b < M; ++b) {
      double v = 0.;
      if (sp_species[a] == sp_species[b]) {
        double dot = 0.;
        for (int d = 0; d < D; ++d) dot += T[size_t(a) * D + d] * T[size_t(b) * D + d];
        v = pow_zeta(dot, zeta);
      }
      out[size_t(a) * M + b] = v;
    }
}

}  // namespace orc

/* ======================================================================== */
// C interface for ctypes (tests and the CPU baseline only).
extern "C" {

static void set_err(char * err, int errlen, const char * msg) {
  if (err && errlen > 0) {
    std::snprintf(err, size_t(errlen), "%s", msg);
  }
}

double orc_hyp1f1(double a, double b, double z, int der, int mmax, double tol) {
  orc::Hyp1f1 h(a, b, size_t(mmax), tol);
  return h.calc(z, der != 0);
}

int orc_hyp1f1_table(int nmax, int lmax, double r, double alpha,
                     const double * fac_b, int recursion, double tol,
                     double * values, double * derivatives) {
  orc::Hyp1f1SphericalExpansion h(recursion != 0, tol, 200);
  h.precompute(size_t(nmax), size_t(lmax));
  std::vector<double> fb(fac_b, fac_b + nmax);
  h.calc(r, alpha, fb, true);
  std::copy(h.values.begin(), h.values.end(), values);
  std::copy(h.derivatives.begin(), h.derivatives.end(), derivatives);
  return 0;
}

int orc_spherical_harmonics(int lmax, const double * dir, double * Y, double * dY) {
  orc::SphericalHarmonics s(lmax);
  s.calc(dir, dY != nullptr);
  std::copy(s.Y.begin(), s.Y.end(), Y);
  if (dY) std::copy(s.dY.begin(), s.dY.end(), dY);
  return 0;
}

void * orc_calc_new(double rc, double sw, double sigma, int nmax, int lmax,
                    int use_spline, double accuracy, int normalize, char * err,
                    int errlen) {
  try {
    return new orc::Calculator(rc, sw, sigma, nmax, lmax, use_spline != 0,
                               accuracy, normalize != 0);
  } catch (std::exception & e) {
    set_err(err, errlen, e.what());
    return nullptr;
  }
}

void orc_calc_free(void * c) { delete static_cast<orc::Calculator *>(c); }

void orc_calc_set_radial_scaling(void * c, double rate, double scale, double exponent) {
  auto * C = static_cast<orc::Calculator *>(c);
  C->radial_scaling = true;
  C->rs_rate = rate;
  C->rs_scale = scale;
  C->rs_exponent = exponent;
}

int orc_calc_spline_size(void * c) {
  auto * calc = static_cast<orc::Calculator *>(c);
  return calc->spline ? calc->spline->G : 0;
}

int orc_calc_spline_table(void * c, double * grid, double * y, double * y2h) {
  auto * calc = static_cast<orc::Calculator *>(c);
  if (!calc->spline) return -1;
  std::copy(calc->spline->grid.begin(), calc->spline->grid.end(), grid);
  std::copy(calc->spline->y.begin(), calc->spline->y.end(), y);
  std::copy(calc->spline->y2h.begin(), calc->spline->y2h.end(), y2h);
  return 0;
}

int orc_calc_gto(void * c, double * ortho_norm, double * center_final,
                 double * fac_b) {
  auto * calc = static_cast<orc::Calculator *>(c);
  int n = calc->nmax;
  std::copy(calc->gto.ortho_norm.begin(), calc->gto.ortho_norm.end(), ortho_norm);
  std::copy(calc->center_final.begin(), calc->center_final.end(), center_final);
  std::copy(calc->gto.fac_b.begin(), calc->gto.fac_b.end(), fac_b);
  (void)n;
  return 0;
}

int orc_calc_radial(void * c, double r, double * RI, double * dRI) {
  auto * calc = static_cast<orc::Calculator *>(c);
  calc->radial(r, RI, dRI);
  return 0;
}

void * orc_run(void * c, int n_struct, const long * atom_off, const double * pos,
               const int * types, const double * cells, const int * pbc,
               const unsigned char * mask, int n_species, const int * species,
               int grads, char * err, int errlen) {
  auto * calc = static_cast<orc::Calculator *>(c);
  auto * R = new orc::Run();
  try {
    R->n_struct = n_struct;
    R->atom_off.assign(atom_off, atom_off + n_struct + 1);
    R->species.assign(species, species + n_species);
    std::sort(R->species.begin(), R->species.end());
    R->grads = grads != 0;
    orc::compute_run(*calc, *R, pos, types, cells, pbc, mask);
    return R;
  } catch (std::exception & e) {
    set_err(err, errlen, e.what());
    delete R;
    return nullptr;
  }
}

void orc_run_free(void * r) { delete static_cast<orc::Run *>(r); }

long orc_run_n_centers(void * r) {
  return long(static_cast<orc::Run *>(r)->center_atom.size());
}
long orc_run_n_pairs(void * r) {
  return long(static_cast<orc::Run *>(r)->pairs.size());
}
int orc_run_dim(void * r) { return static_cast<orc::Run *>(r)->D; }

int orc_run_centers(void * r, int * center_atom, int * center_struct,
                    long * pair_off) {
  auto * R = static_cast<orc::Run *>(r);
  std::copy(R->center_atom.begin(), R->center_atom.end(), center_atom);
  std::copy(R->center_struct.begin(), R->center_struct.end(), center_struct);
  std::copy(R->pair_off.begin(), R->pair_off.end(), pair_off);
  return 0;
}

int orc_run_pairs(void * r, int * center, int * j_global, int * shift,
                  double * dist, double * dir, int * j_type) {
  auto * R = static_cast<orc::Run *>(r);
  for (size_t p = 0; p < R->pairs.size(); ++p) {
    const auto & q = R->pairs[p];
    center[p] = q.center;
    j_global[p] = R->pair_jglobal[p];
    for (int c = 0; c < 3; ++c) {
      shift[3 * p + c] = q.shift[c];
      dir[3 * p + c] = q.dir[c];
    }
    dist[p] = q.dist;
    j_type[p] = q.j_type;
  }
  return 0;
}

int orc_run_expansion(void * r, double * out) {
  auto * R = static_cast<orc::Run *>(r);
  std::copy(R->C.begin(), R->C.end(), out);
  return 0;
}
int orc_run_expansion_grad(void * r, double * out) {
  auto * R = static_cast<orc::Run *>(r);
  if (!R->grads) return -1;
  std::copy(R->dC.begin(), R->dC.end(), out);
  return 0;
}
int orc_run_powerspectrum(void * r, double * out) {
  auto * R = static_cast<orc::Run *>(r);
  std::copy(R->X.begin(), R->X.end(), out);
  return 0;
}
int orc_run_powerspectrum_grad(void * r, double * out) {
  auto * R = static_cast<orc::Run *>(r);
  if (!R->grads) return -1;
  std::copy(R->dX.begin(), R->dX.end(), out);
  return 0;
}

int orc_run_gap(void * r, int M, const int * sp_species, const double * T,
                const double * alpha, int zeta, double * energies,
                double * forces) {
  auto * R = static_cast<orc::Run *>(r);
  if (forces && !R->grads) return -1;
  orc::gap_predict(*R, M, sp_species, T, alpha, zeta, energies, forces);
  return 0;
}

int orc_run_gap_stress(void * r, int M, const int * sp_species, const double * T,
                       const double * alpha, int zeta, double * energies,
                       double * forces, double * neg_stress) {
  auto * R = static_cast<orc::Run *>(r);
  if (!R->grads || !forces || !neg_stress) return -1;
  orc::gap_predict(*R, M, sp_species, T, alpha, zeta, energies, forces, neg_stress);
  return 0;
}


int orc_run_kernel_nm(void * r, int M, const int * sp_species, const double * T, int zeta,
                      int atom_target, double * out) {
  orc::kernel_nm(*static_cast<orc::Run *>(r), M, sp_species, T, zeta, atom_target != 0, out);
  return 0;
}

int orc_run_kernel_nm_derivative(void * r, int M, const int * sp_species, const double * T, int zeta,
                                 int neg_stress, double * out) {
  auto * R = static_cast<orc::Run *>(r);
  if (!R->grads) return -1;
  orc::kernel_nm_derivative(*R, M, sp_species, T, zeta, neg_stress != 0, out);
  return 0;
}

int orc_kernel_mm(int M, int D, const int * sp_species, const double * T, int zeta, double * out) {
  orc::kernel_mm(M, D, sp_species, T, zeta, out);
  return 0;
}

}  // extern "C"
