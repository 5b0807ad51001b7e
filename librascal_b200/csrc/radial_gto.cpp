// Host-side FP64 construction of the GTO radial basis table.
//
// The expansion kernels read the orthonormalised GTO radial integral
// RI_nl(r) and its derivative from a natural cubic spline. This file builds
// that spline once per calculator, on the host and in FP64, exactly as the
// reference does (it is part of calculator construction there too):
//   * 1F1 series / asymptotic forms and the switching point:
//       src/rascal/math/hyp1f1.cc:51-356
//   * the (n,l) table by downward recursion in l:   hyp1f1.cc:395-457
//   * GTO sigmas, norms, overlap, S^-1/2:
//       representations/calculator_spherical_expansion.hh:404-680
//   * neighbour radial integral: calculator_spherical_expansion.hh:518-557
//   * spline refinement: math/interpolator.hh:167-185,705-712,1230-1248;
//     second derivatives and the grid search: math/interpolator.cc:148-230.
// Floating point follows the reference's evaluation order; the build adds
// -ffp-contract=off so that the table is reproducible bit for bit.
#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <vector>

#include "rgpu_internal.h"

namespace rgpu {
namespace {

constexpr double kFtol = 100.0 * std::numeric_limits<double>::epsilon();
constexpr double kInf = std::numeric_limits<double>::infinity();

double upow(double x, size_t n) {
  double v{1};
  do {
    if (n & 1) v *= x;
    n >>= 1;
    x *= x;
  } while (n);
  return v;
}
double ipow(double x, int n) {
  if (n < 0) return upow(1.0 / x, size_t(-n));
  return upow(x, size_t(n));
}

// Power series of 1F1(a, b, z), terms summed four at a time.
class Series {
 public:
  Series(double a, double b, size_t mmax, double tol)
      : a_(a), b_(b), mmax_(mmax), tol_(tol),
        prefac_(std::tgamma(a) / std::tgamma(b)) {
    exp_ = std::fabs(1 - b / a) < kFtol;
    if (!exp_) {
      c_.resize(mmax);
      cd_.resize(mmax);
      c_[0] = a / b;
      cd_[0] = (a + 1) / (b + 1);
      for (size_t i = 1; i < mmax; ++i) {
        double u = (a + i) / ((i + 1) * (b + i));
        c_[i] = c_[i - 1] * u;
        u = (a + i + 1) / ((i + 1) * (b + i + 1));
        cd_[i] = cd_[i - 1] * u;
      }
    }
  }
  double f(double z, bool der) const {
    if (exp_) return std::exp(z);
    return der ? sum(z, cd_) * a_ / b_ : sum(z, c_);
  }
  double g(double z, double z2, double ez2, bool der) const {
    if (exp_) return prefac_ * std::exp(z + z2);
    return prefac_ * f(z, der) * ez2;
  }

 private:
  double sum(double z, const std::vector<double> & c) const {
    double res = 1.0, zp = z, z4 = z * z;
    z4 *= z4;
    for (size_t i = 0; i < mmax_ - 3; i += 4) {
      double t = zp * (c[i] + z * (c[i + 1] + z * (c[i + 2] + z * c[i + 3])));
      if (t < tol_ * res) {
        res += t;
        break;
      }
      zp *= z4;
      res += t;
    }
    if (res > kInf) throw Error(RGPU_ERR_OVERFLOW, "Hyp1f1Series overflow");
    return res;
  }
  double a_, b_;
  size_t mmax_;
  double tol_, prefac_;
  bool exp_;
  std::vector<double> c_, cd_;
};

// Asymptotic (2F0) form of 1F1(a, b, z) for large z.
class Asymptotic {
 public:
  Asymptotic(double a, double b, size_t mmax, double tol)
      : a_(a), b_(b), mmax_(mmax), tol_(tol),
        prefac_(std::tgamma(b) / std::tgamma(a)) {
    double ip;
    int_power_ = std::fabs(std::modf(2 * (a - b), &ip)) < 1e-14;
    exp_ = std::fabs(1 - b / a) < kFtol;
    if (!exp_) {
      c_.resize(mmax);
      cd_.resize(mmax);
      double bma = b - a, oma = 1 - a, oma1 = 1 - a - 1;
      c_[0] = bma * oma;
      cd_[0] = bma * oma1;
      for (size_t i = 1; i < mmax; ++i) {
        double u = (bma + i) * (oma + i) / (i + 1);
        c_[i] = c_[i - 1] * u;
        u = (bma + i) * (oma1 + i) / (i + 1);
        cd_[i] = cd_[i - 1] * u;
      }
    }
  }
  double f(double z, bool der) const {
    if (exp_) return std::exp(z);
    double r = prefac_ * std::exp(z) * zab(z) * sum(z, der ? cd_ : c_);
    return std::isnan(r) ? kInf : r;
  }
  double g(double z, double z2, bool der) const {
    if (exp_) return std::exp(z + z2) / prefac_;
    double fac = zab(z);
    return sum(z, der ? cd_ : c_) * std::exp(z + z2) * fac;
  }

 private:
  double zab(double z) const {
    if (int_power_) return std::sqrt(ipow(z, static_cast<int>(2 * (a_ - b_))));
    return std::pow(z, a_ - b_);
  }
  double sum(double z, const std::vector<double> & c) const {
    double iz = 1.0 / z, res = 1., izp = 1.;
    for (size_t i = 0; i < mmax_; ++i) {
      izp *= iz;
      double s = c[i] * izp;
      if (res > 0 && std::fabs(s) < tol_ * res) break;
      res += s;
    }
    if (res > kInf) throw Error(RGPU_ERR_OVERFLOW, "Hyp1f1Asymptotic overflow");
    return res;
  }
  double a_, b_;
  size_t mmax_;
  double tol_, prefac_;
  bool int_power_, exp_;
  std::vector<double> c_, cd_;
};

// 1F1 with the series/asymptotic switching point found by bracketing and
// bisection on the relative agreement of the two forms.
class Hyp1f1 {
 public:
  Hyp1f1(double a, double b, size_t mmax, double tol)
      : s_(a, b, mmax, tol), as_(a, b, mmax, tol), tol_(tol) {
    if (std::fabs(1 - b / a) > kFtol) {
      locate_switch();
      probe();
    }
  }
  double g(double z, double z2, double ez2, bool der) const {
    return z > zs_ ? as_.g(z, z2, der) : s_.g(z, z2, ez2, der);
  }

 private:
  void probe() {
    hs_ = s_.f(zs_, false);
    ha_ = as_.f(zs_, false);
  }
  double mismatch() const { return std::fabs(1 - hs_ / ha_); }
  void locate_switch() {
    const int max_it = 100;
    probe();
    double lo = zs_, hi = zs_;
    int it = 0;
    if (mismatch() > tol_) {
      while (mismatch() > 100 * tol_ && it < max_it) {
        zs_ *= 1.5;
        probe();
        ++it;
      }
      hi = zs_;
    } else {
      while (mismatch() < 100 * tol_ && it < max_it) {
        zs_ *= 0.5;
        probe();
        ++it;
      }
      lo = zs_;
    }
    zs_ = (hi + lo) * 0.5;
    probe();
    it = 0;
    while (hi - lo > tol_ && it < max_it) {
      if (std::fabs(1 - hs_ / ha_) > tol_)
        lo = zs_;
      else
        hi = zs_;
      zs_ = (hi + lo) * 0.5;
      probe();
      ++it;
    }
  }
  Series s_;
  Asymptotic as_;
  double tol_, zs_{1.}, hs_{0}, ha_{0};
};

// Symmetric eigen-decomposition (cyclic Jacobi) for the small GTO overlap.
void sym_eigen(int n, std::vector<double> A, std::vector<double> & w,
               std::vector<double> & V) {
  V.assign(size_t(n) * n, 0.);
  for (int i = 0; i < n; ++i) V[i * n + i] = 1.;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[p * n + q] * A[p * n + q];
    if (off < 1e-300) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p * n + q];
        if (apq == 0.) continue;
        double th = (A[q * n + q] - A[p * n + p]) / (2. * apq);
        double t = (th >= 0 ? 1. : -1.) / (std::fabs(th) + std::sqrt(th * th + 1.));
        double c = 1. / std::sqrt(t * t + 1.), s = t * c;
        for (int k = 0; k < n; ++k) {
          double x = A[k * n + p], y = A[k * n + q];
          A[k * n + p] = c * x - s * y;
          A[k * n + q] = s * x + c * y;
        }
        for (int k = 0; k < n; ++k) {
          double x = A[p * n + k], y = A[q * n + k];
          A[p * n + k] = c * x - s * y;
          A[q * n + k] = s * x + c * y;
        }
        for (int k = 0; k < n; ++k) {
          double x = V[k * n + p], y = V[k * n + q];
          V[k * n + p] = c * x - s * y;
          V[k * n + q] = s * x + c * y;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = A[i * n + i];
}

std::vector<double> linspace(int num, double lo, double hi) {
  std::vector<double> v(num);
  if (num == 1) {
    v[0] = hi;
    return v;
  }
  double step = (hi - lo) / double(num - 1);
  bool flip = std::fabs(hi) < std::fabs(lo);
  for (int i = 0; i < num; ++i) {
    if (flip)
      v[i] = (i == 0) ? lo : (hi - double(num - 1 - i) * step);
    else
      v[i] = (i == num - 1) ? hi : (lo + double(i) * step);
  }
  return v;
}

// GTO radial integrals for one calculator.
class GtoBasis {
 public:
  GtoBasis(int n, int l, double rc, double sigma) : n_(n), l_(l) {
    fa_ = 0.5 * ipow(sigma, -2);
    std::vector<double> sig(n);
    fb_.resize(n);
    std::vector<double> norm(n), nfac(n);
    for (int i = 0; i < n; ++i) {
      sig[i] = std::max(std::sqrt(double(i)), 1.0) * rc / double(n);
      fb_[i] = 0.5 * ipow(sig[i], -2);
      norm[i] = 0.25 * std::sqrt(2.0 / (std::tgamma(1.5 + i) * upow(sig[i], 3 + 2 * size_t(i))));
      nfac[i] = std::tgamma(0.5 * (3.0 + i)) / std::tgamma(1.5);
    }
    std::vector<double> S(size_t(n) * n);
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b)
        S[a * n + b] = std::pow(0.5 / ipow(sig[a], 2) + 0.5 / ipow(sig[b], 2),
                                -0.5 * (3.0 + a + b)) /
                       (upow(sig[a], size_t(a)) * upow(sig[b], size_t(b))) *
                       std::tgamma(0.5 * (3.0 + a + b)) /
                       (std::pow(sig[a] * sig[b], 1.5) *
                        std::sqrt(std::tgamma(1.5 + a) * std::tgamma(1.5 + b)));
    std::vector<double> w, V;
    sym_eigen(n, S, w, V);
    on_.assign(size_t(n) * n, 0.);  // diag(norm) * S^-1/2
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double s = 0.;
        for (int k = 0; k < n; ++k) s += V[i * n + k] * (1. / std::sqrt(w[k])) * V[j * n + k];
        on_[i * n + j] = norm[i] * s;
      }
    // Centre contribution (1F1(a,b,0) = 1), orthonormalised.
    std::vector<double> cen(n);
    for (int i = 0; i < n; ++i) {
      double v;
      if (i % 2 == 0)
        v = std::sqrt(ipow(fa_ + fb_[i], -1 * static_cast<int>(3 + i)));
      else
        v = ipow(fa_ + fb_[i], -1 * static_cast<int>(3 + i) / 2);
      cen[i] = nfac[i] * v;
    }
    center_.assign(n, 0.);
    for (int i = 0; i < n; ++i) {
      double s = 0.;
      for (int k = 0; k < n; ++k) s += on_[k * n + i] * cen[k];
      center_[i] = s;
    }
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < l + 1; ++b)
        h_.emplace_back(0.5 * (a + b + 3), b + 1.5, 200, 1e-13);
  }
  const std::vector<double> & center() const { return center_; }

  // out[n][l] = (ortho_norm^T * RI(r))[n][l]
  void eval(double r, double * out) const {
    const int L1 = l_ + 1;
    std::vector<double> dfal(L1), abl(n_), G(size_t(n_) * L1), raw(size_t(n_) * L1);
    dfal[0] = 1.;
    double dfa = r * fa_;
    for (int l = 1; l < L1; ++l) dfal[l] = dfal[l - 1] * dfa;
    for (int i = 0; i < n_; ++i) abl[i] = 1.0 / std::sqrt(fa_ + fb_[i]);
    gvalues(r, G.data());
    for (int i = 0; i < n_; ++i) {
      double ab = upow(abl[i], 3 + size_t(i));
      for (int l = 0; l < L1; ++l) {
        if (l > 0) ab = ab * abl[i];
        raw[i * L1 + l] = (ab * G[i * L1 + l]) * dfal[l];
      }
    }
    for (int i = 0; i < n_; ++i)
      for (int l = 0; l < L1; ++l) {
        double s = 0.;
        for (int k = 0; k < n_; ++k) s += on_[k * n_ + i] * raw[k * L1 + l];
        out[i * L1 + l] = s;
      }
  }

 private:
  // Modified 1F1 values G_nl(r); downward recursion in l when l_max >= 3.
  void gvalues(double r, double * G) const {
    const int L1 = l_ + 1;
    double ar = fa_ * r;
    double z2 = -r * ar;
    double ez2 = std::exp(z2);
    for (int i = 0; i < n_; ++i) {
      double z = (ar * fa_) * (1.0 / (fa_ + fb_[i]));
      z *= r;
      if (l_ < 3) {
        for (int l = 0; l < L1; ++l) G[i * L1 + l] = h_[i * L1 + l].g(z, z2, ez2, false);
        continue;
      }
      auto A = [](int nn, int ll) { return 0.5 * (nn + ll + 3); };
      auto B = [](int ll) { return ll + 1.5; };
      int l = l_;
      double v1 = h_[i * L1 + l].g(z, z2, ez2, false);
      double d1 = h_[i * L1 + l].g(z, z2, ez2, true);
      double v2 = h_[i * L1 + l - 1].g(z, z2, ez2, false);
      double d2 = h_[i * L1 + l - 1].g(z, z2, ez2, true);
      G[i * L1 + l] = v1;
      G[i * L1 + l - 1] = v2;
      for (l -= 2; l > 0; l -= 2) {
        double a = A(i, l), b = B(l);
        double dd = z * d1 + v1 * (b + 1);
        double vv = (z * (a - b) * v1 + dd * b) / a;
        G[i * L1 + l] = vv;
        d1 = dd;
        v1 = vv;
        a = A(i, l - 1);
        b = B(l - 1);
        dd = z * d2 + v2 * (b + 1);
        vv = (z * (a - b) * v2 + dd * b) / a;
        G[i * L1 + l - 1] = vv;
        d2 = dd;
        v2 = vv;
      }
      if (l_ % 2 == 0) {
        double a = A(i, 0), b = B(0);
        double dd = z * d1 + v1 * (b + 1);
        G[i * L1 + 0] = (z * (a - b) * v1 + dd * b) / a;
      }
    }
  }
  int n_, l_;
  double fa_;
  std::vector<double> fb_, on_, center_;
  std::vector<Hyp1f1> h_;
};

}  // namespace

// Natural cubic spline of the orthonormalised radial integral over
// [1e-5, r_c], refined by doubling until the mean absolute error on the
// interval midpoints is below `accuracy`.
void build_radial_spline(const Hypers & hy, RadialSpline & out) {
  GtoBasis gto(hy.max_radial, hy.max_angular, hy.cutoff, hy.sigma);
  const int W = hy.max_radial * (hy.max_angular + 1);
  const double x1 = 1e-5, x2 = hy.cutoff;
  out.width = W;
  out.center = gto.center();
  int dof = 5;
  const int max_points = 100000;
  std::vector<double> vi(W), ve(W);
  while (true) {
    int G = 2 << dof;
    std::vector<double> grid = linspace(G, x1, x2);
    std::vector<double> y(size_t(G) * W);
    for (int i = 0; i < G; ++i) gto.eval(grid[i], &y[size_t(i) * W]);
    double h = grid[1] - grid[0];
    double hh6 = h * h / 6.0;
    // tridiagonal sweep for y'' with y''(x1) = y''(x2) = 0
    std::vector<double> y2(size_t(G) * W, 0.), u(size_t(G) * W, 0.);
    for (int i = 1; i < G - 1; ++i)
      for (int c = 0; c < W; ++c) {
        double p = 0.5 * y2[size_t(i - 1) * W + c] + 2.0;
        y2[size_t(i) * W + c] = (0.5 - 1.0) / p;
        double uu = (3. * (y[size_t(i + 1) * W + c] - 2 * y[size_t(i) * W + c] +
                           y[size_t(i - 1) * W + c])) /
                    (h * h);
        uu -= 0.5 * u[size_t(i - 1) * W + c];
        u[size_t(i) * W + c] = uu / p;
      }
    for (int c = 0; c < W; ++c) y2[size_t(G - 1) * W + c] = 0.;
    for (int k = G - 2; k > 0; --k)
      for (int c = 0; c < W; ++c)
        y2[size_t(k) * W + c] = y2[size_t(k) * W + c] * y2[size_t(k + 1) * W + c] + u[size_t(k) * W + c];
    for (int c = 0; c < W; ++c) y2[c] = 0.;
    for (auto & v : y2) v *= hh6;
    out.grid = grid;
    out.y = y;
    out.y2h = y2;
    out.grid_size = G;
    out.x1 = grid[0];
    out.h = h;
    out.points_per_unit = G / (grid[G - 1] - grid[0]);
    out.search_size = G - 2;
    // mean absolute error at the midpoints
    int tn = 2 << std::max(dof, 5);
    double off = (x2 - x1) / (2 * (tn - 1));
    std::vector<double> test = linspace(tn - 1, x1 + off, x2 - off);
    double err = 0.;
    for (double x : test) {
      out.interpolate(x, vi.data());
      gto.eval(x, ve.data());
      for (int c = 0; c < W; ++c) err += std::fabs(vi[c] - ve[c]);
    }
    err /= double(test.size() * size_t(W));
    if (err < hy.spline_accuracy || G >= max_points) break;
    ++dof;
  }
}

void RadialSpline::interpolate(double x, double * o) const {
  int k = std::max(0, std::min(search_size, static_cast<int>((x - x1) * points_per_unit) - 1));
  double a = (grid[k + 1] - x) / h;
  double b = 1 - a;
  const double *y0 = &y[size_t(k) * width], *y1 = y0 + width;
  const double *d0 = &y2h[size_t(k) * width], *d1 = d0 + width;
  for (int c = 0; c < width; ++c)
    o[c] = a * (y0[c] + (a * a - 1) * d0[c]) + b * (y1[c] + (b * b - 1) * d1[c]);
}

}  // namespace rgpu
