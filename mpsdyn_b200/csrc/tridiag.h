// Lowest eigenpair of a real symmetric tridiagonal matrix (the projected
// Rayleigh-Ritz problem of the Lanczos iteration, kept in FP64 on the host:
// k <= 256, O(k) per bisection step).
//
// Eigenvalue: bisection on the Gershgorin interval with Sturm-sequence
// counts (the number of negative pivots of the LDL^T factorisation of
// T - x I equals the number of eigenvalues below x; Wilkinson, "The
// Algebraic Eigenvalue Problem", 5.38).  Eigenvector: inverse iteration
// on T - theta I with a row-pivoted tridiagonal elimination.
#pragma once

#include <algorithm>
#include <cmath>
#include <vector>

namespace mpsgpu {

struct TridiagLowest {
  std::vector<double> d, u, u2, sub, y;

  static int count_below(const std::vector<double>& a, const std::vector<double>& b, int k, double x) {
    int cnt = 0;
    double q = a[0] - x;
    if (q < 0) cnt++;
    for (int i = 1; i < k; i++) {
      const double den = (q == 0.0) ? 1e-300 : q;
      q = a[i] - x - b[i - 1] * b[i - 1] / den;
      if (q < 0) cnt++;
    }
    return cnt;
  }

  // a: diagonal (k), b: off-diagonal (b[i] couples i and i+1; b[k-1] unused).
  void solve(const std::vector<double>& a, const std::vector<double>& b, int k, double& theta,
             std::vector<double>& s, double& normT) {
    double lo = a[0], hi = a[0];
    for (int i = 0; i < k; i++) {
      const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i < k - 1 ? std::fabs(b[i]) : 0.0);
      lo = std::min(lo, a[i] - r);
      hi = std::max(hi, a[i] + r);
    }
    normT = std::max(std::fabs(lo), std::fabs(hi));
    double l = lo, h = hi;
    for (int it = 0; it < 200; it++) {
      if (!(h - l > 4e-16 * std::max(std::fabs(l), std::fabs(h)) + 1e-300)) break;
      const double mid = 0.5 * (l + h);
      if (mid == l || mid == h) break;
      if (count_below(a, b, k, mid) >= 1) h = mid;
      else l = mid;
    }
    theta = 0.5 * (l + h);
    s.assign(k, 1.0);
    if (k == 1) return;
    const double shift = theta - 1e-14 * std::max(normT, 1e-300);
    const double tiny = 1e-15 * std::max(normT, 1e-300);
    d.resize(k); u.resize(k); u2.resize(k); sub.resize(k); y.resize(k);
    for (int rep = 0; rep < 3; rep++) {
      for (int i = 0; i < k; i++) {
        d[i] = a[i] - shift;
        u[i] = (i < k - 1) ? b[i] : 0.0;
        sub[i] = (i < k - 1) ? b[i] : 0.0;
        u2[i] = 0.0;
        y[i] = s[i];
      }
      for (int i = 0; i < k - 1; i++) {
        if (std::fabs(sub[i]) > std::fabs(d[i])) {
          // pivot: row i+1 becomes row i
          const double nd = sub[i], nu = d[i + 1], nu2 = (i + 1 < k - 1) ? u[i + 1] : 0.0;
          const double od = d[i], ou = u[i], ou2 = u2[i];
          d[i] = nd; u[i] = nu; u2[i] = nu2;
          std::swap(y[i], y[i + 1]);
          const double m = od / nd;
          d[i + 1] = ou - m * nu;
          u[i + 1] = ou2 - m * nu2;
          y[i + 1] -= m * y[i];
        } else {
          const double den = (std::fabs(d[i]) < tiny) ? tiny : d[i];
          const double m = sub[i] / den;
          d[i + 1] -= m * u[i];
          if (i + 1 < k - 1) u[i + 1] -= m * u2[i];
          y[i + 1] -= m * y[i];
        }
      }
      for (int i = k - 1; i >= 0; i--) {
        double acc = y[i];
        if (i + 1 < k) acc -= u[i] * y[i + 1];
        if (i + 2 < k) acc -= u2[i] * y[i + 2];
        const double den = (std::fabs(d[i]) < tiny) ? tiny : d[i];
        y[i] = acc / den;
      }
      double nrm = 0.0;
      for (int i = 0; i < k; i++) nrm += y[i] * y[i];
      nrm = std::sqrt(nrm);
      for (int i = 0; i < k; i++) s[i] = y[i] / nrm;
    }
  }
};

}  // namespace mpsgpu
