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
#include <cstdint>
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
    invit(a, b, k, theta - 1e-14 * std::max(normT, 1e-300), 1e-15 * std::max(normT, 1e-300), s);
  }

  // As solve(), with the bracket started below an upper bound `ub` of the
  // lowest eigenvalue (the lowest Ritz value of the previous step: by
  // Cauchy interlacing the lowest eigenvalue of T_k is at most that of
  // T_{k-1}) at a guessed distance `step`, widened until the Sturm count
  // shows no eigenvalue below it; bisection then needs only the steps that
  // the bracket's width calls for.  Falls back to the Gershgorin interval.
  void solve_from(const std::vector<double>& a, const std::vector<double>& b, int k, double ub, double step,
                  double& theta, std::vector<double>& s, double& normT) {
    double lo = a[0], hi = a[0];
    for (int i = 0; i < k; i++) {
      const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i < k - 1 ? std::fabs(b[i]) : 0.0);
      lo = std::min(lo, a[i] - r);
      hi = std::max(hi, a[i] + r);
    }
    normT = std::max(std::fabs(lo), std::fabs(hi));
    double h = std::min(hi, ub + 8e-16 * normT);
    if (!(std::isfinite(h) && count_below(a, b, k, h) >= 1)) h = hi;
    double st = std::max(std::fabs(step), 1e-15 * normT);
    double l = lo;
    for (int it = 0; it < 64; it++) {
      const double cand = h - st;
      if (!(cand > lo)) break;
      if (count_below(a, b, k, cand) == 0) {
        l = cand;
        break;
      }
      h = cand;  // still an upper bound
      st *= 16.0;
    }
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
    invit(a, b, k, theta - 1e-14 * std::max(normT, 1e-300), 1e-15 * std::max(normT, 1e-300), s);
  }

  // Three steps of inverse iteration on T - shift I from the start vector s
  // (overwritten by the normalised result).
  void invit(const std::vector<double>& a, const std::vector<double>& b, int k, double shift, double tiny,
             std::vector<double>& s) {
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

// i-th smallest eigenvalue (0-based) of the k x k tridiagonal (a, b) by
// bisection on the Sturm counts.
inline double tridiag_eigenvalue(const std::vector<double>& a, const std::vector<double>& b, int k, int i) {
  double lo = a[0], hi = a[0];
  for (int r = 0; r < k; r++) {
    const double rad = (r > 0 ? std::fabs(b[r - 1]) : 0.0) + (r < k - 1 ? std::fabs(b[r]) : 0.0);
    lo = std::min(lo, a[r] - rad);
    hi = std::max(hi, a[r] + rad);
  }
  for (int it = 0; it < 200; it++) {
    if (!(hi - lo > 4e-16 * std::max(std::fabs(lo), std::fabs(hi)) + 1e-300)) break;
    const double mid = 0.5 * (lo + hi);
    if (mid == lo || mid == hi) break;
    if (TridiagLowest::count_below(a, b, k, mid) >= i + 1) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

// Thick restart of the Lanczos factorisation H V = V T + f e_m^T (Wu &
// Simon, "Thick-restart Lanczos method for large symmetric eigenvalue
// problems", SIAM J. Matrix Anal. Appl. 22, 2000), kept in tridiagonal form:
//   1. Y (m x keep): orthonormal approximations of the keep lowest Ritz
//      vectors of T (bisection + inverse iteration + modified Gram-Schmidt);
//   2. B = Y^T T Y and the coupling s = |f| Y^T e_m, both exact for this Y;
//   3. Lanczos on the small matrix B from s / |s| with full
//      reorthogonalisation gives Z with Z^T B Z tridiagonal and
//      Z^T s = |s| e_1; the order is reversed so that the last kept vector
//      carries the coupling.
// With G = Y Z (reversed), H (V G) = (V G) T' + (f / |f|) |s| e_r^T plus
// terms in span(V) that the continued reorthogonalised Lanczos absorbs; the
// relation holds for any orthonormal Y, so near-degenerate Ritz values only
// cost filtering quality, never consistency.  (Exact-shift implicit QR,
// the alternative, is not forward stable when converged Ritz values are
// used as shifts: Parlett & Le, SIAM J. Matrix Anal. Appl. 14, 1993.)
struct ThickRestart {
  TridiagLowest tri;
  std::vector<double> Y, TY, B, Z, w, s, v;

  // v -= Y[:, 0..i) Y[:, 0..i)^T v, twice
  void project_out(int m, int i) {
    for (int pass = 0; pass < 2; pass++)
      for (int q = 0; q < i; q++) {
        const double* yq = &Y[(size_t)q * m];
        double dot = 0.0;
        for (int r = 0; r < m; r++) dot += yq[r] * v[r];
        for (int r = 0; r < m; r++) v[r] -= dot * yq[r];
      }
  }

  double norm2(int m) const {
    double nrm = 0.0;
    for (int r = 0; r < m; r++) nrm += v[r] * v[r];
    return std::sqrt(nrm);
  }

  // a, b: T (m); fnorm = |f|.  Out: r kept vectors, a', b' (b'[r-1] = |s|,
  // the coupling to f / |f|), G (m x r, column-major).  Returns r.
  int compress(std::vector<double>& a, std::vector<double>& b, int m, int keep, double fnorm,
               std::vector<double>& G) {
    double lo = a[0], hi = a[0];
    for (int r = 0; r < m; r++) {
      const double rad = (r > 0 ? std::fabs(b[r - 1]) : 0.0) + (r < m - 1 ? std::fabs(b[r]) : 0.0);
      lo = std::min(lo, a[r] - rad);
      hi = std::max(hi, a[r] + rad);
    }
    const double normT = std::max(std::max(std::fabs(lo), std::fabs(hi)), 1e-300);
    Y.assign((size_t)m * keep, 0.0);
    v.assign(m, 0.0);
    double prev = 0.0;
    for (int i = 0; i < keep; i++) {
      double lam = tridiag_eigenvalue(a, b, m, i);
      // separate repeated values so that inverse iteration can tell them apart
      if (i > 0 && lam - prev < 1e-12 * normT) lam = prev + 1e-12 * normT;
      prev = lam;
      uint64_t z = 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
      for (int r = 0; r < m; r++) {  // deterministic, distinct start vectors
        z ^= z >> 31; z *= 0xBF58476D1CE4E5B9ull; z ^= z >> 29;
        v[r] = 1.0 + (double)(z >> 11) * (1.0 / 9007199254740992.0);
      }
      tri.invit(a, b, m, lam - 1e-14 * normT, 1e-15 * normT, v);
      project_out(m, i);
      double nrm = norm2(m);
      for (int e = 0; e < m && !(nrm > 1e-8); e++) {
        // lost to the previous vectors: take a unit vector instead
        for (int r = 0; r < m; r++) v[r] = (r == (e + i) % m) ? 1.0 : 0.0;
        project_out(m, i);
        nrm = norm2(m);
      }
      for (int r = 0; r < m; r++) Y[(size_t)i * m + r] = v[r] / nrm;
    }
    // B = Y^T T Y (symmetrised), s = |f| Y^T e_m
    TY.assign((size_t)m * keep, 0.0);
    for (int i = 0; i < keep; i++) {
      const double* y = &Y[(size_t)i * m];
      double* t = &TY[(size_t)i * m];
      for (int r = 0; r < m; r++) {
        double acc = a[r] * y[r];
        if (r > 0) acc += b[r - 1] * y[r - 1];
        if (r + 1 < m) acc += b[r] * y[r + 1];
        t[r] = acc;
      }
    }
    B.assign((size_t)keep * keep, 0.0);
    for (int i = 0; i < keep; i++)
      for (int j = 0; j < keep; j++) {
        double acc = 0.0;
        for (int r = 0; r < m; r++) acc += Y[(size_t)i * m + r] * TY[(size_t)j * m + r];
        B[(size_t)i * keep + j] = acc;
      }
    for (int i = 0; i < keep; i++)
      for (int j = 0; j < i; j++)
        B[(size_t)i * keep + j] = B[(size_t)j * keep + i] = 0.5 * (B[(size_t)i * keep + j] + B[(size_t)j * keep + i]);
    s.assign(keep, 0.0);
    double snorm = 0.0;
    for (int i = 0; i < keep; i++) {
      s[i] = fnorm * Y[(size_t)i * m + (m - 1)];
      snorm += s[i] * s[i];
    }
    snorm = std::sqrt(snorm);
    // Lanczos on B from s / |s| (Z columns z_0 .. z_{r-1})
    std::vector<double> al, be;
    Z.assign((size_t)keep * keep, 0.0);
    int r = 0;
    if (snorm > 0.0) {
      for (int i = 0; i < keep; i++) Z[i] = s[i] / snorm;
      w.assign(keep, 0.0);
      for (r = 1;; r++) {
        const double* zc = &Z[(size_t)(r - 1) * keep];
        for (int i = 0; i < keep; i++) {
          double acc = 0.0;
          for (int j = 0; j < keep; j++) acc += B[(size_t)i * keep + j] * zc[j];
          w[i] = acc;
        }
        double alpha = 0.0;
        for (int i = 0; i < keep; i++) alpha += zc[i] * w[i];
        al.push_back(alpha);
        if (r == keep) break;
        for (int pass = 0; pass < 2; pass++)
          for (int q = 0; q < r; q++) {
            const double* zq = &Z[(size_t)q * keep];
            double dot = 0.0;
            for (int i = 0; i < keep; i++) dot += zq[i] * w[i];
            for (int i = 0; i < keep; i++) w[i] -= dot * zq[i];
          }
        double bn = 0.0;
        for (int i = 0; i < keep; i++) bn += w[i] * w[i];
        bn = std::sqrt(bn);
        if (!(bn > 1e-13 * normT)) break;  // the rest of Y is decoupled from f: dropped
        be.push_back(bn);
        for (int i = 0; i < keep; i++) Z[(size_t)r * keep + i] = w[i] / bn;
      }
    } else {
      // f is orthogonal to every kept vector: keep the lowest one alone
      Z[0] = 1.0;
      al.push_back(B[0]);
      r = 1;
    }
    // reversed order: u_p = z_{r-1-p}; G = Y u
    a.assign(r, 0.0);
    b.assign(r, 0.0);
    for (int p = 0; p < r; p++) {
      a[p] = al[r - 1 - p];
      if (p + 1 < r) b[p] = be[r - 2 - p];
    }
    b[r - 1] = snorm;
    G.assign((size_t)m * r, 0.0);
    for (int p = 0; p < r; p++) {
      const double* zc = &Z[(size_t)(r - 1 - p) * keep];
      double* g = &G[(size_t)p * m];
      for (int i = 0; i < keep; i++) {
        const double c = zc[i];
        if (c == 0.0) continue;
        const double* y = &Y[(size_t)i * m];
        for (int q = 0; q < m; q++) g[q] += c * y[q];
      }
    }
    return r;
  }
};

}  // namespace mpsgpu
