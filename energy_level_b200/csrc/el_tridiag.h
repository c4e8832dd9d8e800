// Host-side symmetric tridiagonal eigen-solver used by the Lanczos drivers.
//
// T has diagonal a[0..m-1] and off-diagonal b[0..m-2] (b[i] couples i, i+1).
// Eigenvalues: Sturm-sequence bisection (the number of negative pivots of the
// LDL^T factorisation of T - s I counts eigenvalues below s).  Eigenvectors:
// inverse iteration with a tridiagonal LU factorisation with partial pivoting.
// All arithmetic in FP64.
#pragma once

#include <cmath>
#include <vector>
#include <algorithm>

namespace el {

inline int sturm_count(const double *a, const double *b, int m, double s) {
  int count = 0;
  double q = a[0] - s;
  const double tiny = 1e-300;
  if (q < 0) ++count;
  for (int i = 1; i < m; ++i) {
    if (std::fabs(q) < tiny) q = (q < 0 ? -tiny : tiny);
    q = a[i] - s - b[i - 1] * b[i - 1] / q;
    if (q < 0) ++count;
  }
  return count;
}

inline void gersh_bounds(const double *a, const double *b, int m, double *lo, double *hi) {
  double l = 1e300, h = -1e300;
  for (int i = 0; i < m; ++i) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(b[i]) : 0.0);
    l = std::min(l, a[i] - r);
    h = std::max(h, a[i] + r);
  }
  const double pad = 1e-12 * std::max(1.0, std::max(std::fabs(l), std::fabs(h)));
  *lo = l - pad;
  *hi = h + pad;
}

// k-th smallest eigenvalue (k = 0-based).
inline double tridiag_eig(const double *a, const double *b, int m, int k) {
  double lo, hi;
  gersh_bounds(a, b, m, &lo, &hi);
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (sturm_count(a, b, m, mid) > k) hi = mid; else lo = mid;
  }
  return 0.5 * (lo + hi);
}

// Largest eigenvalue.
inline double tridiag_eig_max(const double *a, const double *b, int m) {
  return tridiag_eig(a, b, m, m - 1);
}

// Unit eigenvector for eigenvalue lam by inverse iteration.
inline void tridiag_vec(const double *a, const double *b, int m, double lam,
                        std::vector<double> &x) {
  x.assign(m, 1.0);
  if (m == 1) { x[0] = 1.0; return; }
  double scale = 0.0;
  for (int i = 0; i < m; ++i) scale = std::max(scale, std::fabs(a[i]) + (i < m - 1 ? std::fabs(b[i]) : 0.0));
  const double eps = 2.2e-16 * std::max(scale, 1e-300);
  // LU of (T - lam I) with partial pivoting: rows hold (d, u1, u2)
  std::vector<double> d(m), u1(m, 0.0), u2(m, 0.0), l(m, 0.0);
  std::vector<int> piv(m, 0);
  // working copies
  std::vector<double> dd(m), ee(m, 0.0);
  for (int i = 0; i < m; ++i) dd[i] = a[i] - lam;
  for (int i = 0; i + 1 < m; ++i) ee[i] = b[i];
  // Gaussian elimination on the band [sub=b, diag=dd, super=ee]
  double cur_d = dd[0], cur_u1 = ee[0], cur_u2 = 0.0;
  for (int i = 0; i < m - 1; ++i) {
    const double sub = b[i];
    const double nd = dd[i + 1], nu1 = (i + 1 < m - 1) ? ee[i + 1] : 0.0;
    if (std::fabs(cur_d) >= std::fabs(sub)) {
      piv[i] = 0;
      double dv = cur_d;
      if (std::fabs(dv) < eps) dv = (dv < 0 ? -eps : eps);
      const double f = sub / dv;
      l[i] = f;
      d[i] = dv; u1[i] = cur_u1; u2[i] = cur_u2;
      cur_d = nd - f * cur_u1;
      cur_u1 = nu1 - f * cur_u2;
      cur_u2 = 0.0;
    } else {
      piv[i] = 1;
      const double f = cur_d / sub;
      l[i] = f;
      d[i] = sub; u1[i] = nd; u2[i] = nu1;
      cur_d = cur_u1 - f * nd;
      cur_u1 = cur_u2 - f * nu1;
      cur_u2 = 0.0;
    }
  }
  if (std::fabs(cur_d) < eps) cur_d = (cur_d < 0 ? -eps : eps);
  d[m - 1] = cur_d;
  // deterministic, non-degenerate start
  for (int i = 0; i < m; ++i) x[i] = 1.0 + 0.01 * std::sin(1.0 + i);
  for (int it = 0; it < 3; ++it) {
    // forward: apply L^{-1} with the recorded row swaps
    std::vector<double> y(x);
    for (int i = 0; i < m - 1; ++i) {
      if (piv[i]) std::swap(y[i], y[i + 1]);
      y[i + 1] -= l[i] * y[i];
    }
    // back substitution with U (diag d, super u1, u2)
    for (int i = m - 1; i >= 0; --i) {
      double s = y[i];
      if (i + 1 < m) s -= u1[i] * y[i + 1];
      if (i + 2 < m) s -= u2[i] * y[i + 2];
      y[i] = s / d[i];
    }
    double nrm = 0.0;
    for (int i = 0; i < m; ++i) nrm += y[i] * y[i];
    nrm = std::sqrt(nrm);
    if (!(nrm > 0) || !std::isfinite(nrm)) break;
    for (int i = 0; i < m; ++i) x[i] = y[i] / nrm;
  }
  // fix the sign so that the largest component is positive (deterministic)
  int imax = 0;
  for (int i = 1; i < m; ++i) if (std::fabs(x[i]) > std::fabs(x[imax])) imax = i;
  if (x[imax] < 0) for (int i = 0; i < m; ++i) x[i] = -x[i];
}

}  // namespace el
