// Host-side dense eigensolvers (see eigen.hpp for the published algorithms).
#include "eigen.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace qed {

namespace {

constexpr double kEps = 2.220446049250313e-16;

// sqrt(f^2 + g^2) without the cost of std::hypot; falls back to it only when
// the squares under- or overflow.
inline double pythag(double f, double g) {
  const double r = std::sqrt(f * f + g * g);
  if ((r == 0.0 && (f != 0.0 || g != 0.0)) || !std::isfinite(r)) return std::hypot(f, g);
  return r;
}

// Implicit-shift QL on (d, e); e[i] couples i and i+1, e has n entries (last unused).
// rot(i, c, s) is called for every plane rotation acting on columns (i, i+1) of
// the eigenvector matrix, so a caller can accumulate all of it or one row.
template <class Rot>
bool ql_implicit(int n, double *d, double *e, Rot &&rot) {
  if (n <= 1) return true;
  e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    while (true) {
      int m = l;
      for (; m < n - 1; ++m) {
        double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= kEps * dd) break;
      }
      if (m == l) break;
      if (++iter > 100) return false;
      // Wilkinson-type shift from the leading 2x2 block.
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = pythag(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool underflow = false;
      for (; i >= l; --i) {
        double f = s * e[i];
        double b = c * e[i];
        r = pythag(f, g);
        e[i + 1] = r;
        if (r == 0.0) {  // split: recover and restart the sweep
          d[i + 1] -= p;
          e[m] = 0.0;
          underflow = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        rot(i, c, s);
      }
      if (underflow) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  return true;
}

}  // namespace

bool tridiag_eig(int n, std::vector<double> &d, std::vector<double> e, std::vector<double> *z) {
  e.resize(std::max(n, 1));
  if (z) {
    z->assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) (*z)[i + (size_t)n * i] = 1.0;
  }
  double *Z = z ? z->data() : nullptr;
  bool ok = ql_implicit(n, d.data(), e.data(), [&](int i, double c, double s) {
    if (!Z) return;
    double *ci = Z + (size_t)n * i, *cj = Z + (size_t)n * (i + 1);
    for (int k = 0; k < n; ++k) {
      double f = cj[k];
      cj[k] = s * ci[k] + c * f;
      ci[k] = c * ci[k] - s * f;
    }
  });
  if (!ok) return false;
  // sort ascending (stable on ties), permuting eigenvector columns
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return d[a] < d[b]; });
  std::vector<double> d2(n);
  for (int k = 0; k < n; ++k) d2[k] = d[idx[k]];
  d = d2;
  if (Z) {
    std::vector<double> z2((size_t)n * n);
    for (int k = 0; k < n; ++k)
      std::copy(Z + (size_t)n * idx[k], Z + (size_t)n * (idx[k] + 1), z2.data() + (size_t)n * k);
    *z = std::move(z2);
  }
  return true;
}

bool tridiag_lowest_last(int n, const double *alpha, const double *beta, double *lambda0,
                         double *last) {
  if (n == 1) {
    *lambda0 = alpha[0];
    *last = 1.0;
    return true;
  }
  std::vector<double> d(alpha, alpha + n), e(n, 0.0);
  for (int i = 0; i < n - 1; ++i) e[i] = beta[i];
  std::vector<double> row(n, 0.0);  // last row of the eigenvector matrix
  row[n - 1] = 1.0;
  bool ok = ql_implicit(n, d.data(), e.data(), [&](int i, double c, double s) {
    double f = row[i + 1];
    row[i + 1] = s * row[i] + c * f;
    row[i] = c * row[i] - s * f;
  });
  if (!ok) return false;
  int k = 0;
  for (int i = 1; i < n; ++i)
    if (d[i] < d[k]) k = i;
  *lambda0 = d[k];
  *last = row[k];
  return true;
}

void tridiag_lowest_fast(int n, const double *alpha, const double *beta, double upper,
                         double *lambda0, double *last, std::vector<double> *vec) {
  if (n == 1) {
    *lambda0 = alpha[0];
    *last = 1.0;
    if (vec) vec->assign(1, 1.0);
    return;
  }
  // Gershgorin interval
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? std::fabs(beta[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(beta[i]) : 0.0);
    lo = std::min(lo, alpha[i] - r);
    hi = std::max(hi, alpha[i] + r);
  }
  if (std::isfinite(upper) && upper < hi) hi = upper + 1e-12 * (std::fabs(upper) + 1.0);
  // number of eigenvalues < x (Sturm count via the LDL^T pivots)
  auto count_below = [&](double x) {
    int c = 0;
    double q = alpha[0] - x;
    if (q < 0) ++c;
    for (int i = 1; i < n; ++i) {
      const double b2 = beta[i - 1] * beta[i - 1];
      q = alpha[i] - x - b2 / (q != 0.0 ? q : 1e-300);
      if (q < 0) ++c;
    }
    return c;
  };
  if (count_below(hi) < 1) hi = hi + 2.0 * (hi - lo) + 1.0;  // guard a too-tight warm start
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (count_below(mid) >= 1) hi = mid;
    else lo = mid;
    if (hi - lo <= 2.0 * kEps * std::max(std::fabs(lo), std::fabs(hi))) break;
  }
  const double lam = 0.5 * (lo + hi);
  // backward recurrence: u[n-1] = 1, (T - lam) u = 0 row by row from the bottom
  std::vector<double> u(n);
  u[n - 1] = 1.0;
  u[n - 2] = (beta[n - 2] != 0.0) ? (lam - alpha[n - 1]) / beta[n - 2] : 0.0;
  double scale = 1.0;  // u is stored divided by `scale` (rescaled to stay finite)
  for (int k = n - 2; k >= 1; --k) {
    double v = (beta[k - 1] != 0.0) ? ((lam - alpha[k]) * u[k] - beta[k] * u[k + 1]) / beta[k - 1] : 0.0;
    u[k - 1] = v;
    if (std::fabs(v) > 1e150) {  // rescale everything computed so far
      for (int i = k - 1; i < n; ++i) u[i] *= 1e-150;
      scale *= 1e-150;
    }
  }
  double nrm = 0.0;
  for (int i = 0; i < n; ++i) nrm += u[i] * u[i];
  nrm = std::sqrt(nrm);
  *lambda0 = lam;
  *last = u[n - 1] / nrm;
  if (vec) {
    vec->resize(n);
    for (int i = 0; i < n; ++i) (*vec)[i] = u[i] / nrm;
  }
  (void)scale;
}

void tridiag_lowest_track(int n, const double *alpha, const double *beta, RitzTracker &tr, double *lambda0,
                          double *last) {
  auto fallback = [&] {
    const double upper = ((int)tr.vec.size() == n - 1 && n > 1) ? tr.lambda : std::numeric_limits<double>::infinity();
    tridiag_lowest_fast(n, alpha, beta, upper, lambda0, last, &tr.vec);
    tr.lambda = *lambda0;
    tr.last = *last;
  };
  if (n <= 2 || (int)tr.vec.size() != n - 1) return fallback();
  double tnorm = 0.0;
  for (int i = 0; i < n; ++i)
    tnorm = std::max(tnorm, std::fabs(alpha[i]) + (i ? std::fabs(beta[i - 1]) : 0.0) +
                                (i + 1 < n ? std::fabs(beta[i]) : 0.0));
  const double r = std::fabs(beta[n - 2] * tr.last);
  if (!(r <= 1e-2 * tnorm)) return fallback();
  const double sigma = tr.lambda - r - 1e-13 * tnorm;
  // LDL^T of T - sigma: all pivots positive <=> no eigenvalue below sigma
  std::vector<double> dpiv(n), l(n, 0.0);
  dpiv[0] = alpha[0] - sigma;
  if (!(dpiv[0] > 0.0)) return fallback();
  for (int i = 0; i + 1 < n; ++i) {
    l[i] = beta[i] / dpiv[i];
    dpiv[i + 1] = alpha[i + 1] - sigma - beta[i] * l[i];
    if (!(dpiv[i + 1] > 0.0)) return fallback();
  }
  std::vector<double> x(n), y(n);
  for (int i = 0; i + 1 < n; ++i) x[i] = tr.vec[i];
  x[n - 1] = 0.0;
  double rho = tr.lambda;
  for (int it = 0; it < 4; ++it) {
    // y = (T - sigma)^{-1} x
    y[0] = x[0];
    for (int i = 1; i < n; ++i) y[i] = x[i] - l[i - 1] * y[i - 1];
    for (int i = 0; i < n; ++i) y[i] /= dpiv[i];
    for (int i = n - 2; i >= 0; --i) y[i] -= l[i] * y[i + 1];
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) nrm += y[i] * y[i];
    nrm = std::sqrt(nrm);
    for (int i = 0; i < n; ++i) x[i] = y[i] / nrm;
    // Rayleigh quotient and residual of x
    double num = 0.0, res2 = 0.0;
    for (int i = 0; i < n; ++i) {
      double tx = alpha[i] * x[i];
      if (i) tx += beta[i - 1] * x[i - 1];
      if (i + 1 < n) tx += beta[i] * x[i + 1];
      y[i] = tx;
      num += x[i] * tx;
    }
    rho = num;
    for (int i = 0; i < n; ++i) res2 += (y[i] - rho * x[i]) * (y[i] - rho * x[i]);
    if (std::sqrt(res2) <= 1e-14 * tnorm) {
      *lambda0 = rho;
      *last = x[n - 1];
      tr.lambda = rho;
      tr.last = x[n - 1];
      tr.vec = x;
      return;
    }
  }
  fallback();
}

bool sym_eig(int n, const std::vector<double> &A, std::vector<double> &w, std::vector<double> *V) {
  w.assign(n, 0.0);
  if (n == 0) return true;
  // Householder reduction A = Q T Q^T, working on a full copy; column-major a(i,j) = a[i + n*j].
  std::vector<double> a(A);
  auto at = [&](int i, int j) -> double & { return a[i + (size_t)n * j]; };
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < j; ++i) at(i, j) = at(j, i);  // symmetrise from the lower triangle
  std::vector<double> d(n), e(n, 0.0);
  std::vector<double> Q;
  if (V) {
    Q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Q[i + (size_t)n * i] = 1.0;
  }
  std::vector<double> v(n), p(n), q(n);
  for (int k = 0; k < n - 2; ++k) {
    // Householder vector annihilating a(k+2:n, k)
    double alpha = 0.0;
    for (int i = k + 1; i < n; ++i) alpha += at(i, k) * at(i, k);
    alpha = std::sqrt(alpha);
    if (alpha == 0.0) { e[k] = 0.0; continue; }
    double x0 = at(k + 1, k);
    if (x0 > 0) alpha = -alpha;
    // v = x - alpha e1, normalised so that H = I - 2 v v^T / (v^T v)
    for (int i = 0; i < n; ++i) v[i] = 0.0;
    v[k + 1] = x0 - alpha;
    for (int i = k + 2; i < n; ++i) v[i] = at(i, k);
    double vv = 0.0;
    for (int i = k + 1; i < n; ++i) vv += v[i] * v[i];
    if (vv == 0.0) { e[k] = at(k + 1, k); continue; }
    double beta2 = 2.0 / vv;
    // p = beta2 * A v (trailing block), K = beta2/2 * v^T p, q = p - K v
    for (int i = k; i < n; ++i) {  // A symmetric: row i of A == column i
      double s = 0.0;
      const double *ci = a.data() + (size_t)n * i;
      for (int j = k + 1; j < n; ++j) s += ci[j] * v[j];
      p[i] = beta2 * s;
    }
    double K = 0.0;
    for (int i = k + 1; i < n; ++i) K += v[i] * p[i];
    K *= 0.5 * beta2;
    for (int i = k; i < n; ++i) q[i] = p[i] - K * v[i];
    // A <- A - v q^T - q v^T on rows/cols k..n-1 (v[k] = 0)
    for (int j = k; j < n; ++j)
      for (int i = k; i < n; ++i) at(i, j) -= v[i] * q[j] + q[i] * v[j];
    if (V) {  // Q <- Q H = Q - beta2 (Q v) v^T
      std::fill(q.begin(), q.end(), 0.0);
      for (int j = k + 1; j < n; ++j) {
        const double *cj = Q.data() + (size_t)n * j;
        for (int i = 0; i < n; ++i) q[i] += cj[i] * v[j];
      }
      for (int j = k + 1; j < n; ++j) {
        double *cj = Q.data() + (size_t)n * j;
        double f = beta2 * v[j];
        for (int i = 0; i < n; ++i) cj[i] -= q[i] * f;
      }
    }
  }
  for (int i = 0; i < n; ++i) d[i] = at(i, i);
  for (int i = 0; i < n - 1; ++i) e[i] = at(i + 1, i);
  std::vector<double> Z;
  if (!tridiag_eig(n, d, e, V ? &Z : nullptr)) return false;
  w = d;
  if (V) {  // V = Q Z
    V->assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < n; ++k) {
        double zkj = Z[k + (size_t)n * j];
        if (zkj == 0.0) continue;
        const double *qk = Q.data() + (size_t)n * k;
        double *vj = V->data() + (size_t)n * j;
        for (int i = 0; i < n; ++i) vj[i] += qk[i] * zkj;
      }
  }
  return true;
}

namespace {
// Reduces the symmetric band matrix A (column-major n x n, half-bandwidth b,
// lower triangle used) to tridiagonal form in place by Givens rotations with
// bulge chasing (H. R. Schwarz, Numer. Math. 12, 1968). Every rotation of rows
// and columns (p, p+1) is also passed to rot(p, c, s), so that a caller can
// accumulate the transformation. On return d, e hold the tridiagonal.
template <class Rot>
void band_to_tridiagonal(int n, int b, const std::vector<double> &A, std::vector<double> &d, std::vector<double> &e,
                         Rot &&rot) {
  // Work array: the band |i - j| <= B = b + 2 (the band, the bulge at b + 1 and
  // the reach of one rotation), column j at offset (i - j + B). Nothing outside
  // it is ever read or written, and it stays cache-resident.
  const int B = b + 2, W = 2 * B + 1;
  std::vector<double> ab((size_t)W * n, 0.0);
  auto a = [&](int i, int j) -> double & { return ab[(size_t)(i - j + B) + (size_t)W * j]; };
  // symmetric band from the lower triangle of A
  for (int j = 0; j < n; ++j)
    for (int i = j; i < std::min(n, j + b + 1); ++i) {
      const double x = A[(size_t)i + (size_t)n * j];
      a(i, j) = x;
      a(j, i) = x;
    }
  // rotation in the (p, p+1) plane: A <- G A G^T, G = [[c, s], [-s, c]];
  // rows/columns p, p+1 have nonzeros only within [p-b-1, p+b+2]
  auto rotate = [&](int p, double c, double s) {
    const int q = p + 1;
    const int lo = std::max(0, p - b - 1), hi = std::min(n - 1, q + b + 1);
    for (int j = lo; j <= hi; ++j) {
      const double x = a(p, j), y = a(q, j);
      a(p, j) = c * x + s * y;
      a(q, j) = -s * x + c * y;
    }
    for (int i = lo; i <= hi; ++i) {
      const double x = a(i, p), y = a(i, q);
      a(i, p) = c * x + s * y;
      a(i, q) = -s * x + c * y;
    }
    rot(p, c, s);
  };
  auto zero_with = [&](int p, int col) {  // zero a(p+1, col) using rows p, p+1
    const double f = a(p, col), g = a(p + 1, col);
    if (g == 0.0) return false;
    const double r = pythag(f, g);
    rotate(p, f / r, g / r);
    a(p + 1, col) = 0.0;
    a(col, p + 1) = 0.0;
    return true;
  };
  for (int k = 0; k < n - 2; ++k) {
    for (int i = std::min(k + b, n - 1); i >= k + 2; --i) {
      if (!zero_with(i - 1, k)) continue;
      // the rotation of rows i-1, i creates a bulge at (i+b, i-1); chase it down
      for (int r = i; r + b < n; r += b) {
        const int row = r + b, col = r - 1;
        if (a(row, col) == 0.0) break;
        zero_with(row - 1, col);
      }
    }
  }
  d.assign(n, 0.0);
  e.assign(n, 0.0);
  for (int i = 0; i < n; ++i) d[i] = a(i, i);
  for (int i = 0; i + 1 < n; ++i) e[i] = a(i + 1, i);
}
}  // namespace

bool band_eigenvalues(int n, int b, std::vector<double> A, std::vector<double> &w) {
  w.assign(n, 0.0);
  if (n == 0) return true;
  if (b < 1) b = 1;
  std::vector<double> d, e;
  band_to_tridiagonal(n, b, A, d, e, [](int, double, double) {});
  if (!tridiag_eig(n, d, e, nullptr)) return false;
  w = d;
  return true;
}

namespace {
// LDL^T of (A - s I), A symmetric with half-bandwidth b in lower band storage;
// L in the same layout (unit diagonal implied). False on a pivot <= 0.
bool band_ldlt(int n, int b, const std::vector<double> &B, double s, std::vector<double> &L, std::vector<double> &D) {
  const int w = b + 1;
  L.assign((size_t)n * w, 0.0);
  D.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    const int j0 = std::max(0, i - b);
    for (int j = j0; j < i; ++j) {
      double v = B[(size_t)i * w + (i - j)];
      for (int m = std::max(j0, j - b); m < j; ++m) v -= L[(size_t)i * w + (i - m)] * D[m] * L[(size_t)j * w + (j - m)];
      L[(size_t)i * w + (i - j)] = v / D[j];
    }
    double d = B[(size_t)i * w] - s;
    for (int m = j0; m < i; ++m) {
      const double l = L[(size_t)i * w + (i - m)];
      d -= l * l * D[m];
    }
    if (!(d > 0.0)) return false;
    D[i] = d;
  }
  return true;
}

void band_ldlt_solve(int n, int b, const std::vector<double> &L, const std::vector<double> &D, std::vector<double> &x) {
  const int w = b + 1;
  for (int i = 0; i < n; ++i)
    for (int m = std::max(0, i - b); m < i; ++m) x[i] -= L[(size_t)i * w + (i - m)] * x[m];
  for (int i = 0; i < n; ++i) x[i] /= D[i];
  for (int i = n - 1; i >= 0; --i)
    for (int r = i + 1; r <= std::min(n - 1, i + b); ++r) x[i] -= L[(size_t)r * w + (r - i)] * x[r];
}

// x^T A x for A in lower band storage
double band_quadratic(int n, int b, const std::vector<double> &B, const std::vector<double> &x) {
  const int w = b + 1;
  double s = 0.0;
  for (int i = 0; i < n; ++i) {
    double t = B[(size_t)i * w] * x[i];
    for (int k = 1; k <= std::min(i, b); ++k) t += 2.0 * B[(size_t)i * w + k] * x[i - k];
    s += t * x[i];
  }
  return s;
}

// inverse iteration on A - s I from x (normalised in place); Rayleigh quotient
bool inverse_iteration(int n, int b, const std::vector<double> &B, double s, std::vector<double> &x, double *rq) {
  std::vector<double> L, D;
  if (!band_ldlt(n, b, B, s, L, D)) return false;
  double prev = 0.0;
  for (int it = 0; it < 80; ++it) {
    band_ldlt_solve(n, b, L, D, x);
    double nrm = 0.0;
    for (double v : x) nrm += v * v;
    nrm = std::sqrt(nrm);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) return false;
    for (double &v : x) v /= nrm;
    const double r = band_quadratic(n, b, B, x);
    if (it >= 2 && std::fabs(r - prev) <= 1e-15 * (1.0 + std::fabs(r))) {
      *rq = r;
      return true;
    }
    prev = r;
  }
  return false;
}
}  // namespace

bool band_lowest(int n, int b, const std::vector<double> &B, BandLowest &st, double *lambda) {
  if (n <= 0 || b < 1) return false;
  const int w = b + 1;
  if (!st.valid || (int)st.x.size() > n) {
    // cold start: all eigenvalues, then the eigenvector by inverse iteration
    std::vector<double> A((size_t)n * n, 0.0), ev;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k <= std::min(i, b); ++k) A[(size_t)i + (size_t)n * (i - k)] = A[(size_t)(i - k) + (size_t)n * i] = B[(size_t)i * w + k];
    if (!band_eigenvalues(n, b, A, ev)) return false;
    const double gap = n > 1 ? ev[1] - ev[0] : 1.0;
    std::vector<double> x(n, 1.0);
    double rq = 0.0;
    st.valid = inverse_iteration(n, b, B, ev[0] - std::max(1e-3 * gap, 1e-12 * (1.0 + std::fabs(ev[0]))), x, &rq);
    st.x = x;
    st.lambda = ev[0];
    st.drop = 0.0;
    *lambda = ev[0];
    return true;
  }
  std::vector<double> x(n, 0.0);
  std::copy(st.x.begin(), st.x.end(), x.begin());
  double delta = std::max(2.0 * st.drop, 1e-9 * (1.0 + std::fabs(st.lambda)));
  double rq = 0.0;
  bool ok = false;
  for (int t = 0; t < 12 && !ok; ++t, delta *= 8.0) {
    std::vector<double> y = x;
    if (inverse_iteration(n, b, B, st.lambda - delta, y, &rq)) {
      x = y;
      ok = true;
    }
  }
  if (!ok) return false;
  std::vector<double> L, D;
  if (!band_ldlt(n, b, B, rq - 1e-14 * (1.0 + std::fabs(rq)), L, D)) return false;  // certificate
  st.drop = std::max(0.0, st.lambda - rq);
  st.lambda = rq;
  st.x = x;
  *lambda = rq;
  return true;
}

bool band_eig_rows(int n, int b, std::vector<double> A, int m, std::vector<double> &w, std::vector<double> &Z) {
  w.assign(n, 0.0);
  Z.assign((size_t)m * n, 0.0);
  if (n == 0) return true;
  if (b < 1) b = 1;
  m = std::min(m, n);
  // rows 0..m-1 of the accumulated orthogonal transformation, column-major m x n
  std::vector<double> Q((size_t)m * n, 0.0);
  for (int r = 0; r < m; ++r) Q[r + (size_t)m * r] = 1.0;
  auto rot_cols = [&](int i, double c, double s) {  // columns (i, i+1) <- (c x + s y, -s x + c y)
    double *x = Q.data() + (size_t)m * i, *y = x + m;
    for (int r = 0; r < m; ++r) {
      const double u = x[r], v = y[r];
      x[r] = c * u + s * v;
      y[r] = -s * u + c * v;
    }
  };
  std::vector<double> d, e;
  band_to_tridiagonal(n, b, A, d, e, rot_cols);
  bool ok = ql_implicit(n, d.data(), e.data(), [&](int i, double c, double s) {
    double *ci = Q.data() + (size_t)m * i, *cj = ci + m;
    for (int r = 0; r < m; ++r) {
      const double f = cj[r];
      cj[r] = s * ci[r] + c * f;
      ci[r] = c * ci[r] - s * f;
    }
  });
  if (!ok) return false;
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return d[x] < d[y]; });
  for (int k = 0; k < n; ++k) {
    w[k] = d[idx[k]];
    std::copy(Q.data() + (size_t)m * idx[k], Q.data() + (size_t)m * (idx[k] + 1), Z.data() + (size_t)m * k);
  }
  return true;
}

bool complex_inverse(int n, std::complex<double> *a) {
  auto at = [&](int i, int j) -> std::complex<double> & { return a[i + (size_t)n * j]; };
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int pr = k;
    double best = std::abs(at(k, k));
    for (int i = k + 1; i < n; ++i)
      if (std::abs(at(i, k)) > best) { best = std::abs(at(i, k)); pr = i; }
    if (best == 0.0) return false;
    piv[k] = pr;
    if (pr != k)
      for (int j = 0; j < n; ++j) std::swap(at(k, j), at(pr, j));
    std::complex<double> inv = 1.0 / at(k, k);
    at(k, k) = 1.0;
    for (int j = 0; j < n; ++j) at(k, j) *= inv;
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      std::complex<double> f = at(i, k);
      if (f == 0.0) continue;
      at(i, k) = 0.0;
      for (int j = 0; j < n; ++j) at(i, j) -= f * at(k, j);
    }
  }
  for (int k = n - 1; k >= 0; --k)
    if (piv[k] != k)
      for (int i = 0; i < n; ++i) std::swap(at(i, k), at(i, piv[k]));
  return true;
}

}  // namespace qed
