// Oracle build shim: LAPACK-backed definitions of the dense linear-algebra
// members of the reference's matrix<T> (declared in src_util/matrix.hpp).
//
// Test infrastructure only. The reference implements these members with Eigen
// (src_util/matrix.cpp:24-230), which is not installed in this image. This file
// gives the same contracts: eigenvalues ascending with orthonormal eigenvector
// columns (LAPACK dsyev/zheev of the image's OpenBLAS), inverse by Gauss-Jordan,
// determinant with the permutation sign, lower Cholesky factor (dpotrf). Eigenvector
// signs/phases may differ from Eigen's; every quantity the ED path builds from
// them (Q = P.U, Lehmann sums) is invariant under a per-column phase.
#include <cmath>
#include <stdexcept>
#include "matrix.hpp"

using namespace std;

namespace {

int lapack_dsyev(char jobz, int n, double *a, double *w) {
  char uplo = 'L';
  integer nn = n, lda = n, lwork = -1, info = 0;
  double wq = 0.0;
  dsyev_(&jobz, &uplo, &nn, a, &lda, w, &wq, &lwork, &info);
  lwork = (integer)wq;
  vector<double> work(lwork > 1 ? lwork : 1);
  dsyev_(&jobz, &uplo, &nn, a, &lda, w, work.data(), &lwork, &info);
  return (int)info;
}

int lapack_zheev(char jobz, int n, Complex *a, double *w) {
  char uplo = 'L';
  integer nn = n, lda = n, lwork = -1, info = 0;
  doublecomplex wq;
  vector<double> rwork(3 * n > 2 ? 3 * n - 2 : 1);
  zheev_(&jobz, &uplo, &nn, (doublecomplex *)a, &lda, w, &wq, &lwork, rwork.data(), &info);
  lwork = (integer)wq.r;
  vector<doublecomplex> work(lwork > 1 ? lwork : 1);
  zheev_(&jobz, &uplo, &nn, (doublecomplex *)a, &lda, w, work.data(), &lwork, rwork.data(), &info);
  return (int)info;
}

}  // namespace

// Gauss-Jordan elimination with partial pivoting, in place (column-major).
// Kept free of LAPACK so that the oracle does not depend on which LU routine
// the dynamic linker binds when other libraries (e.g. PyTorch's
// libtorch_cpu, which exports zgetrf_) are already loaded.
// Pivot magnitude |re| + |im| (LAPACK's dcabs1), computed inline so no libm
// complex routine is involved.
static double mag1(double x) { return fabs(x); }
static double mag1(const Complex &z) { return fabs(z.real()) + fabs(z.imag()); }

template <class T> static bool gauss_jordan_inverse(size_t n, T *a) {
  auto at = [&](size_t i, size_t j) -> T & { return a[i + n * j]; };
  vector<size_t> piv(n);
  for (size_t k = 0; k < n; ++k) {
    size_t p = k;
    double best = mag1(at(k, k));
    for (size_t i = k + 1; i < n; ++i)
      if (mag1(at(i, k)) > best) { best = mag1(at(i, k)); p = i; }
    if (best == 0.0) return false;
    piv[k] = p;
    if (p != k)
      for (size_t j = 0; j < n; ++j) std::swap(at(k, j), at(p, j));
    T inv = T(1.0) / at(k, k);
    at(k, k) = T(1.0);
    for (size_t j = 0; j < n; ++j) at(k, j) *= inv;
    for (size_t i = 0; i < n; ++i) {
      if (i == k) continue;
      T f = at(i, k);
      if (f == T(0.0)) continue;
      at(i, k) = T(0.0);
      for (size_t j = 0; j < n; ++j) at(i, j) -= f * at(k, j);
    }
  }
  for (size_t k = n; k-- > 0;)
    if (piv[k] != k)
      for (size_t i = 0; i < n; ++i) std::swap(at(i, k), at(i, piv[k]));
  return true;
}

template <> void matrix<double>::inverse() {
  QCM_ASSERT(r == c);
  if (r == 0) return;
  if (r == 1) { v[0] = 1 / v[0]; return; }
  QCM_ASSERT(gauss_jordan_inverse<double>(r, v.data()));
}

template <> bool matrix<Complex>::is_real(double accuracy) {
  for (auto &z : v)
    if (fabs(z.imag()) > accuracy) return false;
  return true;
}

template <> void matrix<double>::eigensystem(vector<double> &d, matrix<double> &U) const {
  QCM_ASSERT(r == c);
  QCM_ASSERT(U.r == r and U.c == c);
  QCM_ASSERT(d.size() == r);
  if (r == 0) return;
  U.v = v;
  if (lapack_dsyev('V', (int)r, U.v.data(), d.data()) != 0)
    throw std::runtime_error("dsyev failed (eigensystem<double>)");
}

template <> void matrix<double>::eigenvalues(vector<double> &d) {
  QCM_ASSERT(r == c);
  if (r == 0) return;
  vector<double> a(v);
  if (d.size() < r) d.resize(r);
  QCM_ASSERT(lapack_dsyev('N', (int)r, a.data(), d.data()) == 0);
}

template <> void matrix<Complex>::inverse() {
  QCM_ASSERT(r == c);
  if (r == 0) return;
  QCM_ASSERT(gauss_jordan_inverse<Complex>(r, v.data()));
}

// Determinant by Gaussian elimination with partial pivoting (sign included).
template <> Complex matrix<Complex>::determinant() {
  if (r == 0) return Complex(0);
  vector<Complex> a(v);
  auto at = [&](size_t i, size_t j) -> Complex & { return a[i + r * j]; };
  Complex det(1.0);
  for (size_t k = 0; k < r; ++k) {
    size_t p = k;
    for (size_t i = k + 1; i < r; ++i)
      if (mag1(at(i, k)) > mag1(at(p, k))) p = i;
    if (at(p, k) == Complex(0.0)) return Complex(0.0);
    if (p != k) {
      for (size_t j = 0; j < r; ++j) std::swap(at(k, j), at(p, j));
      det = -det;
    }
    det *= at(k, k);
    for (size_t i = k + 1; i < r; ++i) {
      Complex f = at(i, k) / at(k, k);
      for (size_t j = k; j < r; ++j) at(i, j) -= f * at(k, j);
    }
  }
  return det;
}

template <> void matrix<Complex>::eigensystem(vector<double> &d, matrix<Complex> &U) const {
  QCM_ASSERT(r == c);
  if (r == 0) return;
  U.set_size(r, c);
  U.v = v;
  if (d.size() < r) d.resize(r);
  if (lapack_zheev('V', (int)r, U.v.data(), d.data()) != 0)
    throw std::runtime_error("zheev failed (eigensystem<complex>)");
}

template <> void matrix<Complex>::eigenvalues(vector<double> &d) {
  QCM_ASSERT(r == c);
  if (r == 0) return;
  vector<Complex> a(v);
  if (d.size() < r) d.resize(r);
  QCM_ASSERT(lapack_zheev('N', (int)r, a.data(), d.data()) == 0);
}

template <> double matrix<double>::norm2() {
  double s = 0.0;
  for (double x : v) s += x * x;
  return s;
}
template <> double matrix<Complex>::norm2() {
  double s = 0.0;
  for (auto &z : v) s += std::norm(z);
  return s;
}
template <> double matrix<double>::norm() { return sqrt(norm2()); }
template <> double matrix<Complex>::norm() { return sqrt(norm2()); }

template <> bool matrix<double>::is_orthogonal(double accuracy) {
  if (r != c) return false;
  for (size_t i = 0; i < c; ++i)
    for (size_t j = 0; j < c; ++j) {
      double s = 0.0;
      for (size_t k = 0; k < r; ++k) s += v[k + r * i] * v[k + r * j];
      if (fabs(s - (i == j ? 1.0 : 0.0)) > accuracy) return false;
    }
  return true;
}

template <> bool matrix<double>::cholesky(matrix<double> &A) {
  vector<double> a(A.v);
  char uplo = 'L';
  integer n = A.r, lda = A.r, info = 0;
  dpotrf_(&uplo, &n, a.data(), &lda, &info);
  if (info != 0) return false;
  set_size(A.r);
  for (size_t j = 0; j < A.r; ++j)
    for (size_t i = 0; i < A.r; ++i) v[i + r * j] = (i >= j) ? a[i + A.r * j] : 0.0;
  return true;
}

template <> bool matrix<double>::triangular_inverse() {
  char uplo = 'L', diag = 'N';
  integer n = r, lda = r, info = 0;
  for (size_t j = 0; j < c; ++j)
    for (size_t i = 0; i < j; ++i) v[i + r * j] = 0.0;
  dtrtri_(&uplo, &diag, &n, v.data(), &lda, &info);
  return info == 0;
}

matrix<Complex> to_complex_matrix(const matrix<double> &x) {
  matrix<Complex> xc(x.r, x.c);
  for (size_t i = 0; i < x.v.size(); ++i) xc.v[i] = x.v[i];
  return xc;
}

matrix<Complex> hermitian_matrix_from_real_vector(size_t d, const vector<double> &x) {
  matrix<Complex> M(d);
  size_t k = 0;
  for (size_t i = 0; i < d; ++i) {
    M(i, i) = x[k++];
    for (size_t j = 0; j < i; ++j, k += 2) {
      M(i, j) = Complex(x[k], x[k + 1]);
      M(j, i) = conj(M(i, j));
    }
  }
  return M;
}

void hermitian_matrix_to_real_vector(const matrix<Complex> &M, double *x) {
  size_t k = 0;
  for (size_t i = 0; i < M.r; ++i) {
    x[k++] = M(i, i).real();
    for (size_t j = 0; j < i; ++j) {
      x[k++] = M(i, j).real();
      x[k++] = M(i, j).imag();
    }
  }
}
