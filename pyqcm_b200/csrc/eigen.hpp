// Host-side dense eigensolvers for the small projected problems of the ED
// solver: the Lanczos tridiagonal (Ritz test, src_ed/Hamiltonian/Lanczos.cpp:25-52),
// the band-Lanczos projected matrix (src_ed/Hamiltonian/Lanczos.hpp:340-384)
// and the Q-matrix streamlining (src_ed/Q_matrix.hpp:286-318).
//
// Algorithms: Householder reduction to tridiagonal form followed by the
// implicit-shift QL iteration (Wilkinson shift), as published by Bowdler,
// Martin, Reinsch and Wilkinson (Handbook for Automatic Computation II,
// procedures tred2/tql2). Eigenvalues are returned in ascending order with
// orthonormal eigenvector columns, the contract of LAPACK dstev/dsyev that the
// reference relies on.
#pragma once
#include <complex>
#include <vector>

namespace qed {

// Symmetric tridiagonal eigenproblem: diagonal d[n], off-diagonal e[n-1].
// On return d holds the eigenvalues ascending. If z != nullptr it receives the
// n x n eigenvector matrix (column-major, column k <-> d[k]).
// Returns false if the QL iteration did not converge.
bool tridiag_eig(int n, std::vector<double> &d, std::vector<double> e, std::vector<double> *z);

// Lowest eigenvalue of the tridiagonal (alpha[n], beta[n-1]) and the last
// component of its normalised eigenvector, in O(n^2): QL rotations applied to
// the last row of the eigenvector matrix only. This is exactly what the
// reference's Ritz-residual test consumes (evector.back(), Lanczos.hpp:82-83).
bool tridiag_lowest_last(int n, const double *alpha, const double *beta, double *lambda0,
                         double *last);

// Same quantities in O(n) per call: the lowest eigenvalue by Sturm-sequence
// bisection (Givens' method), started from `upper` (an upper bound, e.g. the
// previous Lanczos step's value by Cauchy interlacing; pass +inf if unknown),
// and the eigenvector by the three-term recurrence run backwards from the last
// component, which is stable for an eigenvector whose weight sits at the start.
// vec (optional) receives the whole normalised eigenvector.
void tridiag_lowest_fast(int n, const double *alpha, const double *beta, double upper,
                         double *lambda0, double *last, std::vector<double> *vec);

// Incremental version for a growing Lanczos tridiagonal: called with n = 1, 2,
// 3, ... on the same alpha/beta arrays (beta[n-2] couples the newest row). The
// previous eigenvector [u; 0] has Rayleigh quotient lambda_prev and residual
// r = |beta[n-2] u_last| for T_n, so T_n has an eigenvalue in
// [lambda_prev - r, lambda_prev]; if T_n - sigma (sigma just below that
// interval) is positive definite (all LDL^T pivots > 0, i.e. a Sturm count of
// zero) that eigenvalue is the lowest and a few steps of inverse iteration from
// [u; 0] give it with its eigenvector in O(n). Otherwise, or if the iteration
// does not reach a residual of 1e-14 ||T||, it falls back to
// tridiag_lowest_fast.
struct RitzTracker {
  double lambda = 0.0, last = 0.0;
  std::vector<double> vec;  // eigenvector of the previous call
};
void tridiag_lowest_track(int n, const double *alpha, const double *beta, RitzTracker &tr, double *lambda0,
                          double *last);

// Dense symmetric eigenproblem, A column-major n x n (lower triangle used).
// w receives eigenvalues ascending; V (if non-null) the eigenvectors.
bool sym_eig(int n, const std::vector<double> &A, std::vector<double> &w, std::vector<double> *V);

// Eigenvalues (ascending) of a symmetric band matrix of half-bandwidth b,
// given as a full column-major n x n array (entries outside the band ignored).
// Reduces to tridiagonal form by Givens rotations with bulge chasing
// (H. R. Schwarz, "Tridiagonalization of a symmetric band matrix", Numer. Math.
// 12, 1968), O(n^2 b), then QL. Used for the band-Lanczos convergence test.
bool band_eigenvalues(int n, int b, std::vector<double> A, std::vector<double> &w);

// Lowest eigenvalue of a growing sequence of band matrices (each the leading
// block of the next, as in the band-Lanczos convergence test), in lower band
// storage B[i * (b + 1) + k] = A(i, i - k), k = 0..min(i, b). The first call
// takes all eigenvalues (band_eigenvalues); later calls run inverse iteration
// on A - s I (banded LDL^T, O(n b^2)) from the previous eigenvector, with the
// shift s below the previous lowest eigenvalue (which, by interlacing, is not
// below the new one), and certify the Rayleigh quotient r: the LDL^T of
// A - (r - eps) I, eps = 1e-14 (1 + |r|), must have positive pivots, so the
// lowest eigenvalue lies in [r - eps, r]. Returns false where that fails (the
// caller then takes band_eigenvalues).
struct BandLowest {
  std::vector<double> x;  // eigenvector of the last call
  double lambda = 0.0, drop = 0.0;
  bool valid = false;
};
bool band_lowest(int n, int b, const std::vector<double> &B, BandLowest &st, double *lambda);

// Eigenvalues (ascending) of the same band matrix and the first m rows of its
// eigenvector matrix, Z column-major m x n (column k <-> w[k]): the band
// reduction and the QL rotations are accumulated on those m rows only, O(n^2 b)
// instead of the O(n^3) of a full eigensystem. The band-Lanczos Q-matrix needs
// only the first p rows (Q = P U with P zero beyond the p start vectors).
bool band_eig_rows(int n, int b, std::vector<double> A, int m, std::vector<double> &w, std::vector<double> &Z);

// In-place inverse of a complex n x n column-major matrix (Gauss-Jordan with
// partial pivoting). Returns false if singular.
bool complex_inverse(int n, std::complex<double> *a);

}  // namespace qed
