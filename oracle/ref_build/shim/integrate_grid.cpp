// Project-written stand-in for the reference's src_util/integrate.cpp, which
// needs the third-party Cubature library (absent here). TEST INFRASTRUCTURE
// ONLY: linked into the oracle library, never into the product.
//
// k_integral_grid restates the reference's fixed-grid wavevector sum
// (src_util/integrate.cpp:177-240): k = (i/nkx, j/nky, l/nkz) in the reciprocal
// superlattice basis, summed and multiplied by 1/(nkx nky nkz). The partial
// sums are added in index order on one thread, so the oracle's grid integral
// does not depend on the OpenMP thread count. The adaptive-cubature routines
// (wk_integral, k_integral) and the HDF5-backed external hybridisation
// (lattice_hybrid, src_qcm/lattice_hybrid.cpp) throw: the oracle drives the
// Potthoff functional through the discrete (frequency, k) grid path only.
#include <functional>
#include <stdexcept>
#include <vector>

#include "QCM.hpp"
#include "lattice_hybrid.hpp"
#include "vector3D.hpp"

using namespace std;

void QCM::k_integral_grid(int dim, int nkx, int nky, int nkz,
                          function<void(vector3D<double> &k, const int *nv, double I[])> f, vector<double> &Iv) {
  const int nv = (int)Iv.size();
  vector<double> sum(nv, 0.0), Ik(nv);
  const int nx = nkx, ny = dim >= 2 ? nky : 1, nz = dim >= 3 ? nkz : 1;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int l = 0; l < nz; l++) {
        vector3D<double> k(i * (1.0 / nkx), dim >= 2 ? j * (1.0 / nky) : 0.0, dim >= 3 ? l * (1.0 / nkz) : 0.0);
        f(k, &nv, Ik.data());
        for (int a = 0; a < nv; a++) sum[a] += Ik[a];
      }
  double w = 1.0 / nkx;
  if (dim >= 2) w *= 1.0 / nky;
  if (dim >= 3) w *= 1.0 / nkz;
  for (int a = 0; a < nv; a++) Iv[a] += sum[a] * w;
}

void QCM::wk_integral(int, function<void(Complex w, vector3D<double> &k, const int *nv, double I[])>, vector<double> &,
                      const double, bool) {
  throw runtime_error("oracle: adaptive (frequency, k) cubature is not built (Cubature absent); set a discrete grid");
}

void QCM::k_integral(int, function<void(vector3D<double> &k, const int *nv, double I[])>, vector<double> &,
                     const double, bool) {
  throw runtime_error("oracle: adaptive k cubature is not built (Cubature absent); set a wavevector grid");
}

lattice_hybrid::lattice_hybrid(const string &) {
  throw runtime_error("oracle: external lattice hybridisation needs HDF5, which is absent");
}
