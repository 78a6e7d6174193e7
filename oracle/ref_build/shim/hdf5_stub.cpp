// Oracle build shim: the reference's HDF5 helper functions (declared in
// src_util/hdf5_io.hpp) and its interrupt hook (src_python/common_Py.cpp:29),
// replaced for the CPU oracle build.
//
// Test infrastructure only. HDF5 and Python signal handling are not part of the
// ED hot path; every HDF5 helper throws so that a stray checkpoint call fails
// loudly, and check_signals() does nothing (no interpreter to poll).
#include "hdf5_io.hpp"

using namespace std;

namespace {
[[noreturn]] void no_hdf5() { throw H5::Exception("HDF5 is not available in the oracle build"); }
}  // namespace

void h5_write_attr(H5::Group &, const string &, double) { no_hdf5(); }
void h5_write_attr(H5::Group &, const string &, int) { no_hdf5(); }
void h5_write_attr(H5::Group &, const string &, const string &) { no_hdf5(); }
double h5_read_attr_double(const H5::Group &, const string &) { no_hdf5(); }
int h5_read_attr_int(const H5::Group &, const string &) { no_hdf5(); }
string h5_read_attr_string(const H5::Group &, const string &) { no_hdf5(); }
void h5_write_vec(H5::Group &, const string &, const vector<double> &) { no_hdf5(); }
void h5_read_vec(const H5::Group &, const string &, vector<double> &) { no_hdf5(); }
void h5_write_mat(H5::Group &, const string &, const matrix<double> &) { no_hdf5(); }
void h5_read_mat(const H5::Group &, const string &, matrix<double> &) { no_hdf5(); }
void h5_write_mat(H5::Group &, const string &, const matrix<Complex> &) { no_hdf5(); }
void h5_read_mat(const H5::Group &, const string &, matrix<Complex> &) { no_hdf5(); }

void check_signals() {}
