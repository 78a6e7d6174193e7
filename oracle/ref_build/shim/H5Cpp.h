// Oracle build shim: a do-nothing stand-in for the HDF5 C++ API.
//
// Test infrastructure only. The reference ED sources include <H5Cpp.h> for
// their checkpoint code (instance write/read), which the oracle never calls.
// HDF5 is not installed in this image, so this header declares just enough of
// the API surface for those sources to compile; every operation that would
// touch a file throws H5::Exception, so an accidental call fails loudly.
#pragma once
#include <string>
#include <stdexcept>

namespace H5 {

struct Exception {
  std::string msg;
  explicit Exception(const std::string &m = "HDF5 is not available in the oracle build") : msg(m) {}
  std::string getDetailMsg() const { return msg; }
};

struct PredType {
  static const PredType NATIVE_DOUBLE;
  static const PredType NATIVE_INT;
  static const PredType C_S1;
};

struct DataSpace {};
struct StrType {};
struct DataSet {};
struct Attribute {};

struct Group {
  Group createGroup(const std::string &) const { throw Exception(); }
  Group openGroup(const std::string &) const { throw Exception(); }
  bool nameExists(const std::string &) const { throw Exception(); }
  bool attrExists(const std::string &) const { throw Exception(); }
};

struct H5File : Group {
  H5File(const std::string &, unsigned) { throw Exception(); }
  void unlink(const std::string &) const { throw Exception(); }
};

}  // namespace H5

static const unsigned H5F_ACC_RDONLY = 0u;
static const unsigned H5F_ACC_RDWR = 1u;
static const unsigned H5F_ACC_TRUNC = 2u;
