// Global options of the ED solver. Names, types and defaults are those of the
// reference's QCM initialisation (src_util/global_parameter.cpp:10-92), which is
// what pyqcm installs (src_python/qcm_lib.cpp:63). Options of the lattice layer
// are accepted and stored so that callers can keep setting them, but only the
// ED options listed in options.cpp influence this solver.
#pragma once
#include <string>

namespace qed {

bool opt_bool(const std::string &name);
long opt_int(const std::string &name);
double opt_double(const std::string &name);
char opt_char(const std::string &name);

void set_opt_bool(const std::string &name, bool v);
void set_opt_int(const std::string &name, long v);
void set_opt_double(const std::string &name, double v);
void set_opt_char(const std::string &name, char v);

// Incremented by every set_opt_*: a value read in a hot path can be cached per
// thread and read again only when this changes.
unsigned long long options_generation();

}  // namespace qed
