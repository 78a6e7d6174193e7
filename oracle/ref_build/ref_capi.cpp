// CPU oracle: a flat C entry layer over the reference's own ED library
// (namespace ED, src_ed/qcm_ED.hpp:23-340), compiled from the reference sources.
//
// TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline / reference arm load the library this file is linked into. It is
// never part of the product path.
//
// Conventions follow the reference's Python binding (src_python/qcm_ED_wrap.hpp):
//  - the QCM global-parameter defaults are installed (src_util/global_parameter.cpp:10-92),
//    which is what pyqcm uses (src_python/qcm_lib.cpp:63);
//  - operator matrix elements are passed 0-based (the binding subtracts 1,
//    src_python/qcm_ED_wrap.hpp:199-200);
//  - complex outputs are interleaved (re, im) doubles, column-major like matrix<T>.
// Every entry returns 0 on success; on a thrown qcm_error it returns 1 and the
// message is available from ref_last_error().
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "qcm_ED.hpp"
#include "model_instance.hpp"
#include "ED_basis.hpp"
#include "symmetry_group.hpp"
#include "global_parameter.hpp"
#include "QCM.hpp"
#include "lattice_model.hpp"
#include "lattice_model_instance.hpp"

namespace QCM { void global_parameter_init(); }

// Globals of the reference's lattice layer (src_qcm/QCM.cpp:34-41).
extern shared_ptr<lattice_model> qcm_model;
extern map<int, unique_ptr<lattice_model_instance>> lattice_model_instances;
extern vector<double> grid_freqs;
extern vector<double> grid_weights;

// Globals defined by the reference at src_ed/qcm_ED.cpp:25-26.
extern map<string, shared_ptr<model>> models;
extern map<size_t, shared_ptr<model_instance_base>> model_instances;

namespace {
std::string g_err;

template <class F> int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    g_err = e.what();
    return 1;
  } catch (const H5::Exception &e) {
    g_err = e.getDetailMsg();
    return 1;
  }
}

void put_complex(const matrix<Complex> &g, double *out) {
  for (size_t i = 0; i < g.v.size(); ++i) {
    out[2 * i] = g.v[i].real();
    out[2 * i + 1] = g.v[i].imag();
  }
}

struct hv_handle {
  std::unique_ptr<Hamiltonian<double>> H;
};
}  // namespace

extern "C" {

int ref_last_error(char *buf, int n) {
  if (n > 0) {
    std::strncpy(buf, g_err.c_str(), (size_t)n - 1);
    buf[n - 1] = 0;
  }
  return (int)g_err.size();
}

int ref_init(void) {
  return guarded([] {
    // QCM::qcm_init (src_python/qcm_lib.cpp:61-63) without the OpenMP banner
    if (!qcm_model) qcm_model = make_shared<lattice_model>();
    QCM::global_parameter_init();
  });
}

int ref_set_int(const char *name, long v) {
  return guarded([&] { set_global_int(name, (size_t)v); });
}
int ref_set_double(const char *name, double v) {
  return guarded([&] { set_global_double(name, v); });
}
int ref_set_char(const char *name, char v) {
  return guarded([&] { set_global_char(name, v); });
}
int ref_set_bool(const char *name, int v) {
  return guarded([&] { set_global_bool(name, v != 0); });
}

int ref_new_model(const char *name, int n_sites, int n_bath) {
  return guarded([&] { ED::new_model(name, n_sites, n_bath, {}, false); });
}

// The reference's symmetry_group for 0-based generators (as ED::new_model
// takes them): order, character phases, symmetric orbitals, orbitals per irrep.
static std::vector<std::vector<int>> gen_rows(int n_orb, int n_gen, const int *gen) {
  std::vector<std::vector<int>> g(n_gen, std::vector<int>(n_orb));
  for (int j = 0; j < n_gen; ++j)
    for (int i = 0; i < n_orb; ++i) g[j][i] = gen[j * n_orb + i];
  return g;
}

int ref_symmetry_group(int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep, int *g, int *phi,
                       double *S_re, double *S_im, int *dims) {
  return guarded([&] {
    symmetry_group G(n_sites + n_bath, n_sites, gen_rows(n_sites + n_bath, n_gen, gen), bath_irrep != 0);
    *g = G.g;
    for (int a = 0; a < G.g; ++a)
      for (int b = 0; b < G.g; ++b) phi[a * G.g + b] = G.phi(a, b);
    for (int k = 0; k < n_sites; ++k)
      for (int i = 0; i < n_sites; ++i) {
        S_re[k * n_sites + i] = G.S(k, i).real();
        S_im[k * n_sites + i] = G.S(k, i).imag();
      }
    for (int r = 0; r < G.g; ++r) dims[r] = G.site_irrep_dim[r];
  });
}

// symmetry_group::Representative of n states in irrep `irrep`.
int ref_representatives(int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep, int irrep, long n,
                        const uint64_t *states, uint64_t *rep, int *phase, int *length) {
  return guarded([&] {
    symmetry_group G(n_sites + n_bath, n_sites, gen_rows(n_sites + n_bath, n_gen, gen), bath_irrep != 0);
    for (long i = 0; i < n; ++i) {
      rep_map m = G.Representative(binary_state(states[i]), irrep);
      rep[i] = m.b.b;
      phase[i] = m.phase;
      length[i] = m.length;
    }
  });
}

// ED_mixed_basis of a sector string ("R1:N6:S0") under the group: the sorted
// representative states. With out == nullptr only *dim is set.
int ref_mixed_basis(int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep, const char *sec, uint64_t *out,
                    long *dim) {
  return guarded([&] {
    auto G = std::make_shared<symmetry_group>(n_sites + n_bath, n_sites, gen_rows(n_sites + n_bath, n_gen, gen),
                                              bath_irrep != 0);
    ED_mixed_basis B(sector(std::string(sec)), G);
    *dim = (long)B.dim;
    if (out)
      for (size_t i = 0; i < B.dim; ++i) out[i] = B.binlist[i].b;
  });
}

// A cluster model with symmetry generators, given as pyqcm takes them (n_gen rows
// of n_sites + n_bath entries, 1-based sites; bath entries 1-based orbitals, or
// irrep phases when bath_irrep is set), converted to ED::new_model's 0-based form
// as the reference's Python binding does (src_python/qcm_ED_wrap.hpp:145-163).
int ref_new_model_gen(const char *name, int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep) {
  return guarded([&] {
    const int n_orb = n_sites + n_bath;
    std::vector<std::vector<int>> g(n_gen, std::vector<int>(n_orb));
    for (int j = 0; j < n_gen; ++j)
      for (int i = 0; i < n_orb; ++i) {
        int v = gen[j * n_orb + i];
        if (i < n_sites || !bath_irrep) v -= 1;
        g[j][i] = v;
      }
    ED::new_model(name, n_sites, n_bath, g, bath_irrep != 0);
  });
}

int ref_new_operator(const char *model_name, const char *op, const char *type, int n, const int *r,
                     const int *c, const double *v) {
  return guarded([&] {
    std::vector<matrix_element<double>> el(n);
    for (int i = 0; i < n; ++i) el[i] = matrix_element<double>(r[i], c[i], v[i]);
    ED::new_operator(model_name, op, type, el);
  });
}

// `format` is the Hamiltonian_format letter for this instance. The reference
// reads that option only when its first instance is built
// (src_ed/model_instance_base.cpp:38-48); the global it sets is assigned here
// before every instance so that one process can hold instances of both the
// factorized ('F') and CSR ('S') formats.
int ref_new_instance(const char *model_name, int n, const char **names, const double *values,
                     const char *sectors, int label, char format) {
  return guarded([&] {
    set_global_char("Hamiltonian_format", format);
    switch (format) {
      case 'F': Hamiltonian_format = H_FORMAT::H_format_factorized; break;
      case 'S': Hamiltonian_format = H_FORMAT::H_format_csr; break;
      case 'O': Hamiltonian_format = H_FORMAT::H_format_ops; break;
      case 'N': Hamiltonian_format = H_FORMAT::H_format_onthefly; break;
      default: throw qcm_error(std::string("ref_new_instance: unsupported format ") + format);
    }
    map<string, double> p;
    for (int i = 0; i < n; ++i) p[names[i]] = values[i];
    ED::new_model_instance(model_name, p, sectors, (size_t)label);
  });
}

int ref_erase_instance(int label) {
  return guarded([&] { ED::erase_model_instance((size_t)label); });
}

int ref_ground_state(int label, double *E0, char *sec, int seclen) {
  return guarded([&] {
    auto r = ED::ground_state_solve((size_t)label);
    *E0 = r.first;
    std::strncpy(sec, r.second.c_str(), (size_t)seclen - 1);
    sec[seclen - 1] = 0;
  });
}

int ref_green_solve(int label) {
  return guarded([&] { ED::Green_function_solve((size_t)label); });
}

int ref_gf_dim(int label) { return (int)ED::Green_function_dimension((size_t)label); }

int ref_mixing(int label) { return ED::mixing((size_t)label); }

// G(z) for nz frequencies; G_out holds nz blocks of n x n complex, column-major.
int ref_green_function(int label, int spin_down, int nz, const double *z, double *G_out) {
  return guarded([&] {
    for (int k = 0; k < nz; ++k) {
      Complex w(z[2 * k], z[2 * k + 1]);
      auto g = ED::Green_function(w, spin_down != 0, (size_t)label, false);
      put_complex(g, G_out + 2 * (size_t)k * g.v.size());
    }
  });
}

int ref_self_energy(int label, int spin_down, int nz, const double *z, double *S_out) {
  return guarded([&] {
    for (int k = 0; k < nz; ++k) {
      Complex w(z[2 * k], z[2 * k + 1]);
      auto g = ED::self_energy(w, spin_down != 0, (size_t)label);
      put_complex(g, S_out + 2 * (size_t)k * g.v.size());
    }
  });
}

int ref_hybridization_function(int label, int spin_down, int nz, const double *z, double *out) {
  return guarded([&] {
    for (int k = 0; k < nz; ++k) {
      Complex w(z[2 * k], z[2 * k + 1]);
      auto g = ED::hybridization_function(w, spin_down != 0, (size_t)label);
      put_complex(g, out + 2 * (size_t)k * g.v.size());
    }
  });
}

int ref_green_function_average(int label, int spin_down, double *out) {
  return guarded([&] {
    auto g = ED::Green_function_average(spin_down != 0, (size_t)label);
    put_complex(g, out);
  });
}

int ref_green_function_average_dim(int label, int spin_down, int *d) {
  return guarded([&] { *d = (int)ED::Green_function_average(spin_down != 0, (size_t)label).r; });
}

// cluster_averages: n operators (name, average, variance); names '\n'-separated.
int ref_cluster_averages(int label, int cap, int *n, double *ave, double *var, char *names, int names_size) {
  return guarded([&] {
    auto a = ED::cluster_averages((size_t)label);
    if ((int)a.size() > cap) throw qcm_error("ref_cluster_averages: capacity too small");
    *n = (int)a.size();
    std::string all;
    for (size_t i = 0; i < a.size(); ++i) {
      ave[i] = std::get<1>(a[i]);
      var[i] = std::get<2>(a[i]);
      all += std::get<0>(a[i]);
      all += '\n';
    }
    if ((int)all.size() + 1 > names_size) throw qcm_error("ref_cluster_averages: name buffer too small");
    std::memcpy(names, all.c_str(), all.size() + 1);
  });
}

int ref_model_size(const char *name, int *ns, int *nb, int *ne) {
  return guarded([&] {
    auto t = ED::model_size(name);
    *ns = (int)std::get<0>(t);
    *nb = (int)std::get<1>(t);
    *ne = (int)std::get<2>(t);
  });
}

int ref_exists(const char *model, const char *op, int *found) {
  return guarded([&] { *found = ED::exists(model, op) ? 1 : 0; });
}

int ref_matrix_elements(const char *model, const char *op, char *type, int type_size, int cap, int *n, int *r,
                        int *c, double *v) {
  return guarded([&] {
    auto m = ED::matrix_elements(model, op);
    if ((int)m.first.size() + 1 > type_size || (int)m.second.size() > cap)
      throw qcm_error("ref_matrix_elements: buffer too small");
    std::memcpy(type, m.first.c_str(), m.first.size() + 1);
    for (size_t i = 0; i < m.second.size(); ++i) {
      r[i] = (int)m.second[i].r;
      c[i] = (int)m.second[i].c;
      v[i] = m.second[i].v.real();
    }
    *n = (int)m.second.size();
  });
}

int ref_gf_density(int label, double *d) {
  return guarded([&] { *d = ED::Green_function_density((size_t)label); });
}

int ref_hopping_matrix(int label, int spin_down, int *d, double *H) {
  return guarded([&] {
    auto g = ED::hopping_matrix(spin_down != 0, (size_t)label);
    *d = (int)g.r;
    if (H) put_complex(g, H);
  });
}

int ref_hopping_matrix_full(int label, int spin_down, int diag, int *d, double *H) {
  return guarded([&] {
    auto g = ED::hopping_matrix_full(spin_down != 0, diag != 0, (size_t)label);
    *d = (int)g.r;
    if (H) put_complex(g, H);
  });
}

int ref_interactions(int label, int cap, int *n, int *r, int *c, double *v) {
  return guarded([&] {
    auto V = ED::interactions((size_t)label);
    if ((int)V.size() > cap) throw qcm_error("ref_interactions: capacity too small");
    for (size_t i = 0; i < V.size(); ++i) {
      r[i] = std::get<0>(V[i]);
      c[i] = std::get<1>(V[i]);
      v[i] = std::get<2>(V[i]);
    }
    *n = (int)V.size();
  });
}

int ref_tr_sigma_inf(int label, double *value) {
  return guarded([&] { *value = ED::tr_sigma_inf((size_t)label); });
}

int ref_susceptibility(int label, const char *op, int nw, const double *w, double *chi) {
  return guarded([&] {
    std::vector<Complex> z(nw);
    for (int i = 0; i < nw; ++i) z[i] = Complex(w[2 * i], w[2 * i + 1]);
    auto c = ED::susceptibility(op, z, (size_t)label);
    for (int i = 0; i < nw; ++i) {
      chi[2 * i] = c[i].real();
      chi[2 * i + 1] = c[i].imag();
    }
  });
}

int ref_susceptibility_poles(int label, const char *op, int cap, int *n, double *e, double *r) {
  return guarded([&] {
    auto p = ED::susceptibility_poles(op, (size_t)label);
    if ((int)p.size() > cap) throw qcm_error("ref_susceptibility_poles: capacity too small");
    for (size_t i = 0; i < p.size(); ++i) {
      e[i] = p[i].first;
      r[i] = p[i].second;
    }
    *n = (int)p.size();
  });
}

int ref_fidelity(int l1, int l2, double *f) {
  return guarded([&] { *f = ED::fidelity(l1, l2); });
}

int ref_potthoff(int label, double *omega) {
  return guarded([&] { *omega = ED::Potthoff_functional((size_t)label); });
}

// Lehmann representation: eigenvalues e[M], residues v (L x M complex, column-major).
// On entry *M is the capacity; on exit the actual number of poles.
int ref_qmatrix(int label, int spin_down, int *M, int *L, double *e, double *v) {
  return guarded([&] {
    auto q = ED::qmatrix(spin_down != 0, (size_t)label);
    int m = (int)q.first.size();
    int l = m ? (int)(q.second.size() / m) : 0;
    if (m > *M) throw qcm_error("ref_qmatrix: capacity too small");
    *M = m;
    *L = l;
    for (int i = 0; i < m; ++i) e[i] = q.first[i];
    for (size_t i = 0; i < q.second.size(); ++i) {
      v[2 * i] = q.second[i].real();
      v[2 * i + 1] = q.second[i].imag();
    }
  });
}

// Continued-fraction coefficients of the first state, real Hilbert space,
// trivial group: element (o1, o2), o2 <= o1, electron (pm=+1) or hole (pm=-1).
// On entry *n is the capacity of a and b; on exit the number of levels.
int ref_cf_coeffs(int label, int spin_down, int o1, int o2, int pm, int *n, double *a, double *b) {
  return guarded([&] {
    auto inst = dynamic_pointer_cast<model_instance<double>>(model_instances.at((size_t)label));
    if (!inst) throw qcm_error("ref_cf_coeffs: complex instance");
    if (!inst->gf_solved) inst->Green_function_solve();
    auto &st = *inst->states.begin();
    auto cf = dynamic_pointer_cast<continued_fraction_set>(spin_down ? st->gf_down : st->gf);
    if (!cf) throw qcm_error("ref_cf_coeffs: not a continued-fraction instance");
    continued_fraction &f = (pm > 0) ? cf->e[0](o1, o2) : cf->h[0](o1, o2);
    int m = (int)f.a.size();
    if (m > *n) throw qcm_error("ref_cf_coeffs: capacity too small");
    *n = m;
    for (int i = 0; i < m; ++i) a[i] = f.a[i];
    for (int i = 0; i < m && i < (int)f.b.size(); ++i) b[i] = f.b[i];
  });
}

// Ground-state vector of the first (lowest) state: dimension, energy, psi.
int ref_gs_vector(int label, long *dim, double *energy, double *psi) {
  return guarded([&] {
    auto inst = dynamic_pointer_cast<model_instance<double>>(model_instances.at((size_t)label));
    if (!inst) throw qcm_error("ref_gs_vector: complex instance");
    if (!inst->gs_solved) inst->low_energy_states();
    auto &st = *inst->states.begin();
    *dim = (long)st->psi.size();
    *energy = st->energy;
    if (psi) std::memcpy(psi, st->psi.data(), st->psi.size() * sizeof(double));
  });
}

// Sorted N-of-L bit strings of ED_halfbasis (src_ed/ED_basis.cpp:115-125).
int ref_halfbasis(int L, int N, unsigned *out, long *dim) {
  return guarded([&] {
    ED_halfbasis B(L, N);
    *dim = (long)B.dim;
    if (out)
      for (size_t i = 0; i < B.dim; ++i) out[i] = B.bin[i];
  });
}

// Factorized-basis Destroy (src_ed/ED_basis.cpp:79-110) applied to every state
// of sector (Nup, Ndn) of an L-orbital model for orbital a (a >= L: spin down).
// Writes, per source state, the target index (or -1) and the phase bit.
int ref_destroy_table(int L, int Nup, int Ndn, int a, long *target, int *phase) {
  return guarded([&] {
    sector sx(Nup + Ndn, Nup - Ndn, 0);
    int up = (a >= L) ? 0 : 1;
    sector sy(Nup + Ndn - 1, (Nup - up) - (Ndn - (1 - up)), 0);
    ED_factorized_basis Bx(sx, L), By(sy, L);
    for (uint32_t I = 0; I < Bx.dim; ++I) {
      auto T = Destroy(a, I, Bx, By);
      target[I] = std::get<3>(T) ? (long)std::get<0>(T) : -1;
      phase[I] = std::get<1>(T);
    }
  });
}

// y += H x in a sector of a solved-or-not instance, through the reference's
// factorized Hamiltonian (src_ed/Hamiltonian/Hamiltonian_Factorized.hpp:51-58).
void *ref_hv_create(int label, const char *sec, long *dim) {
  void *h = nullptr;
  int rc = guarded([&] {
    auto &I = *model_instances.at((size_t)label);
    if (!I.the_model->is_factorized) throw qcm_error("ref_hv_create: model is not factorized");
    auto *hh = new hv_handle;
    hh->H.reset(new Hamiltonian_Factorized<double>(I.the_model, I.value, sector(sec)));
    *dim = (long)hh->H->dim;
    h = hh;
  });
  return rc ? nullptr : h;
}

// The reference's CSR Hamiltonian (src_ed/Hamiltonian/Hamiltonian_CSR.hpp) of a
// sector of a model that is not factorized (one with symmetry generators): the
// symmetry-adapted (mixed) basis, for H.v parity in that basis.
void *ref_hv_create_csr(int label, const char *sec, long *dim) {
  void *h = nullptr;
  int rc = guarded([&] {
    auto &I = *model_instances.at((size_t)label);
    if (I.the_model->is_factorized) throw qcm_error("ref_hv_create_csr: model is factorized");
    auto *hh = new hv_handle;
    hh->H.reset(new Hamiltonian_CSR<double>(I.the_model, I.value, sector(sec)));
    *dim = (long)hh->H->dim;
    h = hh;
  });
  return rc ? nullptr : h;
}

int ref_hv_apply(void *h, const double *x, double *y) {
  return guarded([&] {
    auto *hh = (hv_handle *)h;
    size_t d = hh->H->dim;
    std::vector<double> xv(x, x + d), yv(y, y + d);
    hh->H->mult_add(xv, yv);
    std::memcpy(y, yv.data(), d * sizeof(double));
  });
}

// Timing entry: applies y += H x `reps` times on internally held vectors, so the
// measured time is the reference's mult_add alone (no copies across the FFI).
int ref_hv_bench(void *h, int reps, double *checksum) {
  return guarded([&] {
    auto *hh = (hv_handle *)h;
    size_t d = hh->H->dim;
    std::vector<double> x(d), y(d, 0.0);
    for (size_t i = 0; i < d; ++i) x[i] = 1.0 / (1.0 + (double)(i % 97));
    for (int r = 0; r < reps; ++r) hh->H->mult_add(x, y);
    double s = 0.0;
    for (size_t i = 0; i < d; i += 4099) s += y[i];
    *checksum = s;
  });
}

void ref_hv_destroy(void *h) { delete (hv_handle *)h; }

// ---- lattice layer (namespace QCM), argument conventions of the Python
// binding src_python/qcm_wrap.hpp:57-260 (orbital labels from 1, vectors as
// 3 integers, the unit cell defaulting to the identity) --------------------

int ref_qcm_great_reset(void) {
  return guarded([] { QCM::great_reset(); });
}

int ref_qcm_add_cluster(const long *cpos, int n, const long *pos, int ref, int conj) {
  return guarded([&] {
    vector<vector3D<int64_t>> p(n);
    for (int i = 0; i < n; ++i) p[i] = vector3D<int64_t>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    QCM::add_cluster(vector3D<int64_t>(cpos[0], cpos[1], cpos[2]), p, ref, conj != 0);
  });
}

int ref_qcm_add_system(const char *name, int clus) {
  return guarded([&] { QCM::add_system(name, clus); });
}

int ref_qcm_lattice_model(const char *name, int nvec, const long *super, const long *unit) {
  return guarded([&] {
    vector<int64_t> sl(super, super + 3 * nvec), uc(3 * nvec, 0);
    if (unit)
      uc.assign(unit, unit + 3 * nvec);
    else
      for (int i = 0; i < nvec; ++i) uc[4 * i] = 1;
    QCM::new_lattice_model(name, sl, uc);
  });
}

int ref_qcm_hopping_operator(const char *name, const long *link, double amp, int orb1, int orb2, int tau,
                             int sigma) {
  return guarded([&] {
    vector3D<int64_t> lk(link[0], link[1], link[2]);
    QCM::hopping_operator(name, lk, amp, orb1, orb2, tau, sigma);
  });
}

int ref_qcm_interaction_operator(const char *name, const long *link, double amp, int orb1, int orb2,
                                 const char *type) {
  return guarded([&] {
    vector3D<int64_t> lk(0, 0, 0);
    if (link) lk = vector3D<int64_t>(link[0], link[1], link[2]);
    QCM::interaction_operator(name, lk, amp, orb1, orb2, type);
  });
}

int ref_qcm_density_wave(const char *name, const char *type, const double *Q, const long *link, double amp,
                         int orb, double phase) {
  return guarded([&] {
    vector3D<int64_t> lk(0, 0, 0);
    if (link) lk = vector3D<int64_t>(link[0], link[1], link[2]);
    QCM::density_wave(name, lk, Complex(amp, 0.0), orb, vector3D<double>(Q[0], Q[1], Q[2]), phase, type);
  });
}

int ref_qcm_set_target_sectors(int n, const char **sectors) {
  return guarded([&] {
    if ((size_t)n != qcm_model->nsys)
      throw qcm_error("number of sector strings differs from the number of systems");
    qcm_model->sector_strings.assign(sectors, sectors + n);
  });
}

int ref_qcm_set_parameters(int nv, const char **names, const double *values, int ne, const char **enames,
                           const double *mult, const char **refs) {
  return guarded([&] {
    vector<pair<string, double>> v;
    for (int i = 0; i < nv; ++i) v.push_back({names[i], values[i]});
    vector<tuple<string, double, string>> e;
    for (int i = 0; i < ne; ++i) e.push_back({enames[i], mult[i], refs[i]});
    QCM::set_parameters(v, e);
  });
}

int ref_qcm_set_parameter(const char *name, double value) {
  return guarded([&] { QCM::set_parameter(name, value); });
}

int ref_qcm_new_model_instance(int label) {
  return guarded([&] { QCM::new_model_instance(label); });
}

int ref_qcm_erase_instance(int label) {
  return guarded([&] { QCM::erase_lattice_model_instance((size_t)label); });
}

int ref_qcm_dims(int *mixing, int *dim_gf, int *nsys) {
  return guarded([&] {
    *mixing = QCM::mixing();
    *dim_gf = (int)QCM::Green_function_dimension();
    *nsys = (int)qcm_model->nsys;
  });
}

int ref_qcm_set_wavevector_grid(int nkx, int nky, int nkz) {
  return guarded([&] { QCM::set_wavevector_grid(nkx, nky, nkz); });
}

int ref_qcm_frequency_grid(int n, const double *freqs, const double *weights) {
  return guarded([&] {
    grid_freqs.assign(freqs, freqs + n);
    grid_weights.assign(weights, weights + n);
  });
}

int ref_qcm_potthoff(int label, double *omega) {
  return guarded([&] { *omega = QCM::Potthoff_functional(label); });
}

// cluster one-body matrix of cluster `clus` (dim x dim complex, column-major)
int ref_qcm_cluster_hopping(int label, int clus, int spin_down, int *dim, double *out) {
  return guarded([&] {
    auto h = QCM::cluster_hopping_matrix((size_t)clus, spin_down != 0, label);
    *dim = (int)h.r;
    if (out) put_complex(h, out);
  });
}

// V(k) = t(k) - t' (src_qcm/CPT.cpp:22-64) at a wavevector given in the
// superdual basis (fractions of the reduced zone, as the grid integral uses)
int ref_qcm_V_superdual(int label, int spin_down, double w_re, double w_im, const double *k, int *dim,
                        double *out) {
  return guarded([&] {
    auto &inst = *lattice_model_instances.at(label);
    Green_function G = inst.cluster_Green_function(Complex(w_re, w_im), false, spin_down != 0);
    Green_function_k M(G, vector3D<double>(k[0], k[1], k[2]));
    inst.set_V(M);
    *dim = (int)M.V.r;
    if (out) put_complex(M.V, out);
  });
}

// the cluster Green function the lattice layer uses (remixed), dim x dim
int ref_qcm_cluster_gf(int label, int spin_down, double w_re, double w_im, int *dim, double *out) {
  return guarded([&] {
    auto &inst = *lattice_model_instances.at(label);
    Green_function G = inst.cluster_Green_function(Complex(w_re, w_im), false, spin_down != 0);
    *dim = (int)G.G.r;
    if (out) put_complex(G.G.build_matrix(), out);
  });
}

// CDMFT (src_qcm/CPT.cpp:356-560): variational parameters of cluster 0, the
// host function on a frequency grid, its matrices, and the distance
int ref_qcm_cdmft_variational_set(int n, const char **names) {
  return guarded([&] {
    vector<vector<string>> v(1);
    for (int i = 0; i < n; ++i) v[0].push_back(names[i]);
    QCM::CDMFT_variational_set(v);
  });
}

int ref_qcm_cdmft_host(int label, int n, const double *freqs, const double *weights) {
  return guarded([&] {
    vector<double> f(freqs, freqs + n), w(weights, weights + n);
    QCM::CDMFT_host(f, w, label);
  });
}

int ref_qcm_get_cdmft_host(int label, int spin_down, int iw, int clus, int *dim, double *out) {
  return guarded([&] {
    auto H = QCM::get_CDMFT_host(spin_down != 0, label);
    const matrix<Complex> &m = H.at((size_t)iw).at((size_t)clus);
    *dim = (int)m.r;
    if (out) put_complex(m, out);
  });
}

int ref_qcm_cdmft_distance(int label, int n, const double *p, int clus, double *d) {
  return guarded([&] {
    vector<double> v(p, p + n);
    *d = QCM::CDMFT_distance(v, clus, label);
  });
}

// ED label of system s of lattice instance `label` (nsys * label + s)
int ref_qcm_ed_label(int label, int s) { return (int)(qcm_model->nsys * (size_t)label + (size_t)s); }

}  // extern "C"
