// Model instance (see instance.hpp).
#include "instance.hpp"
#include "symmetry.hpp"

#include <algorithm>
#include <cmath>
#include <iomanip>
#include <limits>
#include <sstream>

#include "eigen.hpp"
#include "options.hpp"
#include "profile.hpp"

namespace qed {

namespace {
constexpr double kSmall = 1.0e-12;   // SMALL_VALUE (src_util/vector_num.hpp:23)
constexpr double kMiddle = 1.0e-8;   // MIDDLE_VALUE (src_util/vector_num.hpp:24)
constexpr double kMinGap = 1.0e-6;   // MIN_GAP (src_ed/model.hpp:20)

double max_gap() {
  double g = -std::log(opt_double("minimum_weight")) * opt_double("temperature");
  return g < kMinGap ? kMinGap : g;
}
}  // namespace

// symmetry_group::sector_is_valid (src_ed/symmetry_group.cpp:515-532): irrep below the group order
bool sector_is_valid(const Sector &s, int n_orb, int g) {
  if (s.N < Sector::odd) {
    if (s.N < 0 || s.N > 2 * n_orb) return false;
    if (s.S < Sector::odd) {
      if (s.S > s.N || s.S < -s.N) return false;
      if ((s.N + s.S) % 2) return false;
    }
  }
  if (s.S < Sector::odd && (s.S > n_orb || s.S < -n_orb)) return false;
  return s.irrep >= 0 && s.irrep < g;
}

// symmetry_group::shift_sector (src_ed/symmetry_group.cpp:540-558)
Sector shift_sector(const Sector &s, int pm, int spin) {
  Sector t = s;
  t.N += pm;
  t.S += spin ? -pm : pm;
  return t;
}

Instance::Instance(int lab, std::shared_ptr<Model> m, std::map<std::string, double> val,
                   const std::string &sectors)
    : label(lab), model(std::move(m)), value(std::move(val)) {
  // model_instance_base ctor (src_ed/model_instance_base.cpp:14-130)
  if (value.empty())
    fail(QED_ERR_ARGUMENT, "ED model instance (label = " + std::to_string(label) + ") for model " +
                               model->name + " has no parameters!");
  char gf = opt_char("GF_method");
  if (gf == 'L' && opt_bool("continued_fraction")) gf = 'F';
  if (gf == 'L' && opt_bool("combine_mcf"))
    fail(QED_ERR_UNSUPPORTED, "Q-matrix to matrix-continued-fraction conversion (GF_method 'L' with combine_mcf) "
                              "is not in this solver");
  if (gf == 'M' && opt_bool("combine_mcf"))
    fail(QED_ERR_UNSUPPORTED, "combining the electron and hole matrix continued fractions (combine_mcf) is not in "
                              "this solver");
  use_cf = (gf == 'F');
  use_mcf = (gf == 'M');
  mcf_qr = opt_bool("block_Lanczos_QR");
  if (opt_char("Ground_state_method") != 'L')
    fail(QED_ERR_UNSUPPORTED, "only the Lanczos ground-state method ('L') is in this solver");
  if (opt_int("n_states") > 1)
    fail(QED_ERR_UNSUPPORTED, "n_states > 1 needs the Davidson solver, not in this solver");
  for (auto &v : value) {
    const Operator &op = *model->term.at(v.first);
    mix |= op.mix;
    if (op.is_interaction) is_correlated = true;
  }
  if (mix > 5) mix &= mixing::full;
  if (mix == 5) mix &= mixing::anomalous;
  if (model->mix == -1) model->mix = mix;
  else if ((mix | model->mix) != model->mix)
    fail(QED_ERR_ARGUMENT, "The new instance mixing state of model " + model->name + " (" +
                               std::to_string(mix) + ") is not compatible with the first instance mixing (" +
                               std::to_string(model->mix) + ")");
  else mix = model->mix;
  if (mix != mixing::normal && mix != mixing::up_down)
    fail(QED_ERR_UNSUPPORTED, "mixing " + std::to_string(mix) +
                                  " (anomalous / spin-flip) is outside the spin-factorized solver");
  {
    std::lock_guard<std::mutex> l(model->mtx);
    if (!model->format) {
      const char f = opt_char("Hamiltonian_format");
      if (f != 'O' && f != 'S' && f != 'N' && f != 'F' && f != 'E')
        fail(QED_ERR_ARGUMENT, "Hamiltonian_format is not one of : N, S, O, F, E");
      model->format = f;
      // every operator this solver accepts is factorizable, and the mixing is
      // normal or up_down here, so the format alone decides
      model->factorized = (f == 'F');
    }
  }
  dim_GF = model->n_sites;
  // sectors: slash-separated list
  std::stringstream ss(sectors);
  std::string item;
  while (std::getline(ss, item, '/')) {
    if (item.empty()) continue;
    Sector S(item);
    if (!sector_is_valid(S, model->n_orb, model->group ? model->group->g() : 1))
      fail(QED_ERR_ARGUMENT, "sector " + item + " is not valid");
    if (S.S && mix == mixing::normal) mix = mixing::up_down;
    if (S.S >= Sector::odd)
      fail(QED_ERR_ARGUMENT, "sector string " + S.name() +
                                 " defines a non conserved spin, but spin is conserved in the model (instance " +
                                 std::to_string(label) + ")");
    if (S.N >= Sector::odd)
      fail(QED_ERR_ARGUMENT, "sector string " + S.name() +
                                 " defines a non conserved particle number, but particle number is conserved in the model (instance " +
                                 std::to_string(label) + ")");
    target_sectors.insert(S);
  }
  if (target_sectors.empty()) fail(QED_ERR_ARGUMENT, "no target sectors were specified for model " + model->name);
  terms = collect_terms(*model, value);
  set_hopping_matrix();
}

// set_hopping_matrix (src_ed/model_instance.hpp:424-474), real case.
void Instance::set_hopping_matrix() {
  if (hopping_solved) return;
  const int no = model->n_orb, ns = model->n_sites, nb = model->n_bath;
  SEF_bath = 0.0;
  for (int sp = 0; sp < 2; ++sp) {
    const std::vector<double> &t = sp ? terms.t_dn : terms.t_up;
    tc[sp].assign((size_t)ns * ns, 0.0);
    tb[sp].assign((size_t)nb * nb, 0.0);
    tcb[sp].assign((size_t)ns * nb, 0.0);
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < ns; ++b) tc[sp][a + (size_t)ns * b] = t[(size_t)a * no + b];
    for (int a = 0; a < nb; ++a)
      for (int b = 0; b < nb; ++b) tb[sp][a + (size_t)nb * b] = t[(size_t)(ns + a) * no + ns + b];
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < nb; ++b) tcb[sp][a + (size_t)ns * b] = t[(size_t)a * no + ns + b];
    if (nb) {
      tb_nd[sp] = tb[sp];
      tcb_nd[sp] = tcb[sp];
      bool diag = true;
      for (int a = 0; a < nb; ++a)
        for (int b = 0; b < nb; ++b)
          if (a != b && std::fabs(tb[sp][a + (size_t)nb * b]) > 1e-8) diag = false;
      if (!diag) {
        std::vector<double> d, Sb;
        if (!sym_eig(nb, tb[sp], d, &Sb)) fail(QED_ERR_INTERNAL, "bath diagonalisation failed");
        std::fill(tb[sp].begin(), tb[sp].end(), 0.0);
        for (int a = 0; a < nb; ++a) tb[sp][a + (size_t)nb * a] = d[a];
        std::vector<double> t2((size_t)ns * nb, 0.0);
        for (int a = 0; a < ns; ++a)
          for (int b = 0; b < nb; ++b) {
            double s = 0.0;
            for (int k = 0; k < nb; ++k) s += tcb[sp][a + (size_t)ns * k] * Sb[k + (size_t)nb * b];
            t2[a + (size_t)ns * b] = s;
          }
        tcb[sp] = t2;
      }
      // bath contribution to the Potthoff functional
      if (sp == 0 || (mix & mixing::up_down))
        for (int i = 0; i < nb; ++i)
          if (tb[sp][i + (size_t)nb * i] < 0) SEF_bath -= tb[sp][i + (size_t)nb * i];
    }
  }
  if (mix == mixing::normal) SEF_bath *= 2.0;
  hopping_solved = true;
}

std::vector<double> Instance::hopping_matrix(bool spin_down) const {
  return tc[(spin_down && (mix & mixing::up_down)) ? 1 : 0];
}

// The (n_sites + n_bath)^2 one-body matrix: cluster block, bath block (diagonal
// form when diag, as given otherwise), cluster-bath block and its transpose.
// With diag, the cluster-bath columns carry the bath eigenvectors, whose signs
// are a convention of the eigensolver.
std::vector<double> Instance::hopping_matrix_full(bool spin_down, bool diag) const {
  // the reference keeps spin-down matrices only for up_down mixing (its call
  // fails on the empty ones otherwise)
  if (spin_down && !(mix & mixing::up_down))
    fail(QED_ERR_ARGUMENT, "hopping_matrix_full: no spin-down one-body matrices without up_down mixing");
  const int ns = model->n_sites, nb = model->n_bath, d = ns + nb;
  // likewise it keeps the undiagonalised bath matrices only when there is a bath
  if (!diag && nb == 0)
    fail(QED_ERR_ARGUMENT, "hopping_matrix_full: no undiagonalised bath matrices in a model without bath");
  const int sp = spin_down ? 1 : 0;
  const std::vector<double> &B = diag ? tb[sp] : tb_nd[sp], &CB = diag ? tcb[sp] : tcb_nd[sp];
  std::vector<double> H((size_t)d * d, 0.0);
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < ns; ++b) H[a + (size_t)d * b] = tc[sp][a + (size_t)ns * b];
  for (int a = 0; a < nb; ++a)
    for (int b = 0; b < nb; ++b) H[(ns + a) + (size_t)d * (ns + b)] = B[a + (size_t)nb * b];
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < nb; ++b) {
      H[a + (size_t)d * (ns + b)] = CB[a + (size_t)ns * b];
      H[(ns + b) + (size_t)d * a] = CB[a + (size_t)ns * b];
    }
  return H;
}

std::vector<Element> Instance::interactions() const {
  std::vector<Element> V;
  for (auto &x : value) {
    const Operator &op = *model->term.at(x.first);
    if (!op.is_interaction) continue;
    for (auto &e : op.elements) V.push_back({e.r, e.c, e.v * x.second});
  }
  return V;
}

// Trace of the self-energy at infinite frequency: Re tr Sigma(i / x) at
// x = 1e-5, 2e-5, 3e-5 (both spins, or twice the up one for normal mixing),
// extrapolated to x = 0 by the interpolating polynomial through the three
// points (Lagrange form; the reference uses Neville's scheme for the same
// polynomial, src_ed/model_instance.cpp:186-222).
double Instance::tr_sigma_inf(Workspace &ws) {
  const int n = dim_GF;
  constexpr int kNW = 3;
  double x[kNW], S[kNW];
  std::vector<cplx> z(kNW), sig((size_t)kNW * n * n);
  for (int i = 0; i < kNW; ++i) {
    x[i] = (i + 1) * 1.0e-5;
    z[i] = cplx(0.0, 1.0 / x[i]);
  }
  for (int sd = 0; sd < ((mix & mixing::up_down) ? 2 : 1); ++sd) {
    self_energy(z.data(), kNW, sd == 1, sig.data(), ws);
    for (int i = 0; i < kNW; ++i) {
      double t = 0.0;
      for (int j = 0; j < n; ++j) t += sig[(size_t)i * n * n + j + (size_t)n * j].real();
      S[i] = (sd == 0) ? t : S[i] + t;
    }
  }
  if (mix == mixing::normal)
    for (int i = 0; i < kNW; ++i) S[i] *= 2.0;
  double s0 = 0.0;
  for (int i = 0; i < kNW; ++i) {
    double w = 1.0;
    for (int j = 0; j < kNW; ++j)
      if (j != i) w *= (0.0 - x[j]) / (x[i] - x[j]);
    s0 += w * S[i];
  }
  return s0;
}

std::vector<Instance::SusQ> Instance::susceptibility_qmatrices(const std::string &opname, Workspace &ws) {
  if (!model->term.count(opname)) fail(QED_ERR_ARGUMENT, "Operator " + opname + " is not defined in the model.");
  if (!value.count(opname))
    fail(QED_ERR_ARGUMENT, "operator " + opname + " is not activated in instance " + std::to_string(label));
  if (!gs_solved) low_energy_states(ws);
  const SpinData t = collect_terms(*model, {{opname, 1.0}});
  std::vector<SusQ> out;
  for (auto &sec : target_sectors)
    for (auto &st : states) {
      if (!(st->sec == sec)) continue;
      SectorOp H(terms, sec, ws, &tables);
      if (H.D == 0) continue;
      SectorOp O(t, sec, ws, &op_tables[opname]);
      std::vector<DevBuf<double>> b(1);
      b[0].alloc(H.D);
      SubList none;
      launch_hv(O.op, st->psi.p, 1.0, b[0].p, none, 0, ws.red, ws.stream);  // b = O psi
      SusQ q;
      q.st = st.get();
      int M = 0;
      bool ok;
      if (!model->factorized && (long)H.D < opt_int("max_dim_full")) {
        std::vector<double> U, ph(H.D);
        dense_eigensystem(H, ws, q.e, U);
        b[0].download(ph.data(), H.D, ws.stream);
        ws.sync();
        M = (int)H.D;
        q.V.assign(M, 0.0);
        for (int k = 0; k < M; ++k) {
          double acc = 0.0;
          for (size_t j = 0; j < H.D; ++j) acc += ph[j] * U[(size_t)k * H.D + j];
          q.V[k] = acc;
        }
        ok = true;
      } else {
        ok = band_lanczos_qmatrix(H, ws, b, q.e, q.V, M);
      }
      if (!ok || M == 0) continue;
      q.e.resize(M);
      q.V.resize(M);
      for (auto &x : q.e) x -= st->energy;
      out.push_back(std::move(q));
    }
  return out;
}

void Instance::susceptibility(const std::string &opname, const cplx *w, int nw, cplx *chi, Workspace &ws) {
  const auto qs = susceptibility_qmatrices(opname, ws);
  DevBuf<double> dz(2 * (size_t)std::max(nw, 1)), dG(2 * (size_t)std::max(nw, 1));
  dz.upload(reinterpret_cast<const double *>(w), 2 * (size_t)nw, ws.stream);
  QED_CUDA(cudaMemsetAsync(dG.p, 0, dG.bytes(), ws.stream));
  std::vector<DevBuf<double>> keep;
  for (auto &q : qs) {
    std::vector<double> V(q.V);
    const double sw = std::sqrt(q.st->weight);
    for (auto &x : V) x *= sw;
    keep.emplace_back(q.e.size());
    keep.back().upload(q.e, ws.stream);
    keep.emplace_back(V.size());
    keep.back().upload(V, ws.stream);
    launch_qmatrix_gf(1, (int)q.e.size(), keep[keep.size() - 2].p, keep.back().p, nw, dz.p, dG.p, ws.stream);
  }
  dG.download(reinterpret_cast<double *>(chi), 2 * (size_t)nw, ws.stream);
  ws.sync();
}

std::vector<std::pair<double, double>> Instance::susceptibility_poles(const std::string &opname, Workspace &ws) {
  const auto qs = susceptibility_qmatrices(opname, ws);
  std::vector<std::pair<double, double>> chi, chi2;
  for (auto &q : qs)
    for (size_t i = 0; i < q.e.size(); ++i) {
      if (q.e[i] < 1e-8) continue;
      const double r = q.V[i] * q.V[i] * q.st->weight;
      if (r > 1e-6) chi.push_back({q.e[i], r});
    }
  for (auto &x : chi) {  // poles closer than 1e-4 are merged, in order of appearance
    size_t j = 0;
    for (; j < chi2.size(); ++j)
      if (std::fabs(chi2[j].first - x.first) < 1e-4) {
        chi2[j].second += x.second;
        break;
      }
    if (j == chi2.size()) chi2.push_back(x);
  }
  return chi2;
}

std::string Instance::gs_string() const {
  if (!is_correlated) return "uncorrelated";
  std::map<Sector, double, SectorLess> ws;
  for (auto &s : states) ws[s->sec] += s->weight;
  std::ostringstream out;
  bool first = true;
  for (auto &x : ws) {
    if (!first) out << '/';
    first = false;
    out << x.first.name() << ':' << std::setprecision(3) << x.second;
  }
  return out.str();
}

std::string Instance::where(const Sector &s) const {
  return "\n  in cluster model '" + model->name + "', instance '" + model->name + "_" + std::to_string(label) +
         "', sector '" + s.name() + "'";
}

// one_body_solve (src_ed/model_instance.hpp:1164-1256): without interaction the
// cluster + bath problem is one-body. Per spin, the (n_sites + n_bath)^2
// one-body matrix (bath diagonalised) is diagonalised; the Q-matrix holds all
// its poles with the cluster components of the eigenvectors, the ground-state
// energy is the sum of the negative one-body energies, and M_ab = <c+_b c_a> is
// the sum over occupied orbitals. Reproduced as the reference has it: the
// spin-down branch adds the spin-up negative energies again, and only the
// spin-up Q-matrix is checked for unitarity. The operator averages come from M
// (one_body_operator::average_from_GF, src_ed/Operators/one_body_operator.hpp:420-440);
// their variances are undefined (NaN), as in the reference.
void Instance::one_body_solve(Workspace &ws) {
  const int ns = model->n_sites, nb = model->n_bath, d = ns + nb;
  use_cf = false;  // the one-body Green function is a Q-matrix (GF_format_BL)
  states.clear();
  auto st = std::make_shared<State>();
  double gs = 0.0;
  std::vector<double> Mocc[2];
  const int nsp = (mix & mixing::up_down) ? 2 : 1;
  std::vector<double> eup;
  for (int sp = 0; sp < nsp; ++sp) {
    std::vector<double> H((size_t)d * d, 0.0), e, U;
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < ns; ++b) H[a + (size_t)d * b] = tc[sp][a + (size_t)ns * b];
    for (int a = 0; a < nb; ++a)
      for (int b = 0; b < nb; ++b) H[(ns + a) + (size_t)d * (ns + b)] = tb[sp][a + (size_t)nb * b];
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < nb; ++b) {
        H[a + (size_t)d * (ns + b)] = tcb[sp][a + (size_t)ns * b];
        H[(ns + b) + (size_t)d * a] = tcb[sp][a + (size_t)ns * b];
      }
    if (!sym_eig(d, H, e, &U)) fail(QED_ERR_INTERNAL, "one-body eigensolver failed");
    QMat &q = st->q[sp];
    q.L = ns;
    q.M = d;
    q.e = e;
    q.V.assign((size_t)d * ns, 0.0);
    for (int k = 0; k < d; ++k)
      for (int i = 0; i < ns; ++i) q.V[(size_t)k * ns + i] = U[i + (size_t)d * k];
    Mocc[sp].assign((size_t)d * d, 0.0);
    for (int a = 0; a < d; ++a)
      for (int b = 0; b < d; ++b) {
        double m = 0.0;
        for (int r = 0; r < d; ++r)
          if (e[r] < 0.0) m += U[a + (size_t)d * r] * U[b + (size_t)d * r];
        Mocc[sp][b + (size_t)d * a] = m;
      }
    if (sp == 0) eup = e;
    for (double x : eup)
      if (x < 0.0) gs += x;
    if (sp == 0) {  // Q.check_norm(1e-6)
      double ztot = 0.0;
      for (int i = 0; i < ns; ++i) {
        double z = 0.0;
        for (int k = 0; k < d; ++k) z += q.V[(size_t)k * ns + i] * q.V[(size_t)k * ns + i];
        ztot += (z - 1.0) * (z - 1.0);
        for (int j = 0; j < i; ++j) {
          double zz = 0.0;
          for (int k = 0; k < d; ++k) zz += q.V[(size_t)k * ns + i] * q.V[(size_t)k * ns + j];
          ztot += 2.0 * zz * zz;
        }
      }
      if (ztot > 1e-6) fail(QED_ERR_QMATRIX, "Q-matrix does not satisfy unitary condition by " + std::to_string(ztot));
    }
    q.de.upload(q.e, ws.stream);
    q.dV.upload(q.V, ws.stream);
  }
  ws.sync();
  for (int sp = 0; sp < nsp; ++sp) Mfull[sp].assign(Mocc[sp].begin(), Mocc[sp].end());
  if (mix == mixing::normal) gs *= 2.0;
  GS_energy = gs;
  E0 = gs;
  st->energy = gs;
  st->weight = 1.0;
  states.push_back(st);
  // cluster_averages from M: trace of M times the operator's one-body block
  averages.clear();
  const int no = model->n_orb;
  for (auto &v : value) {
    const Operator &op = *model->term.at(v.first);
    double ave = std::numeric_limits<double>::quiet_NaN();
    if (!op.is_interaction) {
      ave = 0.0;
      for (int sp = 0; sp < nsp; ++sp)
        for (auto &x : op.elements) {
          const bool down = x.r >= no;
          if (down != (sp == 1) || (x.c >= no) != down) continue;
          const int r = x.r - (down ? no : 0), c = x.c - (down ? no : 0);
          ave += Mocc[sp][r + (size_t)d * c] * x.v;
        }
      if (mix == mixing::normal) ave *= 2.0;
      if (op.target == 1) ave *= (v.first == "mu" ? -1.0 : 1.0) / ns;
    }
    averages.emplace_back(v.first, ave, std::numeric_limits<double>::quiet_NaN());
  }
  gs_solved = true;
  finish_gf();
}

size_t Instance::sector_dim(const Sector &s) const {
  const int L = model->n_orb, nu = s.Nup(), nd = s.Ndw();
  if (nu < 0 || nu > L || nd < 0 || nd > L) return 0;
  const size_t d = (size_t)binom(L, nu) * (size_t)binom(L, nd);
  return has_group() ? d / (size_t)model->group->g() + 1 : d;  // a point group: about d / g per irrep
}

// Eigenvalue pass of one sector: Hamiltonian_Dense::states
// (src_ed/Hamiltonian/Hamiltonian_Dense.hpp:110-125) below max_dim_full in the
// non-factorized formats, the Lanczos eigenvalue pass otherwise.
void Instance::solve_sector(const Sector &s, SectorSolve &out, Workspace &ws, DeferredSectors *defer) {
  require_supported_group();
  out.sec = s;
  if (has_group()) {  // the symmetry-adapted basis: dense below max_dim_full, else Lanczos on the CSR product
    try {
      auto H = mixed_sector(s, ws);
      out.dim = H->D;
      if (H->D == 0) return;
      if ((long)H->D < opt_int("max_dim_full")) {
        out.dense = true;
        std::vector<double> A = H->dense(ws.stream);
        if (!sym_eig((int)H->D, A, out.w, &out.U)) fail(QED_ERR_INTERNAL, "dense eigensolver did not converge");
      } else {
        out.lanczos = lanczos_energy_mixed(*H, ws, (uint64_t)opt_int("seed"));
      }
    } catch (const Error &e) {
      fail(e.code, std::string(e.what()) + where(s));
    }
    return;
  }
  try {
    auto Hp = std::make_unique<SectorOp>(terms, s, ws, &tables);
    SectorOp &H = *Hp;
    out.dim = H.D;
    if (H.D == 0) return;
    if (!model->factorized && (long)H.D < opt_int("max_dim_full")) {
      out.dense = true;
      dense_eigensystem(H, ws, out.w, out.U);
    } else if (defer) {
      LanczosBatchItem it;
      it.H = Hp.get();
      it.seed = (uint64_t)opt_int("seed");
      it.out = &out.lanczos;
      it.where = where(s);
      std::lock_guard<std::mutex> l(defer->m);
      (H.D <= lanczos_job_max_dim() ? defer->items : defer->large).push_back(it);
      defer->ops.push_back(std::move(Hp));
    } else {
      out.lanczos = lanczos_energy(H, ws, (uint64_t)opt_int("seed"));
    }
  } catch (const Error &e) {
    fail(e.code, std::string(e.what()) + where(s));
  }
}

// The selection part of low_energy_states (src_ed/model_instance.hpp:268-347),
// in target-sector order: the running minimum of Hamiltonian::states
// (src_ed/Hamiltonian/Hamiltonian_base.hpp:197-206), compute_weights, the
// minimum_weight cut and the renormalisation.
void Instance::select_states(std::vector<SectorSolve> &r) {
  GS_energy = 1.0e12;
  states.clear();
  const double gap = max_gap();
  for (auto &x : r) {
    if (x.dim == 0) continue;
    if (x.dense) {
      if (x.w[0] < GS_energy) GS_energy = x.w[0];
      for (size_t i = 0; i < x.w.size(); ++i) {
        if (x.w[i] - GS_energy > gap) break;
        auto st = std::make_shared<State>();
        st->sec = x.sec;
        st->energy = x.w[i];
        st->dense = true;
        st->hpsi.assign(x.U.begin() + i * x.dim, x.U.begin() + (i + 1) * x.dim);
        states.push_back(st);
      }
      continue;
    }
    auto st = std::make_shared<State>();
    st->sec = x.sec;
    st->energy = x.lanczos.energy;
    if (st->energy < GS_energy) GS_energy = st->energy;
    if (st->energy - GS_energy > gap) continue;
    st->lanczos = std::move(x.lanczos);
    states.push_back(st);
  }
  compute_weights();
  const double wmin = opt_double("minimum_weight");
  std::vector<std::shared_ptr<State>> kept;
  double tot = 0.0;
  for (auto &x : states)
    if (x->weight >= wmin) {
      kept.push_back(x);
      tot += x->weight;
    }
  states = kept;
  for (auto &x : states) x->weight /= tot;
  bool updown = false;
  for (auto &x : states)
    if (x->sec.S) updown = true;
  if (mix == mixing::normal && updown) mix = mixing::up_down;
  GS_energy = 1.0e18;
  E0 = 0.0;
  for (auto &x : states) {
    E0 += x->weight * x->energy;
    if (x->energy < GS_energy) GS_energy = x->energy;
  }
}

// Ground-state vector of a selected state: the eigenvector pass replays the
// Lanczos recurrence (same start vector, same tridiagonal); dense states
// upload their eigenvector.
void Instance::state_vector(State &st, Workspace &ws) {
  try {
    if (st.dense) {
      st.psi.upload(st.hpsi, ws.stream);
      ws.sync();
      st.hpsi = std::vector<double>();
      return;
    }
    if (has_group()) {
      auto H = mixed_sector(st.sec, ws);
      lanczos_eigenvector_mixed(*H, ws, st.lanczos, (uint64_t)opt_int("seed"), st.psi);
    } else {
      SectorOp H(terms, st.sec, ws, &tables);
      lanczos_eigenvector(H, ws, st.lanczos, (uint64_t)opt_int("seed"), st.psi);
    }
  } catch (const Error &e) {
    fail(e.code, std::string(e.what()) + where(st.sec));
  }
  st.lanczos = LanczosResult();
}

// cluster_averages (src_ed/model_instance.hpp:149-173): for each operator O of
// the instance, sum over states of weight * <psi|O|psi> and weight * |O psi|^2
// (HS_Hermitian_operator::expectation_value, src_ed/Operators/HS_Hermitian_operator.hpp:46-52),
// variance = second - first^2; operators on cluster orbitals only (target 1)
// are scaled by norm = 1/n_sites (-1/n_sites for "mu"), Hermitian_operator.hpp:41-43.
// O psi is one H.v with the operator's own tables and the <x,y>, <y,y>
// reductions of the column pass.
void Instance::finish_gs(Workspace &ws) {
  PhaseScope ps(kPhAverages);
  averages.clear();
  for (auto &v : value) {
    const Operator &op = *model->term.at(v.first);
    const SpinData t = collect_terms(*model, {{v.first, 1.0}});
    double ave = 0.0, var = 0.0;
    for (auto &st : states) {
      SubList none;
      if (has_group()) {  // the operator in the state's symmetry-adapted basis
        MixedHamiltonian O(*model->group, mixed_terms(*model, {{v.first, 1.0}}), st->sec.irrep, st->sec.Nup(),
                           st->sec.Ndw(), ws.stream);
        if (O.D == 0) continue;
        DevBuf<double> y(O.D);
        const int nb = O.apply_full(st->psi.p, 1.0, y.p, none, 3, ws.red, ws.stream);
        const double *r = ws.sums(nb, 2);
        ave += st->weight * r[0];
        var += st->weight * r[1];
        continue;
      }
      SectorOp O(t, st->sec, ws, &op_tables[v.first]);
      if (O.D == 0) continue;
      DevBuf<double> y(O.D);
      const int nb = launch_hv(O.op, st->psi.p, 1.0, y.p, none, 3, ws.red, ws.stream);
      const double *r = ws.sums(nb, 2);
      ave += st->weight * r[0];
      var += st->weight * r[1];
    }
    var -= ave * ave;
    if (op.target == 1) {
      const double norm = (v.first == "mu" ? -1.0 : 1.0) / model->n_sites;
      ave *= norm;
      var *= norm * norm;
    }
    averages.emplace_back(v.first, ave, var);
  }
  gs_solved = true;
}

// low_energy_states (src_ed/model_instance.hpp:245-347)
void Instance::require_supported_group() const {
  if (!has_group()) return;
  if (model->group->has_complex_irrep)
    fail(QED_ERR_UNSUPPORTED, "model " + model->name +
                                  ": point group with complex characters (a generator of order above 2) needs "
                                  "a complex Hilbert space, which this solver does not provide");
  if (use_cf || use_mcf)
    fail(QED_ERR_UNSUPPORTED, "model " + model->name +
                                  ": continued-fraction Green functions (GF_method 'F' or 'M') of models with a "
                                  "point group are not in this solver; use the Lehmann form ('L')");
}

std::unique_ptr<MixedHamiltonian> Instance::mixed_sector(const Sector &s, Workspace &ws) const {
  return std::make_unique<MixedHamiltonian>(*model->group, mixed_terms(*model, value), s.irrep, s.Nup(), s.Ndw(),
                                            ws.stream);
}

std::pair<double, std::string> Instance::low_energy_states(Workspace &ws) {
  if (gs_solved) return {GS_energy, gs_string()};
  require_supported_group();
  if (!is_correlated) {
    one_body_solve(ws);
    return {GS_energy, gs_string()};
  }
  std::vector<SectorSolve> r(target_sectors.size());
  size_t i = 0;
  for (auto &s : target_sectors) solve_sector(s, r[i++], ws);
  select_states(r);
  for (auto &x : states) state_vector(*x, ws);
  finish_gs(ws);
  return {GS_energy, gs_string()};
}

// compute_weights (src_ed/model_instance.hpp:356-417)
void Instance::compute_weights() {
  const double T = opt_double("temperature");
  if (T < kMiddle) {
    double e0 = 1e12;
    for (auto &x : states) e0 = std::min(e0, x->energy);
    std::vector<std::shared_ptr<State>> keep;
    for (auto &x : states)
      if (x->energy - e0 <= kSmall) keep.push_back(x);
    states = keep;
    if (states.empty()) fail(QED_ERR_INTERNAL, "instance has no low-energy state!");
    for (auto &x : states) x->weight = 1.0 / states.size();
    E0 = states.front()->energy;
    return;
  }
  const double gap = max_gap();
  std::vector<std::shared_ptr<State>> keep;
  for (auto &x : states)
    if (x->energy - GS_energy <= gap) keep.push_back(x);
  states = keep;
  double Z = 0.0;
  for (auto &x : states) {
    x->weight = std::exp(-(x->energy - GS_energy) / T);
    Z += x->weight;
  }
  E0 = GS_energy - T * std::log(Z);
  for (auto &x : states) x->weight /= Z;
}

void Instance::apply_cdag(const State &st, int pm, int spin, int orb, const SectorOp &H, double *y,
                          double coef, bool accumulate, Workspace &ws) {
  const int L = model->n_orb;
  const int src_nup = st.sec.Nup(), src_ndn = st.sec.Ndw();
  const uint32_t du_s = (uint32_t)((src_nup < 0 || src_nup > L) ? 0 : binom(L, src_nup));
  launch_cdag_gather(L, spin, orb, pm, H.up->bits.p, H.up->dim, H.dn->bits.p, H.dn->dim, src_nup, src_ndn,
                     du_s, st.psi.p, y, coef, accumulate ? 1 : 0, ws.stream);
}

// Q-matrix streamlining (Q_matrix::streamline / streamlineQ, src_ed/Q_matrix.hpp:181-318)
static void streamline(std::vector<double> &e, std::vector<double> &V, int L) {
  const double wtol = opt_double("Qmatrix_wtol"), vtol = opt_double("Qmatrix_vtol");
  if (vtol < 1e-12) return;
  const int M = (int)e.size();
  std::vector<double> e2, V2;
  e2.reserve(M);
  V2.reserve(V.size());
  for (int i = 0; i < M; ++i) {
    int j = i + 1;
    for (; j < M; ++j)
      if (std::fabs(e[j] - e[i]) > wtol) break;
    const int n = j - i;
    if (n == 1) {
      double nn = 0.0;
      for (int a = 0; a < L; ++a) nn += V[(size_t)i * L + a] * V[(size_t)i * L + a];
      if (nn >= vtol) {
        e2.push_back(e[i]);
        V2.insert(V2.end(), V.begin() + (size_t)i * L, V.begin() + (size_t)(i + 1) * L);
      }
    } else {
      std::vector<double> QQ((size_t)L * L, 0.0), d, U;
      for (int a = 0; a < L; ++a)
        for (int b = 0; b < L; ++b) {
          double s = 0.0;
          for (int k = i; k < j; ++k) s += V[(size_t)k * L + a] * V[(size_t)k * L + b];
          QQ[a + (size_t)L * b] = s;
        }
      if (!sym_eig(L, QQ, d, &U)) fail(QED_ERR_INTERNAL, "streamline eigensolver failed");
      for (int k = 0; k < L; ++k)
        if (d[k] > vtol) {
          e2.push_back(e[i]);
          double sq = std::sqrt(d[k]);
          for (int a = 0; a < L; ++a) V2.push_back(U[a + (size_t)L * k] * sq);
        }
    }
    i += n - 1;
  }
  e = e2;
  V = V2;
}

// build_qmatrix (src_ed/model_instance.hpp:711-817), sequential branch.
// One half of build_qmatrix: the hole (s = 0, pm = -1) or electron (s = 1,
// pm = +1) excitations of state st, spin_down or up: start vectors c / c^+ |psi>,
// band Lanczos (or the full eigensystem of a small non-factorized sector),
// energy shift and sign, streamline.
void Instance::qmatrix_part(State &st, bool spin_down, int s, QPart &out, Workspace &ws) {
  if (has_group()) {
    qmatrix_part_mixed(st, spin_down, s, out, ws);
    return;
  }
  const int p = model->n_sites;
  const int pm = 2 * s - 1;
  const int spin = spin_down ? 1 : 0;
  out.e.clear();
  out.V.clear();
  Sector tsec = shift_sector(st.sec, pm, spin);
  if (!sector_is_valid(tsec, model->n_orb)) return;
  SectorOp H(terms, tsec, ws, &tables);
  if (H.D == 0) return;
  std::vector<DevBuf<double>> phi;
  phi.reserve(p);
  {
    PhaseScope ps_cdag(kPhCdag);
    for (int i = 0; i < p; ++i) {
      phi.emplace_back(H.D);
      apply_cdag(st, pm, spin, i, H, phi.back().p, 1.0, false, ws);
    }
    ws.sync();
  }
  std::vector<double> ev, Q;
  int M = 0;
  bool ok;
  if (!model->factorized && (long)H.D < opt_int("max_dim_full")) {
    // Hamiltonian_Dense::build_Q_matrix (src_ed/Hamiltonian/Hamiltonian_Dense.hpp:157-180):
    // all D poles, Q(k, i) = sum_j phi_i[j] U[j, k]
    std::vector<double> U, ph(H.D);
    dense_eigensystem(H, ws, ev, U);
    M = (int)H.D;
    Q.assign((size_t)M * p, 0.0);
    for (int i = 0; i < p; ++i) {
      phi[i].download(ph.data(), H.D, ws.stream);
      ws.sync();
      for (int k = 0; k < M; ++k) {
        const double *uk = U.data() + (size_t)k * H.D;
        double acc = 0.0;
        for (size_t j = 0; j < H.D; ++j) acc += ph[j] * uk[j];
        Q[(size_t)k * p + i] = acc;
      }
    }
    ok = true;
  } else {
    ok = band_lanczos_qmatrix(H, ws, phi, ev, Q, M);
  }
  if (ok && M > 0) {
    out.e = std::move(ev);
    out.V = std::move(Q);
    for (auto &x : out.e) x -= st.energy;
    if (pm == -1)
      for (auto &x : out.e) x = -x;
    streamline(out.e, out.V, p);
  }
}

// The rest of build_qmatrix (src_ed/model_instance.hpp:711-817): append the two
// halves, check_norm, times sqrt(weight), upload for G(z).
void Instance::qmatrix_combine(State &st, bool spin_down, QPart (&parts)[2], Workspace &ws) {
  if (has_group()) {
    qmatrix_combine_mixed(st, spin_down, parts, ws);
    return;
  }
  const int p = model->n_sites;
  QMat &q = st.q[spin_down ? 1 : 0];
  q.L = p;
  q.e = parts[0].e;
  q.e.insert(q.e.end(), parts[1].e.begin(), parts[1].e.end());
  q.V = parts[0].V;
  q.V.insert(q.V.end(), parts[1].V.begin(), parts[1].V.end());
  q.M = (int)q.e.size();
  // check_norm (src_ed/Q_matrix.hpp:236-260), before the weight factor
  double ztot = 0.0;
  for (int i = 0; i < p; ++i) {
    double z = 0.0;
    for (int k = 0; k < q.M; ++k) z += q.V[(size_t)k * p + i] * q.V[(size_t)k * p + i];
    ztot += (z - 1.0) * (z - 1.0);
    for (int j = 0; j < i; ++j) {
      double zz = 0.0;
      for (int k = 0; k < q.M; ++k) zz += q.V[(size_t)k * p + i] * q.V[(size_t)k * p + j];
      ztot += 2.0 * zz * zz;
    }
  }
  if (ztot > opt_double("accur_Q_matrix"))
    fail(QED_ERR_QMATRIX, "Q-matrix does not satisfy unitary condition by " + std::to_string(ztot));
  const double sw = std::sqrt(st.weight);
  for (auto &x : q.V) x *= sw;
  q.de.upload(q.e, ws.stream);
  q.dV.upload(q.V, ws.stream);
  ws.sync();
}

// build_qmatrix for a model with a point group (src_ed/model_instance.hpp:711-817):
// for each irrep r of the symmetric orbitals, the target sector (irrep
// r0 x r for electrons, r0 x conj(r) for holes, shift_sector
// src_ed/symmetry_group.cpp:540-558), the start vectors c^{pm} of the n_r
// orbitals of r on the state (mixed_cdag), band Lanczos on the target's
// symmetry-adapted Hamiltonian (or its full eigensystem below max_dim_full),
// energy shift and sign, streamline in the irrep's orbital basis.
void Instance::qmatrix_part_mixed(State &st, bool spin_down, int s, QPart &out, Workspace &ws) {
  const SymmetryGroup &G = *model->group;
  const int pm = 2 * s - 1;
  const int spin = spin_down ? 1 : 0;
  const int ns = model->n_sites;
  out.e.clear();
  out.V.clear();
  out.segs.clear();
  std::unique_ptr<MixedHamiltonian> Hs;  // the state's own sector, for its basis map
  int off = 0;
  for (int r = 0; r < G.g(); ++r) {
    const int nr = G.site_irrep_dim[r];
    const int r_off = off;
    off += nr;
    if (nr == 0) continue;
    Sector tsec = shift_sector(st.sec, pm, spin);
    const int conj_r = sym_conjugate(G, r);
    tsec.irrep = sym_tensor(G, st.sec.irrep, pm == 1 ? r : conj_r);
    if (!sector_is_valid(tsec, model->n_orb, G.g())) continue;
    auto Ht = mixed_sector(tsec, ws);
    if (Ht->D == 0) continue;
    if (!Hs) Hs = mixed_sector(st.sec, ws);
    std::vector<DevBuf<double>> phi;
    phi.reserve(nr);
    {
      PhaseScope ps_cdag(kPhCdag);
      std::vector<double> coef(ns);
      for (int i = 0; i < nr; ++i) {
        for (int a = 0; a < ns; ++a) coef[a] = G.S[(size_t)(r_off + i) * ns + a].real();
        phi.emplace_back(Ht->D);
        mixed_cdag(*Hs, *Ht, pm, spin, ns, coef.data(), st.psi.p, phi.back().p, ws.stream);
      }
      ws.sync();
    }
    std::vector<double> ev, Q;
    int M = 0;
    bool ok;
    if ((long)Ht->D < opt_int("max_dim_full")) {
      // Hamiltonian_Dense::build_Q_matrix: all D poles, Q(k, i) = <phi_i, u_k>
      std::vector<double> A = Ht->dense(ws.stream), U, ph(Ht->D);
      if (!sym_eig((int)Ht->D, A, ev, &U)) fail(QED_ERR_INTERNAL, "dense eigensolver did not converge");
      M = (int)Ht->D;
      Q.assign((size_t)M * nr, 0.0);
      for (int i = 0; i < nr; ++i) {
        phi[i].download(ph.data(), Ht->D, ws.stream);
        ws.sync();
        for (int k = 0; k < M; ++k) {
          const double *uk = U.data() + (size_t)k * Ht->D;
          double acc = 0.0;
          for (size_t j = 0; j < Ht->D; ++j) acc += ph[j] * uk[j];
          Q[(size_t)k * nr + i] = acc;
        }
      }
      ok = true;
    } else {
      ok = band_lanczos_qmatrix(KrylovOp(*Ht), ws, phi, ev, Q, M);
    }
    if (!ok || M == 0) continue;
    QPart::Seg seg;
    seg.r = r;
    seg.e = std::move(ev);
    seg.V = std::move(Q);
    for (auto &x : seg.e) x -= st.energy;
    if (pm == -1)
      for (auto &x : seg.e) x = -x;
    streamline(seg.e, seg.V, nr);
    out.segs.push_back(std::move(seg));
  }
}

// The rest of build_qmatrix with a point group: per irrep, hole then electron
// poles, check_norm in the irrep's orbital basis, then the consolidated
// Q-matrix in the site basis (Q_matrix_set::consolidated_qmatrix,
// src_ed/Q_matrix_set.hpp:144-163, to_site_basis src_ed/symmetry_group.cpp:487-505:
// site a gets sum over the irrep's orbitals alpha of S(alpha, a) V(alpha)),
// irreps in order, times sqrt(weight).
void Instance::qmatrix_combine_mixed(State &st, bool spin_down, QPart (&parts)[2], Workspace &ws) {
  const SymmetryGroup &G = *model->group;
  const int ns = model->n_sites;
  QMat &q = st.q[spin_down ? 1 : 0];
  q.L = ns;
  q.e.clear();
  q.V.clear();
  int off = 0;
  for (int r = 0; r < G.g(); ++r) {
    const int nr = G.site_irrep_dim[r];
    const int r_off = off;
    off += nr;
    if (nr == 0) continue;
    std::vector<double> e, V;
    for (int s = 0; s < 2; ++s)
      for (const auto &sg : parts[s].segs)
        if (sg.r == r) {
          e.insert(e.end(), sg.e.begin(), sg.e.end());
          V.insert(V.end(), sg.V.begin(), sg.V.end());
        }
    const int M = (int)e.size();
    // check_norm (src_ed/Q_matrix.hpp:236-260) of the irrep's block
    double ztot = 0.0;
    for (int i = 0; i < nr; ++i) {
      double z = 0.0;
      for (int k = 0; k < M; ++k) z += V[(size_t)k * nr + i] * V[(size_t)k * nr + i];
      ztot += (z - 1.0) * (z - 1.0);
      for (int j = 0; j < i; ++j) {
        double zz = 0.0;
        for (int k = 0; k < M; ++k) zz += V[(size_t)k * nr + i] * V[(size_t)k * nr + j];
        ztot += 2.0 * zz * zz;
      }
    }
    if (ztot > opt_double("accur_Q_matrix"))
      fail(QED_ERR_QMATRIX, "Q-matrix does not satisfy unitary condition by " + std::to_string(ztot) +
                                " (irrep " + std::to_string(r) + ")" + where(st.sec));
    for (int k = 0; k < M; ++k) {
      q.e.push_back(e[k]);
      for (int a = 0; a < ns; ++a) {
        double y = 0.0;
        for (int al = 0; al < nr; ++al) y += V[(size_t)k * nr + al] * G.S[(size_t)(r_off + al) * ns + a].real();
        q.V.push_back(y);
      }
    }
  }
  q.M = (int)q.e.size();
  const double sw = std::sqrt(st.weight);
  for (auto &x : q.V) x *= sw;
  q.de.upload(q.e, ws.stream);
  q.dV.upload(q.V, ws.stream);
  ws.sync();
}

void Instance::build_qmatrix(State &st, bool spin_down, Workspace &ws) {
  QPart parts[2];
  for (int s = 0; s < 2; ++s) qmatrix_part(st, spin_down, s, parts[s], ws);
  qmatrix_combine(st, spin_down, parts, ws);
}

// build_cf (src_ed/model_instance.cpp:34-99), real Hilbert space.
void Instance::build_cf(State &st, bool spin_down, Workspace &ws) {
  PhaseScope ps(kPhCf);
  const int n = model->n_sites;
  CFSet &cf = st.cf[spin_down ? 1 : 0];
  cf.n = n;
  cf.ea.assign((size_t)n * n, {});
  cf.eb.assign((size_t)n * n, {});
  cf.ha.assign((size_t)n * n, {});
  cf.hb.assign((size_t)n * n, {});
  for (int pm = -1; pm < 2; pm += 2) {
    Sector tsec = shift_sector(st.sec, pm, spin_down ? 1 : 0);
    if (!sector_is_valid(tsec, model->n_orb)) continue;
    SectorOp H(terms, tsec, ws, &tables);
    if (H.D == 0) continue;
    DevBuf<double> psi(H.D), q(H.D);
    for (int o1 = 0; o1 < n; ++o1)
      for (int o2 = 0; o2 <= o1; ++o2) {
        apply_cdag(st, pm, spin_down ? 1 : 0, o1, H, psi.p, 1.0, false, ws);
        if (o1 != o2) apply_cdag(st, pm, spin_down ? 1 : 0, o2, H, psi.p, 1.0, true, ws);
        VecList one;
        one.n = 1;
        one.v[0] = psi.p;
        int nb = launch_dots(H.D, psi.p, 1.0, 0, one, ws.red, ws.stream);
        const double norm = ws.sums(nb, 1)[0];
        if (norm <= 1e-14) continue;
        launch_scale(H.D, psi.p, 1.0 / std::sqrt(norm), ws.stream);
        std::vector<double> a, b;
        lanczos_green(H, ws, psi.p, q.p, a, b);
        // continued_fraction ctor (src_ed/continued_fraction.cpp:33-39)
        for (auto &x : b) x *= x;
        b[0] = norm * st.weight;
        if (pm == 1)
          for (auto &x : a) x -= st.energy;
        else
          for (auto &x : a) x = -x + st.energy;
        const size_t idx = (size_t)o1 * n + o2;
        if (pm == 1) { cf.ea[idx] = a; cf.eb[idx] = b; }
        else { cf.ha[idx] = a; cf.hb[idx] = b; }
      }
  }
}

// Green_function_solve (src_ed/model_instance.hpp:517-555)
void Instance::build_mcf(State &st, bool spin_down, Workspace &ws) {
  PhaseScope ps(kPhCf);
  const int n = model->n_sites;
  if (n > kMcfMaxP) fail(QED_ERR_UNSUPPORTED, "matrix continued fractions of more than 16 cluster sites");
  McfSet &m = st.mcf[spin_down ? 1 : 0];
  m = McfSet();
  const double accur_def = opt_double("accur_deflation");
  for (int pm = -1; pm < 2; pm += 2) {
    Sector tsec = shift_sector(st.sec, pm, spin_down ? 1 : 0);
    if (!sector_is_valid(tsec, model->n_orb)) continue;
    SectorOp H(terms, tsec, ws, &tables);
    if (H.D == 0) continue;
    // start block phi_i = c_i^{pm} |state>, then its QR phi = q W
    DevBuf<double> phi(H.D * (size_t)n);
    for (int i = 0; i < n; ++i) apply_cdag(st, pm, spin_down ? 1 : 0, i, H, phi.p + (size_t)i * H.D, 1.0, false, ws);
    std::vector<double> R;
    const int pa = mgs_qr(H.D, n, phi.p, accur_def, R, ws);
    if (pa == 0) continue;
    McfFloors f;
    block_lanczos_mcf(KrylovOp(H), ws, phi.p, pa, mcf_qr, f);
    if (f.M == 0) continue;
    McfPart &part = pm == 1 ? m.e : m.h;
    part.M = f.M;
    part.p = pa;
    part.q = n;
    part.A = std::move(f.A);
    part.B = std::move(f.B);
    for (int j = 0; j < part.M; ++j)  // A_j - e0 (electron) or e0 - A_j (hole)
      for (int r = 0; r < pa; ++r)
        for (int c = 0; c < pa; ++c) {
          double &a = part.A[(size_t)j * pa * pa + (size_t)r * pa + c];
          a = pm == 1 ? a - (r == c ? st.energy : 0.0) : -a + (r == c ? st.energy : 0.0);
        }
    const double sw = std::sqrt(st.weight);
    part.W.assign((size_t)pa * n, 0.0);
    for (int r = 0; r < pa; ++r)
      for (int c = 0; c < n; ++c) part.W[(size_t)r * n + c] = R[(size_t)r * n + c] * sw;
  }
}

void Instance::check_gf_solvable() const {
  if (opt_bool("merge_states") && states.size() > 1 && !use_cf && !use_mcf)
    fail(QED_ERR_UNSUPPORTED, "merge_states is not in this solver");
}

void Instance::green_solve(Workspace &ws) {
  if (gf_solved) return;
  if (!gs_solved) low_energy_states(ws);
  check_gf_solvable();
  for (auto &x : states) {
    for (int sd = 0; sd < ((mix & mixing::up_down) ? 2 : 1); ++sd) {
      if (use_cf) build_cf(*x, sd != 0, ws);
      else if (use_mcf) build_mcf(*x, sd != 0, ws);
      else build_qmatrix(*x, sd != 0, ws);
    }
  }
  finish_gf();
}

void Instance::finish_gf() {
  gf_solved = true;
  green_average();
  // Green_function_density (src_ed/model_instance.hpp:657-675)
  const int ns = model->n_sites;
  double nG = 0.0;
  for (int i = 0; i < ns; ++i) nG += Mave[0][i + (size_t)ns * i].real();
  if (mix & mixing::up_down)
    for (int i = 0; i < ns; ++i) nG += Mave[1][i + (size_t)ns * i].real();
  GF_density = nG / ns;
  if (mix == mixing::normal) GF_density *= 2;
}

// Green_function_average (src_ed/model_instance.hpp:643-652): Q-matrix
// integrated_Green_function (src_ed/Q_matrix.hpp:160-172) or the CF version
// (src_ed/continued_fraction_set.cpp:103-125), accumulated over states.
void Instance::green_average() {
  const int n = model->n_sites;
  for (int sd = 0; sd < 2; ++sd) {
    Mave[sd].assign((size_t)n * n, 0.0);
    if (sd == 1 && !(mix & mixing::up_down)) continue;
    for (auto &st : states) {
      if (use_mcf) {  // mcf_set::integrated_Green_function (src_ed/mcf_set.hpp:140-152): (W_h^T W_h)^T
        const McfPart &h = st->mcf[sd].h;
        for (int a = 0; a < n && h.M; ++a)
          for (int b = 0; b < n; ++b) {
            double acc = 0.0;
            for (int k = 0; k < h.p; ++k) acc += h.W[(size_t)k * n + a] * h.W[(size_t)k * n + b];
            Mave[sd][a + (size_t)n * b] += acc;
          }
      } else if (!use_cf) {
        const QMat &q = st->q[sd];
        for (int i = 0; i < q.M; ++i) {
          if (q.e[i] >= 0.0) continue;
          for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) Mave[sd][b + (size_t)n * a] += q.V[(size_t)i * n + a] * q.V[(size_t)i * n + b];
        }
      } else {
        const CFSet &cf = st->cf[sd];
        auto b0 = [&](size_t idx) { return cf.hb[idx].empty() ? 0.0 : cf.hb[idx][0]; };
        for (int o1 = 0; o1 < n; ++o1) Mave[sd][o1 + (size_t)n * o1] += b0((size_t)o1 * n + o1);
        for (int o1 = 0; o1 < n; ++o1)
          for (int o2 = 0; o2 < o1; ++o2) {
            cplx tmp = 0.5 * (b0((size_t)o1 * n + o2) - Mave[sd][o1 + (size_t)n * o1] - Mave[sd][o2 + (size_t)n * o2]);
            Mave[sd][o1 + (size_t)n * o2] += tmp;
            Mave[sd][o2 + (size_t)n * o1] += tmp;
          }
      }
    }
  }
}

// Green_function (src_ed/model_instance.hpp:566-635), batched over frequencies.
void Instance::green_function(const cplx *z, int nz, bool spin_down, cplx *out, Workspace &ws) {
  if (spin_down && !(mix & mixing::up_down || mix == 0))
    fail(QED_ERR_ARGUMENT, "spin_down=True impossible with Hilbert space mixing " + std::to_string(mix));
  if (!gf_solved) green_solve(ws);
  const int n = model->n_sites;
  const int sd = (spin_down && (mix & mixing::up_down)) ? 1 : 0;
  const size_t nn = (size_t)n * n;
  std::fill(out, out + nn * nz, cplx(0.0));
  if (nz <= 0) return;
  DevBuf<double> dz(2 * (size_t)nz);
  dz.upload(reinterpret_cast<const double *>(z), 2 * (size_t)nz, ws.stream);
  if (use_mcf) {  // mcf_set::Green_function (src_ed/mcf_set.hpp:113-131): G_e + G_h^T, every state
    std::vector<McfDesc> desc;
    std::vector<double> blob;
    for (auto &st : states)
      for (int part = 0; part < 2; ++part) {
        const McfPart &f = part ? st->mcf[sd].h : st->mcf[sd].e;
        if (!f.M) continue;
        McfDesc d;
        d.M = f.M;
        d.p = f.p;
        d.q = n;
        d.transpose = part;
        d.offA = (long long)blob.size();
        blob.insert(blob.end(), f.A.begin(), f.A.end());
        d.offB = (long long)blob.size();
        blob.insert(blob.end(), f.B.begin(), f.B.end());
        d.offW = (long long)blob.size();
        blob.insert(blob.end(), f.W.begin(), f.W.end());
        desc.push_back(d);
      }
    const int nf = (int)desc.size();
    if (!nf) return;
    DevBuf<McfDesc> ddesc(nf);
    DevBuf<double> dblob(blob.size()), dF(2 * (size_t)nf * nz * nn);
    ddesc.upload(desc, ws.stream);
    dblob.upload(blob, ws.stream);
    launch_mcf_eval(nf, ddesc.p, dblob.p, n, nz, dz.p, dF.p, ws.stream);
    std::vector<cplx> F((size_t)nf * nz * nn);
    dF.download(reinterpret_cast<double *>(F.data()), 2 * F.size(), ws.stream);
    ws.sync();
    // F[(f * nz + k) * nn + a * n + b] = G_f(z_k)(a, b); out[k * nn + b + a * n] = G(a, b)
    for (int f = 0; f < nf; ++f)
      for (int k = 0; k < nz; ++k)
        for (size_t i = 0; i < nn; ++i) out[nn * k + i] += F[((size_t)f * nz + k) * nn + i];
    return;
  }
  if (!use_cf) {
    DevBuf<double> dG(2 * nn * nz);
    QED_CUDA(cudaMemsetAsync(dG.p, 0, dG.bytes(), ws.stream));
    for (auto &st : states) {
      const QMat &q = st->q[sd];
      launch_qmatrix_gf(n, q.M, q.de.p, q.dV.p, nz, dz.p, dG.p, ws.stream);
    }
    dG.download(reinterpret_cast<double *>(out), 2 * nn * nz, ws.stream);
    ws.sync();
    return;
  }
  // continued fractions: evaluate every fraction of every state on the GPU,
  // then combine per continued_fraction_set::Green_function (src_ed/continued_fraction_set.cpp:63-98)
  for (auto &st : states) {
    const CFSet &cf = st->cf[sd];
    std::vector<int> off, len;
    std::vector<double> A, B;
    auto push = [&](const std::vector<double> &a, const std::vector<double> &b) {
      off.push_back((int)A.size());
      len.push_back((int)a.size());
      A.insert(A.end(), a.begin(), a.end());
      B.insert(B.end(), b.begin(), b.begin() + std::min(a.size(), b.size()));
      if (b.size() < a.size()) B.resize(A.size(), 0.0);
    };
    for (size_t idx = 0; idx < nn; ++idx) {
      push(cf.ea[idx], cf.eb[idx]);
      push(cf.ha[idx], cf.hb[idx]);
    }
    const int nf = (int)off.size();
    DevBuf<int> doff(nf), dlen(nf);
    DevBuf<double> dA(std::max<size_t>(A.size(), 1)), dB(std::max<size_t>(B.size(), 1)), dF(2 * (size_t)nf * nz);
    doff.upload(off, ws.stream);
    dlen.upload(len, ws.stream);
    if (!A.empty()) { dA.upload(A, ws.stream); dB.upload(B, ws.stream); }
    launch_cf_eval(nf, doff.p, dlen.p, dA.p, dB.p, nz, dz.p, dF.p, ws.stream);
    std::vector<cplx> F((size_t)nf * nz);
    dF.download(reinterpret_cast<double *>(F.data()), 2 * (size_t)nf * nz, ws.stream);
    ws.sync();
    for (int k = 0; k < nz; ++k) {
      const cplx *f = F.data() + (size_t)k * nf;
      cplx *G = out + nn * k;
      auto ev = [&](int o1, int o2) { size_t idx = (size_t)o1 * n + o2; return f[2 * idx] + f[2 * idx + 1]; };
      std::vector<cplx> Gt(n);
      for (int o1 = 0; o1 < n; ++o1) {
        Gt[o1] = ev(o1, o1);
        G[o1 + (size_t)n * o1] += Gt[o1];
      }
      for (int o1 = 0; o1 < n; ++o1)
        for (int o2 = 0; o2 < o1; ++o2) {
          cplx tmp = 0.5 * (ev(o1, o2) - Gt[o1] - Gt[o2]);
          G[o1 + (size_t)n * o2] += tmp;
          G[o2 + (size_t)n * o1] += tmp;
        }
    }
  }
}

void Instance::green_function_device(const cplx *z, int nz, bool spin_down, double *dG, Workspace &ws) {
  if (spin_down && !(mix & mixing::up_down || mix == 0))
    fail(QED_ERR_ARGUMENT, "spin_down=True impossible with Hilbert space mixing " + std::to_string(mix));
  if (!gf_solved) green_solve(ws);
  const int n = model->n_sites;
  const int sd = (spin_down && (mix & mixing::up_down)) ? 1 : 0;
  const size_t nn = (size_t)n * n;
  if (nz <= 0) return;
  if (use_cf || use_mcf) {  // continued fractions: evaluated by green_function, then uploaded
    std::vector<cplx> G(nn * nz);
    green_function(z, nz, spin_down, G.data(), ws);
    QED_CUDA(cudaMemcpyAsync(dG, G.data(), G.size() * sizeof(cplx), cudaMemcpyHostToDevice, ws.stream));
    ws.sync();
    return;
  }
  DevBuf<double> dz(2 * (size_t)nz);
  dz.upload(reinterpret_cast<const double *>(z), 2 * (size_t)nz, ws.stream);
  QED_CUDA(cudaMemsetAsync(dG, 0, 2 * nn * nz * sizeof(double), ws.stream));
  for (auto &st : states) {
    const QMat &q = st->q[sd];
    launch_qmatrix_gf(n, q.M, q.de.p, q.dV.p, nz, dz.p, dG, ws.stream);
  }
  ws.sync();
}

// hybridization_function (src_ed/model_instance.hpp:1004-1018)
void Instance::hybridization(const cplx *z, int nz, bool spin_down, cplx *out) {
  const int n = model->n_sites, nb = model->n_bath;
  const int sd = (spin_down && (mix & mixing::up_down)) ? 1 : 0;
  const size_t nn = (size_t)n * n;
  for (int k = 0; k < nz; ++k) {
    cplx *G = out + nn * k;
    std::fill(G, G + nn, cplx(0.0));
    for (int i = 0; i < nb; ++i) {
      cplx w = 1.0 / (z[k] - tb[sd][i + (size_t)nb * i]);
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
          G[a + (size_t)n * b] += tcb[sd][a + (size_t)n * i] * tcb[sd][b + (size_t)n * i] * w;
    }
  }
}

// self_energy (src_ed/model_instance.hpp:683-700): z - t_c - Gamma(z) - G(z)^-1
void Instance::self_energy(const cplx *z, int nz, bool spin_down, cplx *out, Workspace &ws) {
  const int n = model->n_sites;
  const size_t nn = (size_t)n * n;
  const int sd = (spin_down && (mix & mixing::up_down)) ? 1 : 0;
  green_function(z, nz, spin_down, out, ws);
  std::vector<cplx> Gam(nn * std::max(nz, 1));
  if (model->n_bath) hybridization(z, nz, spin_down, Gam.data());
  for (int k = 0; k < nz; ++k) {
    cplx *S = out + nn * k;
    if (!complex_inverse(n, S)) fail(QED_ERR_INTERNAL, "singular Green function in self_energy");
    for (size_t i = 0; i < nn; ++i) {
      S[i] += tc[sd][i];
      if (model->n_bath) S[i] += Gam[nn * k + i];
      S[i] = -S[i];
    }
    for (int a = 0; a < n; ++a) S[a + (size_t)n * a] += z[k];
  }
}

// Potthoff_functional (src_ed/qcm_ED.cpp:330-334)
double Instance::potthoff(Workspace &ws) {
  if (!gf_solved) green_solve(ws);
  return SEF_bath + E0;
}

}  // namespace qed
