// Device-resident sector Hamiltonian and the Krylov solvers built on it.
//
// SectorOp is this solver's realisation of the reference's Hamiltonian
// plugin (Hamiltonian<double>, src_ed/Hamiltonian/Hamiltonian_base.hpp:43-82)
// in spin-factorized form (Hamiltonian_Factorized, .../Hamiltonian_Factorized.hpp).
// The Krylov drivers follow src_ed/Hamiltonian/Lanczos.hpp step for step; their
// vector work runs in the kernels of kernels.cu, only the small tridiagonal /
// banded projected problems are solved on the host.
#pragma once
#include <functional>
#include <map>
#include <memory>
#include <vector>

#include "common.hpp"
#include "kernels.cuh"
#include "bank_order.hpp"
#include "model.hpp"
#include "winhv.hpp"

namespace qed {

// Per-process device context: stream, reduction buffers.
struct Workspace {
  cudaStream_t stream = nullptr;
  Reducer red;
  DevBuf<double> partials, out;
  double *host = nullptr;
  double *pin = nullptr;  // pinned host staging, grown on demand
  int *wait_flag = nullptr;  // pinned copy of the staged kernels' wait-timeout flag
  size_t pin_n = 0;
  Workspace();
  ~Workspace();
  // pinned host buffer of at least n doubles (contents not kept on growth)
  double *pinned(size_t n);
  // finalize + wait: returns host pointer with nred sums
  const double *sums(int nblocks, int nred);
  void sync();
};

// One spin species: basis strings and hop table on the device.
struct HalfTables {
  int L = 0, N = 0;
  uint32_t dim = 0;
  DevBuf<uint32_t> bits;
  std::vector<uint32_t> hbits;
  DevBuf<uint8_t> cnt;
  DevBuf<uint32_t> ell;
  DevBuf<double> vals, diag;
  int nvals = 0, width = 0;
  // packed, bank-ordered copy of the hops (empty when the table does not fit it)
  DevBuf<uint16_t> pk[2];
  DevBuf<uint8_t> cntw;
  double mag[2] = {0.0, 0.0};
  // the directed hopping pairs (destination r, source c) and their t[r][c]
  std::vector<int> pd, ps;
  std::vector<double> pv;
};

// The directed hopping pairs of one spin (destination r, source c, scanned row by
// row, skipping the diagonal and |t| below SMALL_VALUE) with their value slots:
// vals holds each distinct amplitude v at an even slot and -v after it.
void hop_pairs(int L, const std::vector<double> &t, std::vector<int> &pd, std::vector<int> &ps,
               std::vector<int> &pslot, std::vector<double> &vals);

// One spin's tables computed on the host: the N-of-L strings in increasing order,
// the ELL hops (entry k of string i at ell[k * dim + i] = rank << 8 | value slot,
// cnt[i] entries, the sign in the slot's parity), the one-body + same-spin
// interaction diagonal, and the bank-ordered (for bank_order, the ELL itself)
// and packed copies (bank_order.hpp). The device build gives the same tables.
struct HostHalf {
  std::vector<uint32_t> bits, ell;
  std::vector<uint8_t> cnt;
  std::vector<double> vals, diag;
  int width = 0;
  PackedHops ph;
  bool packed = false;
};
HostHalf host_half_tables(int L, int N, uint32_t dim, const std::vector<double> &tdiag,
                          const std::vector<double> &vsame, const std::vector<int> &pd, const std::vector<int> &ps,
                          const std::vector<int> &pslot, const std::vector<double> &vals, int width, bool bank_order);

// Per-instance cache of the spin tables: a sector (N_up, N_dn) uses the up
// table of N_up and the down table of N_dn, so the sectors of one instance
// share them. Thread-safe; tables live until the cache is destroyed.
struct HalfCache {
  std::mutex m;
  std::map<std::pair<int, int>, std::shared_ptr<const HalfTables>> tab;  // (spin, N)
};

struct SectorOp {
  Sector sec;
  int L = 0;
  std::shared_ptr<const HalfTables> up, dn;
  DevBuf<double> vinter;
  std::shared_ptr<WinBinding> win;  // window H.v kernels of large sectors (winhv.hpp)
  HvOperator op;
  size_t D = 0;
  // Builds (or takes from `cache`) the tables for `sec` from the collected
  // terms, on `ws.stream`.
  SectorOp(const SpinData &terms, const Sector &sec, Workspace &ws, HalfCache *cache = nullptr);
  // y = H x (device vectors)
  void apply(const double *x, double *y, Workspace &ws) const;
  // Plans the window kernels for this sector and binds them to op (large
  // sectors whose hops fit windows; see hv_windows / hv_windows_min_dim).
  void bind_windows();
};

// Ground state by Lanczos (LanczosEigenvalue + LanczosEigenvector,
// src_ed/Hamiltonian/Lanczos.hpp:41-143), as two passes like the reference:
// lanczos_energy runs the recurrence with the Ritz-residual stop and keeps the
// tridiagonal; lanczos_eigenvector replays it from the same seeded start vector
// and accumulates psi. The instance calls the second pass only for the sectors
// whose state survives the Boltzmann-weight selection.
struct LanczosResult {
  double energy = 0.0;
  int iterations = 0;
  std::vector<double> alpha, beta;
};
LanczosResult lanczos_energy(const SectorOp &H, Workspace &ws, uint64_t seed);
// The eigenvalue pass of many sectors of at most lanczos_job_max_dim() states at
// once: one CTA per sector, all sectors advancing by chunks in one launch, the
// Ritz test of each applied on the host after every chunk. Results are those
// of lanczos_energy, which runs a single small sector through the same path.
struct LanczosBatchItem {
  const SectorOp *H = nullptr;
  uint64_t seed = 0;
  LanczosResult *out = nullptr;
  std::string where;  // appended to error messages
};
void lanczos_energy_batch(std::vector<LanczosBatchItem> &items, Workspace &ws);
// Host-side parallel loop used by lanczos_energy_batch for the per-sector Ritz
// tests (the library's worker pool; a plain loop until one is installed).
using ParallelFor = std::function<void(int n, const std::function<void(int)> &fn)>;
void set_parallel_for(ParallelFor f);
void lanczos_eigenvector(const SectorOp &H, Workspace &ws, const LanczosResult &res,
                         uint64_t seed, DevBuf<double> &psi);
// Both passes.
LanczosResult lanczos_ground_state(const SectorOp &H, Workspace &ws, DevBuf<double> &psi,
                                   uint64_t seed);

// Ground-state energy of a sector in the symmetry-adapted basis (mixed.hpp).
struct MixedHamiltonian;
LanczosResult lanczos_energy_mixed(const MixedHamiltonian &H, Workspace &ws, uint64_t seed);
void lanczos_eigenvector_mixed(const MixedHamiltonian &H, Workspace &ws, const LanczosResult &res, uint64_t seed,
                               DevBuf<double> &psi);

// Full diagonalisation of a small sector (Hamiltonian_Dense::states and
// ::build_Q_matrix, src_ed/Hamiltonian/Hamiltonian_Dense.hpp:110-180): the dense
// matrix is assembled on the device from the sector tables, the D x D symmetric
// eigenproblem is solved on the host. w: eigenvalues ascending; U: column-major
// eigenvectors (column k <-> w[k]) in the H.v vector layout.
void dense_eigensystem(const SectorOp &H, Workspace &ws, std::vector<double> &w,
                       std::vector<double> &U);

// The H.v the Krylov drivers below apply: the spin-factorized sector operator
// or the symmetry-adapted (mixed-basis) CSR Hamiltonian. Built implicitly from
// either. apply: y = xs H x - sum_k sub.c[k] sub.z[k] with the reductions of
// launch_hv (nothing when *skip != 0); apply_block: Y_c = H X_c for p vectors.
struct KrylovOp {
  size_t D = 0;
  const SectorOp *fact = nullptr;
  const MixedHamiltonian *mixed = nullptr;
  KrylovOp(const SectorOp &h) : D(h.D), fact(&h) {}
  KrylovOp(const MixedHamiltonian &h);
  int apply(const double *x, double xs, double *y, const SubList &sub, int red_mask, Reducer &r, cudaStream_t s,
            const int *skip = nullptr) const;
  void apply_block(int p, const BlockIn &X, const BlockOut &Y, Reducer &r, cudaStream_t s) const;
};

// LanczosGreen (src_ed/Hamiltonian/Lanczos.hpp:156-183) from a normalised start
// vector psi (overwritten). Returns the (a, b) coefficients.
void lanczos_green(const KrylovOp &H, Workspace &ws, double *psi, double *q,
                   std::vector<double> &a, std::vector<double> &b);

// Band Lanczos (src_ed/Hamiltonian/Lanczos.hpp:214-395) followed by the
// projected eigensystem; returns false when no iteration was possible.
// phi: p device start vectors of length H.D (consumed). Outputs the eigenvalues
// and the Q-matrix residues Q = P U (p x M, column-major), as
// Hamiltonian::build_Q_matrix does (src_ed/Hamiltonian/Hamiltonian_base.hpp:229-254).
bool band_lanczos_qmatrix(const KrylovOp &H, Workspace &ws, std::vector<DevBuf<double>> &phi,
                          std::vector<double> &evals, std::vector<double> &Q, int &M);

// Modified Gram-Schmidt QR, in place, of the p device vectors X + c * D
// (c < p), as the reference orthonormalises a start block
// (src_ed/model_instance.hpp:888-907): column l loses its projections on the
// columns before it one at a time, then is normalised. Stops at the first
// column whose norm falls below tol and returns its index (p if none); R
// (p x p, row-major, upper triangular) holds the coefficients of the columns
// before it, zeros elsewhere.
int mgs_qr(size_t D, int p, double *X, double tol, std::vector<double> &R, Workspace &ws);

// Floors of a block Lanczos run: M diagonal blocks A_j and off-diagonal blocks
// B_j, p x p row-major each (B_{M-1} is the truncation residual).
struct McfFloors {
  int p = 0, M = 0;
  std::vector<double> A, B;
};

// Block Lanczos for matrix continued fractions from the p orthonormal device
// vectors Q0 + c * D (left unchanged): blockLanczos (qr = true: upper-triangular
// B_j by QR of the residual block) or blockLanczosSVD (qr = false: Hermitian
// B_j = G^(1/2) by the eigensystem of the residual's Gram matrix G), with the
// reference's step count min(14 p ln D, max_iter_BL), its convergence test (the
// lowest eigenvalue of the projected block tridiagonal matrix every p steps from
// step 2p, accur_band_lanczos) and its deflation rules (a QR column or a Gram
// eigenvalue below accur_deflation (squared) ends the run)
// (src_ed/Hamiltonian/Lanczos.hpp:426-571, 597-768). The residual block's QR is
// a Cholesky QR done twice on the device; a Cholesky pivot below 1e-4 sends that
// step through mgs_qr, which then decides a deflation exactly as the reference's
// column-by-column QR does.
void block_lanczos_mcf(const KrylovOp &H, Workspace &ws, const double *Q0, int p, bool qr, McfFloors &out);

}  // namespace qed
