// Launch wrappers of the sm_100a kernels of the ED solver. Host C++ code calls
// these; every wrapper enqueues on the given stream and checks the launch.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

namespace qed {

constexpr int kMaxVec = 64;  // vectors per multi-vector kernel call

// Device view of one spin species' basis and hopping table (ELL layout):
//   bits[i]            i-th N-of-L string in ascending order (ED_halfbasis::bin)
//   cnt[i]             number of hops out of string i
//   ell[k*dim + i]     (target index << 8) | value slot   for k < cnt[i]
//   vals[slot]         signed hopping amplitude (sign of the fermion phase folded in)
//   diag[i]            one-body diagonal + same-spin density-density terms of string i
struct SpinTable {
  const uint32_t *bits = nullptr;
  const uint8_t *cnt = nullptr;
  const uint32_t *ell = nullptr;
  const double *vals = nullptr;
  const double *diag = nullptr;
  uint32_t dim = 0;
  int nvals = 0;
  // Packed form of the same hops for the staged-row kernels (null when the
  // table does not fit it; see PackedHops in bank_order.hpp): one list per
  // magnitude class, four 16-bit entries (target | sign << 15) per word, word
  // (k, i) of class c at pk[c][k * dim + i]; cntw[i] = class-0 words | class-1
  // words << 4; the value of an entry is +-mag[c].
  const uint2 *pk[2] = {nullptr, nullptr};
  const uint8_t *cntw = nullptr;
  double mag[2] = {0.0, 0.0};
};

// Inter-spin density-density terms sum_{r,s} v[r][s] dn_r up_s.
//   mode 0: none; 1: diagonal and uniform (u * popc(up & dn));
//   mode 2: diagonal per site (vdiag[r]); 3: general n x n (vfull, row r = dn bit).
struct InterSpin {
  int mode = 0;
  int n = 0;
  double u = 0.0;
  const double *v = nullptr;  // device: n (mode 2) or n*n (mode 3)
};

struct HvOperator {
  SpinTable up, dn;
  InterSpin inter;
  int num_sms = 148;
  const int *skip = nullptr;  // if set and *skip != 0 (device), the H.v passes do nothing
  // host-side binding of the window kernels (WinBinding, winhv.hpp), null when
  // the sector does not use them; device code never reads it
  const void *win = nullptr;
};

// List of (coefficient, vector) pairs subtracted in the row pass epilogue:
// y -= sum_k c[k] * z[k].
struct SubList {
  int n = 0;
  double c[32];
  const double *z[32];
  const double *cdev = nullptr;  // if set, the coefficients are read from device memory cdev[k]
};

// Deterministic two-stage reductions: kernels write per-block partial sums,
// finalize_sums adds them in a fixed order into out[0..nred).
struct Reducer {
  double *partials = nullptr;  // [max_blocks * kMaxRed]
  double *out = nullptr;       // [kMaxRed] device
  double *host = nullptr;      // [kMaxRed] pinned
  int max_blocks = 0;
  static constexpr int kMaxRed = 72;
};

// ---- basis -----------------------------------------------------------------
void launch_unrank(int L, int N, uint32_t dim, uint32_t *out, cudaStream_t s);
void launch_rank(int L, int N, size_t n, const uint32_t *strings, uint32_t *ranks, cudaStream_t s);
// Builds the ELL hop table of one spin species on the device. pairs: directed
// (dst, src) orbital pairs with the value slot of the + sign (slot ^ 1 holds -t).
void launch_build_hops(int L, int N, uint32_t dim, const uint32_t *bits, int npairs,
                       const int *pair_dst, const int *pair_src, const int *pair_slot,
                       uint8_t *cnt, uint32_t *ell, int width, cudaStream_t s);
void launch_diag_half(int L, uint32_t dim, const uint32_t *bits, const double *tdiag,
                      const double *vsame, double *diag, cudaStream_t s);
// c_a / c^+_a gathered onto the target sector (Destroy, src_ed/ED_basis.cpp:79-110)
void launch_cdag_gather(int L, int spin, int a, int pm, const uint32_t *tgt_up_bits,
                        uint32_t du_t, const uint32_t *tgt_dn_bits, uint32_t dd_t, int src_nup,
                        int src_ndn, uint32_t du_s, const double *psi, double *y, double coef,
                        int accumulate, cudaStream_t s);

// Dense D x D matrix of the sector Hamiltonian (row I = up + du*dn, the H.v
// vector layout), for the full-diagonalisation path of small sectors
// (Hamiltonian_Dense, src_ed/Hamiltonian/Hamiltonian_Dense.hpp:60-88). h must
// hold D*D doubles; it is overwritten.
void launch_dense_hamiltonian(const HvOperator &op, double *h, cudaStream_t s);

// ---- device-resident Lanczos step ------------------------------------------
// Scalars of a ground-state Lanczos run kept in device memory, so that a chunk
// of iterations runs without host round trips (LanczosEigenvalue,
// src_ed/Hamiltonian/Lanczos.hpp:41-97, one step = w = H v_j - beta_{j-1} v_{j-1};
// alpha_j = <v_j, w>; w -= alpha_j v_j; beta_j = |w|; v_{j+1} = w / beta_j).
struct LanczosScalars {
  double *alpha_cur = nullptr;   // alpha_j (finalised <v_j, w>)
  double *b2_cur = nullptr;      // |w - alpha_j v_j|^2
  double *beta_prev = nullptr;   // beta_j, read by the next row pass as its subtraction coefficient
  double *alpha_hist = nullptr;  // alpha_j, beta_j appended at index *j
  double *beta_hist = nullptr;
  int *j = nullptr;
};
// y -= (*a_dev) x, with |y|^2 block partials in r.partials; returns the grid size.
int launch_axpy_dev(size_t D, double *y, const double *x, const double *a_dev, Reducer &r, cudaStream_t s,
                    const int *skip = nullptr);
// y *= 1 / sqrt(*b2_cur) (0 if that is 0); records alpha_j, beta_j and advances *j.
void launch_lanczos_advance(size_t D, double *y, const LanczosScalars &ls, cudaStream_t s);
// Largest sector the one-CTA-per-sector job table takes (the option
// lanczos_job_max_dim, at most kLanczosCtaMaxDimCap; larger sectors run the
// whole-GPU kernels step by step). Read once per solve step: the eigenvalue and
// the eigenvector pass of a state must see the same value.
constexpr size_t kLanczosCtaMaxDimCap = 1u << 20;
size_t lanczos_job_max_dim();

// Ground-state Lanczos of many small sectors in one launch, one CTA of kLanczosJobThreads threads per
// sector (dimension at most lanczos_job_max_dim()): the ground-state Lanczos
// chunks of a whole batch of sectors advance together. Buffer roles of a job:
// v_{j-1} = v[rot], v_j = v[(rot + 1) % 3], scratch = v[(rot + 2) % 3]; they
// rotate once per step. out receives alpha then beta of the launch's steps
// (2 * kLanczosJobMaxSteps doubles per job).
constexpr int kLanczosJobThreads = 256;
constexpr int kLanczosJobMaxSteps = 16;
struct LanczosJob {
  HvOperator op;
  double *v[3];
  double *beta_prev;  // beta_{j-1} (0 before the first step)
  double *out;
  unsigned long long seed;
  int nsteps, rot;
};
// v_j = normalised random start vector (the values of launch_random for `seed`),
// v_{j-1} = 0, beta_prev = 0, for every job
void launch_lanczos_start_jobs(const LanczosJob *jobs, int njobs, cudaStream_t s);
void launch_lanczos_jobs(const LanczosJob *jobs, int njobs, cudaStream_t s);

// ---- blocks of p separate vectors (block.cu) ---------------------------------
struct BlockIn {
  const double *v[16] = {};
};
struct BlockOut {
  double *v[16] = {};
};
// Y = a Y + s1 X1 M1 (M1 p x p row-major, device; skipped when X1.v[0] is null;
// Y is not read when a == 0); gram 1: per-CTA partials of Y^T Y of the result,
// gram 2: of L^T Y; partials[b * p * p + i * p + c]. Returns the CTA count.
int launch_bl_update(size_t D, int p, double a, const BlockOut &Y, double s1, const BlockIn &X1, const double *M1,
                     int gram, const BlockIn &L, double *partials, int max_blocks, cudaStream_t s);
// Y_c = H X_c for the p vectors of a block: the staged single-vector H.v per
// vector when the sector has packed tables, else one row and one column launch
// for the whole block (ELL tables, every entry read once per state for all p).
void launch_block_hv(const HvOperator &op, int p, const BlockIn &X, const BlockOut &Y, Reducer &r, cudaStream_t s);

// out[0..n) = fixed-order sums of partials with row stride ld
void launch_finalize_ld(const double *partials, int nblocks, int ld, int n, double *out, cudaStream_t s);
// log |det(V(k) G(iw) - 1)| on the (w, k) grid, V(k) = V0 + sum_e v_e exp(2 pi i k.R_e)
// at (r_e, c_e); G: nw column-major n x n complex matrices. Writes, per w, the
// per-CTA sums partials[w * nblk + b] and returns nblk (n <= 16).
int launch_sef_logdet(int n, int nw, const double *G, const double *V0, int nel, const int *er, const int *ec,
                      const double *eR, const double *ev, int nkx, int nky, int nkz, double *partials,
                      cudaStream_t s);
// Grid average of G (1 - V(k) G)^{-1} per frequency into Gproj (nw n x n
// complex, column-major); V0 holds nw k-independent parts of V (one per
// frequency); k = ((a + off)/nkx, ...). partials: cpt_partials_size(n, nw) doubles.
void launch_cpt_projected(int n, int nw, const double *G, const double *V0, int nel, const int *er, const int *ec,
                          const double *eR, const double *ev, int nkx, int nky, int nkz, double off,
                          double *partials, double *Gproj, cudaStream_t s);
int cpt_partials_size(int n, int nw);
// G = R^T R on the device (p <= 16): R, R^{-1}; *fail = 1 if G is not positive
// definite or a pivot is below pivot_min; with Rprev, B = R Rprev and B^T
void launch_block_chol(int p, const double *G, double pivot_min, double *R, double *Rinv, const double *Rprev,
                       double *B_out, double *Bt_out, double *fail_flag, cudaStream_t s);

// ---- H.v ------------------------------------------------------------------
// Row pass: y = (diag + up hops) x - sum_k sub.c[k] sub.z[k]   (x scaled by xs)
void launch_hv_rows(const HvOperator &op, const double *x, double xs, double *y,
                    const SubList &sub, cudaStream_t s);
// Column pass: y += xs * (dn hops) x ; optional reductions into red slots:
//   red_mask bit0: sum x*y, bit1: sum y*y, bit2: sum x*x   (post-update y)
int launch_hv_cols(const HvOperator &op, const double *x, double xs, double *y, int red_mask,
                    Reducer &r, cudaStream_t s);
// y += xs * (down-spin hops) x for output rows [r0, r1) only (x: every row)
void launch_hv_cols_rows(const HvOperator &op, const double *x, double xs, double *y, uint32_t r0, uint32_t r1,
                         cudaStream_t s);

// Whole H.v with the column pass's reductions: y = xs H x - sum_k sub.c[k]
// sub.z[k], reductions of the final y as launch_hv_cols; returns the block count
// of the reducing launch. Takes the staged-row kernels when the tables are
// packed (down pass first, writing y; then the row pass adding to it), else the
// row pass and the column pass above.
int launch_hv(const HvOperator &op, const double *x, double xs, double *y, const SubList &sub, int red_mask,
              Reducer &r, cudaStream_t s);
// JSON list of the staged H.v launch shapes chosen so far, with the timings
// that chose them (one entry per (dim_up, dim_dn)).
std::string hv_tuning_report();

// ---- vector kernels -------------------------------------------------------
struct VecList {
  int n = 0;
  double *v[kMaxVec];
  double c[kMaxVec];
  const double *cdev = nullptr;   // multi_axpy: coefficients from device memory
  const double *xsdev = nullptr;  // dots: scale of x from device memory
  const int *skip = nullptr;      // if set and *skip != 0 (device), the kernel does nothing
};
// out[i] = sum (xs*x) . y_i  (y_i = list.v[i]); if write_x, x *= xs in place.
int launch_dots(size_t D, double *x, double xs, int write_x, const VecList &ys, Reducer &r,
                 cudaStream_t s);
// y_i -= c_i * (xs*x); if norm_first, out[0] = |y_0|^2 after the update.
int launch_multi_axpy(size_t D, const double *x, double xs, const VecList &ys, int norm_first,
                       Reducer &r, cudaStream_t s);
// y = a*y + b*x ; optional out[0] = |y|^2 (post)
int launch_axpby(size_t D, double a, double *y, double b, const double *x, int norm, Reducer &r,
                  cudaStream_t s);
// LanczosGreen swap: p <- q/beta ; q <- -beta p_old   (src_util/vector_num.hpp:274-282)
void launch_swap_scale(size_t D, double *q, double *p, double beta, cudaStream_t s);
// y = seeded normal random entries (counter-based), out[0] = |y|^2
int launch_random(size_t D, uint64_t seed, double *y, Reducer &r, cudaStream_t s);
void launch_scale(size_t D, double *y, double a, cudaStream_t s);
// y *= *a_dev unless *skip
void launch_scale_dev(size_t D, double *y, const double *a_dev, const int *skip, cudaStream_t s);
// Norm step of a device-resident band-Lanczos step (see k_finalize_norm).
void launch_finalize_norm(const double *partials, int nblocks, double dtol, double *z_out, double *inv_out,
                          int *flag, int step, cudaStream_t s);
// Reduction kernels return their block count; finalize_sums adds the per-block
// partials of `nred` slots in a fixed order into r.out and copies them to
// r.host (the caller synchronises the stream before reading r.host).
void finalize_sums(Reducer &r, int nblocks, int nred, cudaStream_t s);
// Adds per-block partials (stride Reducer::kMaxRed) of `nred` slots into the
// device array out[0..nred), on stream s; nothing is copied to the host.
void launch_finalize(const double *partials, int nblocks, int nred, double *out, cudaStream_t s);
// The staged H.v kernels' bounded waits on their TMA transfers set a sticky
// device flag when they give up. staged_kernels_used(): any staged launch so
// far; read_wait_flag_async enqueues a copy of the flag to (pinned) host
// memory on s; check_wait_flag raises Error(QED_ERR_CUDA) if it was set.
bool staged_kernels_used();
void read_wait_flag_async(int *host_flag, cudaStream_t s);
void check_wait_flag(int flag);
// Number of per-block partial-sum rows a reducing H.v column pass can use.
constexpr int kHvColsMaxBlocks = 8 * 148;

// y = H x with dots = (<x,y>, <y,y>, <x,x>) written to device memory, using
// no memory allocated by anyone: the per-block partial sums go to a fixed
// file-scope device array of kHvColsMaxBlocks rows (see kernels.cu). The first
// call on a device looks up that array's device address (cudaGetSymbolAddress).
// Throws Error(QED_ERR_MEMORY) when the column pass would need more rows.
void launch_hv_dots_noalloc(const HvOperator &op, const double *x, double *y, double *dots,
                            cudaStream_t s);

// ---- Green functions on a frequency grid ----------------------------------
// G[k][b + a*L] += sum_i V[a + i*L] V[b + i*L] / (z_k - e_i)   (real V, L <= 64)
void launch_qmatrix_gf(int L, int M, const double *e, const double *V, int nz, const double *z,
                       double *G, cudaStream_t s);
// Continued fractions: F[k][f] = b_f[0] / (z_k - a_f[0] - b_f[1] / (z_k - ...)), for nf
// fractions with offsets off[f] into a/b and lengths len[f].
void launch_cf_eval(int nf, const int *off, const int *len, const double *a, const double *b,
                    int nz, const double *z, double *F, cudaStream_t s);
// Matrix continued fractions (matrix_continued_fraction::evaluate,
// src_ed/matrix_continued_fraction.hpp:137-187): for fraction f with M floors of
// p x p blocks (A_j, B_j row-major at blob + offA / offB + j p^2) and weight W
// (p x q row-major at blob + offW), G_f(z) = W^T F_0 W with F_M = 0 and
// F_j = (z - A_j - B_j^T F_{j+1} B_j)^{-1}. out[((f * nz + k) * q + a) * q + b]
// = G_f(z_k)(a, b), or G_f(z_k)(b, a) when transpose is set. p <= 16, q <= 32.
struct McfDesc {
  int M = 0, p = 0, q = 0, transpose = 0;
  long long offA = 0, offB = 0, offW = 0;
};
constexpr int kMcfMaxP = 16;
void launch_mcf_eval(int nf, const McfDesc *desc, const double *blob, int q, int nz, const double *z, double *out,
                     cudaStream_t s);

}  // namespace qed
