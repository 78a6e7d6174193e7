// Window form of the spin-factorized H.v for large sectors.
//
// The hops of one spin act on N-of-L strings. Cover the lattice's hopping pairs
// (r, c) with windows of at most eight consecutive sites [lo, lo + w) so that
// every pair lies inside one window (its assigned window). A hop inside a window
// leaves the bits outside it unchanged, and its fermion sign, the parity of the
// occupied sites strictly between r and c (binary_state::one_body,
// src_ed/binary_state.cpp:23-28), only reads bits inside it. So for one window
// the strings fall into groups of equal outside bits; a group with k particles
// inside the window has C(w, k) members, and the window's hops map the group
// onto itself with the same C(w, k) x C(w, k) sparse matrix for every group of
// that k (signs included). The per-spin hop operator is the sum over windows of
// these block-diagonal matrices.
//
// The kernels stage one whole row (up hops) or column (down hops) of x in
// shared memory beside an accumulator tile, give each lane one group, load that
// group's members into registers once per window and apply the window's matrix
// for that k as generated straight-line FMAs (amplitudes from the kernel's
// constant bank): one shared-memory load per state and window instead of one
// per hop. The code depends on the lattice (pairs, L, N) and is compiled at run
// time with NVRTC for sm_100a, once per structure and process.
//
// Opt-in (option hv_windows, off by default). On a B200 these kernels are
// slower than the staged ones: 10.9 ms against 4.6 ms per H.v on the 4x4 sector.
// Holding a group in registers takes up to 255 registers per thread, so only
// eight warps fit on an SM, and the kernels are latency-bound. The down-spin
// pass also copies and stores its columns 8 bytes at a time.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace qed {

constexpr int kWinMaxSites = 8;       // sites per window
constexpr int kWinMaxWindows = 4;     // windows per spin
constexpr int kWinWarps = 8;          // warps per CTA of the window kernels
constexpr int kWinMaxPairs = 256;     // directed hopping pairs per spin (constant-bank amplitudes)
constexpr uint32_t kWinMaxDim = 14300;  // strings per spin: x and accumulator tiles in 227 KB
constexpr uint32_t kWinPadLane = 0xFFFFFFFFu;  // lane constant of a padding lane
constexpr size_t kWinMaxUniform = 7000;         // uniform offsets per spin (constant memory)

// One spin's window plan: the windows, the lane tables and the warp schedule.
struct WindowPlan {
  int L = 0, N = 0;
  uint32_t dim = 0;
  struct Window {
    int lo = 0, w = 0;
    std::vector<int> pairs;  // indices into the spin's pair list, increasing
  };
  std::vector<Window> win;
  std::vector<int> pd, ps;  // the pair list (destination r, source c)
  // Per window, groups come in blocks of 32 with the same (k, nB): k particles
  // inside the window, nB below it. The tile byte offset of member j of a group
  // is tab[base + lane] + cu[ub + j]: a per-group constant (the rank terms of
  // the bits outside the window; kWinPadLane for padding lanes) plus a part
  // uniform over the block (the rank terms of the window's bits). sched:
  // kWinWarps + 1 entry starts per window, then (k, ub, base) triples, each
  // warp's list in turn.
  std::vector<uint32_t> tab, cu;
  std::vector<int> sched;
  int tile_stride = 0;  // doubles from the x tile to the accumulator tile
};

// Plans the windows of one spin; false when the pairs do not fit windows of
// kWinMaxSites sites, need more than kWinMaxWindows windows, or dim is too large.
// bits: the spin's strings in basis order (ascending).
bool plan_windows(int L, int N, const std::vector<uint32_t> &bits, const std::vector<int> &pd,
                  const std::vector<int> &ps, WindowPlan &plan);

// y = (sum over windows of the block matrices) x with amplitudes amp[q] of pair q,
// on the host (the planner's check).
void window_apply_host(const WindowPlan &plan, const std::vector<double> &amp, const double *x, double *y);

// CUDA C++ source of the two window kernels for the (up, dn) plans.
std::string window_source(const WindowPlan &up, const WindowPlan &dn);

// Compiled module and device tables for one (up, dn) structure.
struct WinModule;

// The window binding of a sector operator: module plus this instance's amplitudes.
struct WinBinding {
  std::shared_ptr<const WinModule> mod;
  std::vector<double> amp_up, amp_dn;  // t[r][c] of each pair
};

// The module for (up, dn), compiled on first use and cached by structure; null
// (with the reason in *why) when NVRTC is unavailable or compilation fails.
std::shared_ptr<const WinModule> window_module(const WindowPlan &up, const WindowPlan &dn, std::string *why);

// NVRTC's log of compiling the window source for (up, dn) with ptxas
// diagnostics (registers, spills); empty string on success without a log.
std::string window_compile_log(const WindowPlan &up, const WindowPlan &dn, bool *ok);

// Whether the window kernels can take this call (aligned vectors, no term of the
// subtraction aliasing y).
bool window_usable(const HvOperator &op, const double *x, const double *y, const SubList &sub);

// y = xs H x - sum_k sub.c[k] sub.z[k] (+ the reductions of launch_hv) through
// the window kernels; returns the number of reduction blocks written.
int launch_hv_windows(const HvOperator &op, const double *x, double xs, double *y, const SubList &sub,
                      int red_mask, Reducer &r, cudaStream_t s);

// Window H.v calls so far in this process.
long long window_launches();

}  // namespace qed
