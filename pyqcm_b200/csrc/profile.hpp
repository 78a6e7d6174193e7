// Host-side phase timers of the solver. With the environment variable
// QED_PROFILE set, the accumulated wall time of each phase (summed over all
// host threads) is printed to stderr when the library unloads.
#pragma once
#include <chrono>

namespace qed {

enum Phase {
  kPhSectorSetup,   // per-sector tables (SectorOp)
  kPhGsLanczos,     // ground-state Lanczos, eigenvalue pass
  kPhGsVector,      // ground-state Lanczos, eigenvector pass
  kPhDense,         // full diagonalisation of small sectors
  kPhCdag,          // c / c^+ start vectors
  kPhBandLoop,      // band Lanczos recurrence (device work + syncs)
  kPhBandCheck,     // band Lanczos convergence checks (host eigenvalues)
  kPhBandEig,       // projected eigensystem and Q = P U
  kPhCf,            // continued-fraction Lanczos
  kPhRitz,          // ground-state Lanczos: host Ritz tests (inside kPhGsLanczos)
  kPhBlockLoop,     // block form of the band-Lanczos recurrence
  kPhBlockFallback, // block recurrence abandoned for the band one (count)
  kPhAverages,      // operator averages of the ground state (cluster_averages)
  kPhGsBatch,       // batched eigenvalue pass of small sectors (inside kPhGsLanczos)
  kPhCount
};

bool profiling();
void profile_add(Phase p, double seconds);

struct PhaseScope {
  Phase ph;
  bool on;
  std::chrono::steady_clock::time_point t0;
  explicit PhaseScope(Phase p) : ph(p), on(profiling()) {
    if (on) t0 = std::chrono::steady_clock::now();
  }
  ~PhaseScope() {
    if (on) profile_add(ph, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  }
};

}  // namespace qed
