// Abelian cluster point group acting on basis states: the group tables as a
// plain struct that the host fills once and kernels read by value, and the
// per-state maps (group element on a state, orbit representative) as inline
// functions compiled for both the host and sm_100a.
//
// Restates the reference's symmetry_group (src_ed/symmetry_group.hpp:38-92,
// src_ed/symmetry_group.cpp): each element is a "signed permutation" of the
// orbitals. The first L orbitals (the cluster sites when bath_irrep is set,
// every orbital otherwise) are permuted; each remaining (bath) orbital stays in
// place and multiplies the state by a phase exp(i pi q / g) with q = 2 v[i]
// when it is occupied. Phases are integers in units of pi/g, taken mod 2g, so
// that the fermion sign -1 is q = g even for odd g.
//
// Basis states are 64-bit words, spin up in the low word (orbital i -> bit i),
// spin down in the high word (orbital i -> bit i + 32), as binary_state of the
// reference's mixed basis (src_ed/binary_state.hpp:26-35,
// src_ed/ED_basis.cpp:185-385).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define QED_HD __host__ __device__ __forceinline__
#else
#define QED_HD inline
#endif

namespace qed {

constexpr int kMaxGroup = 16;     // at most 4 commuting generators of order 2, or e.g. C4 x C2 x C2
constexpr int kMaxSymOrb = 32;    // orbitals per spin (the state word is 2 x 32 bits)

struct SymGroup {
  int N;                                // orbitals per spin (sites + bath)
  int L;                                // orbitals permuted by the elements
  int g;                                // group order
  uint8_t perm[kMaxGroup][kMaxSymOrb];  // element e: orbital i < L -> perm[e][i]; i >= L: the bath value v
  int8_t phi[kMaxGroup][kMaxGroup];     // character phase of (element, irrep) in units of 2 pi / g
};

struct RepMap {
  uint64_t rep;  // smallest state of the orbit
  int phase;     // units of pi / g: rep = exp(i pi phase / g) x (element applied to the state)
  int length;    // orbit length g / h, 0 when the projected state vanishes
};

QED_HD int sym_popc(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __popc(x);
#else
  return __builtin_popcount(x);
#endif
}

// One spin's 32-bit string under element e: the permuted string and the phase
// (fermion sign of reordering the permuted sites, plus the bath phases), as
// symmetry_group::apply(v, b) (src_ed/symmetry_group.cpp:118-150).
QED_HD uint32_t sym_apply_half(const SymGroup &G, int e, uint32_t b, int &phase) {
  uint32_t out = 0;
  int inv = 0;
  uint32_t seen = 0;  // permuted positions of the occupied sites visited so far
  for (int i = 0; i < G.L; ++i) {
    if (!((b >> i) & 1u)) continue;
    const int t = G.perm[e][i];
    out |= 1u << t;
    // sites visited earlier that landed above t: one transposition each
    inv += sym_popc(seen >> t);
    seen |= 1u << t;
  }
  for (int i = G.L; i < G.N; ++i) {
    if ((b >> i) & 1u) {
      out |= 1u << i;
      phase += 2 * G.perm[e][i];
    }
  }
  if (inv & 1) phase += G.g;
  return out;
}

// The whole state under element e, projected on irrep r: the spin-up and
// spin-down words transform separately, and the character of (e, r) adds
// 2 phi(e, r) (symmetry_group::apply(elem, irrep, b),
// src_ed/symmetry_group.cpp:197-215).
QED_HD uint64_t sym_apply(const SymGroup &G, int e, int r, uint64_t b, int &phase) {
  int ph = 0;
  const uint32_t up = sym_apply_half(G, e, (uint32_t)b, ph);
  const uint32_t dn = sym_apply_half(G, e, (uint32_t)(b >> 32), ph);
  ph += 2 * G.phi[e][r];
  phase = ph % (2 * G.g);
  return (uint64_t)up | ((uint64_t)dn << 32);
}

// Representative of the orbit of b in irrep r: the smallest image over the
// group (the first element reaching it gives the phase), and the orbit length
// g / h with h the stabiliser's order. The state is null (length 0) when a
// stabiliser element carries a phase q != 0 that divides 2g: the rule of
// symmetry_group::Representative (src_ed/symmetry_group.cpp:231-262), exact
// for real characters (q = g); for complex characters the reference's rule
// keeps some states whose projection vanishes, and this keeps them too.
QED_HD RepMap sym_representative(const SymGroup &G, uint64_t b, int r) {
  RepMap m{b, 0, 0};
  int h = 1;
  for (int e = 1; e < G.g; ++e) {
    int q;
    const uint64_t x = sym_apply(G, e, r, b, q);
    if (x == b) {
      ++h;
      if (q != 0 && (2 * G.g) % q == 0) return RepMap{b, 0, 0};
    }
    if (x < m.rep) {
      m.rep = x;
      m.phase = q;
    }
  }
  m.length = G.g / h;
  return m;
}

}  // namespace qed
