// Hop-list ordering of an up-spin table for the row pass's shared-memory
// gathers (host code, used when a table is built).
#pragma once
#include <cstdint>
#include <vector>

namespace qed {

// Orders the hop lists of an up-spin table for the shared-memory gathers of the
// row pass. k_hv_rows2 reads 16-byte words (two dn-rows of x per up string),
// and shared memory serves a 16-byte warp access in four phases of eight lanes:
// lanes u0..u0+7 (u0 a multiple of 8) gather in one phase, conflict-free when
// their targets u' fall in distinct 16-byte bank groups, u' mod 8. Per group of
// eight strings, each step is a maximum matching of lanes to free bank groups
// (Kuhn's augmenting paths, lanes with the most hops left first); a lane
// without a hop in a free group takes a padding entry of value 0 aimed at a
// free group. Every string of the group then has the group's step count as its
// hop count. The sum of each row is unchanged up to the order of its terms.
// ell: width x dim entries (target << 8 | value slot, row k at k * dim),
// cnt: hops per string; both rewritten in place, width updated; zero_slot is
// the value slot holding 0.0. Returns false (tables untouched) if a group
// would need more than 255 steps.
bool order_for_banks(std::vector<uint32_t> &ell, std::vector<uint8_t> &cnt, uint32_t dim, int &width, int zero_slot);

}  // namespace qed

namespace qed {

// Packed hop table for the staged-row H.v kernels (k_hv_rows16, k_hv_cols16).
// Every hop of a string is one 16-bit entry: target (bits 0-13) | sign
// (bit 15); its value is (sign ? -1 : 1) * mag[class]. The hops of each
// magnitude class form their own list, packed four entries per 8-byte word:
// word (k, i) of class c at pk[c][(k * dim + i) * 4 .. + 4). Per group of eight
// strings each class list is bank-ordered (order_for_banks) and padded to a
// multiple of four entries; every string then carries its group's word counts
// cnt[i] = words of class 0 | words of class 1 << 4. Padding entries point at
// one of eight zero slots dim .. dim + 7 placed in the bank group the padded
// lane needs, so they add 0 * 0.
struct PackedHops {
  std::vector<uint16_t> pk[2];  // per class: 4 * width[c] * dim entries
  std::vector<uint8_t> cnt;     // per string: class-0 words | class-1 words << 4
  double mag[2] = {0.0, 0.0};
  int width[2] = {0, 0};        // words per string of each class table
};

// Packs an ELL table (entry k of string i at ell[k * dim + i] = target << 8 |
// value slot, cnt[i] hops; vals: the value of each slot, zero_slot unused here).
// Returns false when the table does not fit the format: dim + 8 > 2^14, more
// than two distinct magnitudes, or more than 15 words of one class per string.
bool pack_hops16(const std::vector<uint32_t> &ell, const std::vector<uint8_t> &cnt, uint32_t dim,
                 const std::vector<double> &vals, int zero_slot, PackedHops &out);

}  // namespace qed
