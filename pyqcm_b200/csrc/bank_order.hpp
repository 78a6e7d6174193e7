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
