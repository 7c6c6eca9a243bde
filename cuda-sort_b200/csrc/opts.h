// Launch options passed from the C ABI to the packed sort kernels.
#pragma once

namespace b200s {

// B200S_SORTED_CHECK: test each tile before sorting (and, in the transposed
// network, after every stage of span >= 16) and skip the rest of the network
// once it is in order, as the reference's Sorted switch does.
constexpr unsigned kOptSortedCheck = 1u;

}  // namespace b200s
