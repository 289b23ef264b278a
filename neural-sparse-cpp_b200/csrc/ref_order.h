// Host steps of the SEISMIC build that are defined by a C++ standard library
// call of the reference, so the engine makes the same call (same library).
#ifndef NSP_REF_ORDER_H
#define NSP_REF_ORDER_H

#include <cstdint>
#include <vector>

#include "engine.h"

namespace nsp {

// For each posting list in `lists` (terms, ascending) longer than `cap`: the
// doc ids the reference keeps, in its order -- the first `cap` of
// std::ranges::sort over the list's (value, doc) pairs, built in doc order,
// by value descending (invlists/inverted_lists.cpp:110-132). fp32 values.
// out[j * cap + i] is the i-th kept doc of lists[j].
void reference_kept_order(const HostCsr& h, const std::vector<int64_t>& post,
                          const std::vector<int32_t>& lists, int64_t cap,
                          std::vector<int32_t>& out);

}  // namespace nsp

#endif  // NSP_REF_ORDER_H
