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

// The terms a block's summary keeps in the reference (fp32 values): the
// block's docs' rows max-pooled per term in first-touch order (a first value
// clamped at 0; the block mass summed in that order,
// cluster/inverted_list_clusters.cpp:96-114), the (term, value) pairs sorted
// by value descending with std::ranges::sort, and cut where the running sum
// reaches alpha of the mass (:37-51). Which of several equal maxima survive a
// cut between them is whatever that unstable sort leaves.
std::vector<uint16_t> reference_summary_kept(const HostCsr& h, const int32_t* docs, size_t n_docs,
                                             float alpha);

}  // namespace nsp

#endif  // NSP_REF_ORDER_H
