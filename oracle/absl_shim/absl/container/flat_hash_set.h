// Test infrastructure only: lets the reference's sources compile without
// Abseil, which is absent from this image. The reference uses flat_hash_set for
// membership tests and unordered enumeration that it sorts before use, so a
// standard unordered_set gives it the same observable behaviour.
#ifndef NSP_ORACLE_ABSL_FLAT_HASH_SET_SHIM_H
#define NSP_ORACLE_ABSL_FLAT_HASH_SET_SHIM_H
#include <algorithm>
#include <functional>
#include <unordered_set>
namespace absl {
template <class T, class Hash = std::hash<T>, class Eq = std::equal_to<T>>
using flat_hash_set = std::unordered_set<T, Hash, Eq>;
}  // namespace absl
#endif
