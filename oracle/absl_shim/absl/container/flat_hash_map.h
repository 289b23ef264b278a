// Test infrastructure only: lets the reference's sources compile without
// Abseil. The reference uses flat_hash_map only as a key -> value lookup, so a
// standard unordered_map gives it the same observable behaviour.
#ifndef NSP_ORACLE_ABSL_FLAT_HASH_MAP_SHIM_H
#define NSP_ORACLE_ABSL_FLAT_HASH_MAP_SHIM_H
#include <algorithm>
#include <functional>
#include <unordered_map>
namespace absl {
template <class K, class V, class Hash = std::hash<K>, class Eq = std::equal_to<K>>
using flat_hash_map = std::unordered_map<K, V, Hash, Eq>;
}  // namespace absl
#endif
