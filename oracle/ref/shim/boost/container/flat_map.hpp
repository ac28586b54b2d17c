// Ordered std::map / std::multimap standing in for boost::container's flat maps
// (CPU oracle build only; iteration order is the same: sorted by key).
#ifndef HB_REF_SHIM_BOOST_FLAT_MAP_HPP
#define HB_REF_SHIM_BOOST_FLAT_MAP_HPP
#include <map>
namespace boost {
namespace container {
template <class Key, class T, class Compare = std::less<Key>, class Alloc = void>
using flat_map = std::map<Key, T, Compare>;
template <class Key, class T, class Compare = std::less<Key>, class Alloc = void>
using flat_multimap = std::multimap<Key, T, Compare>;
}  // namespace container
}  // namespace boost
#endif
