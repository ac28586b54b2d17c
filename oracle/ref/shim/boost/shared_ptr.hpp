// std::shared_ptr standing in for boost::shared_ptr (CPU oracle build only).
#ifndef HB_REF_SHIM_BOOST_SHARED_PTR_HPP
#define HB_REF_SHIM_BOOST_SHARED_PTR_HPP
#include <memory>
namespace boost {
template <class T>
using shared_ptr = std::shared_ptr<T>;
}  // namespace boost
#endif
