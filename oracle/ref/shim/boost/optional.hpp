// std::optional standing in for boost::optional when HemePure is built as the
// CPU oracle (test infrastructure only; the reference uses *x, bool(x) and assignment).
#ifndef HB_REF_SHIM_BOOST_OPTIONAL_HPP
#define HB_REF_SHIM_BOOST_OPTIONAL_HPP
#include <optional>
#include "std_headers.h"
namespace boost {
template <class T>
using optional = std::optional<T>;
inline constexpr std::nullopt_t none = std::nullopt;
}  // namespace boost
#endif
