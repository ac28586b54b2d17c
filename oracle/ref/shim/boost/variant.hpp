// A boost::variant over std::variant (CPU oracle build only).  HemePure uses
// the member apply_visitor (re-exported by a class deriving from the variant),
// the free boost::apply_visitor(visitor, visitable), converting construction
// and assignment, and default construction to the first alternative.
#ifndef HB_REF_SHIM_BOOST_VARIANT_HPP
#define HB_REF_SHIM_BOOST_VARIANT_HPP
#include <type_traits>
#include "std_headers.h"
#include <utility>
#include <variant>
namespace boost {
template <class R = void>
struct static_visitor {
  typedef R result_type;
};

template <class... Ts>
class variant {
 public:
  variant() = default;
  variant(const variant&) = default;
  variant(variant&&) = default;
  variant& operator=(const variant&) = default;
  variant& operator=(variant&&) = default;
  template <class T, class = std::enable_if_t<!std::is_base_of<variant, std::decay_t<T>>::value>>
  variant(T&& t) : v_(std::forward<T>(t)) {}
  template <class T, class = std::enable_if_t<!std::is_base_of<variant, std::decay_t<T>>::value>>
  variant& operator=(T&& t) {
    v_ = std::forward<T>(t);
    return *this;
  }
  template <class V>
  decltype(auto) apply_visitor(const V& vis) const {
    return std::visit(vis, v_);
  }
  template <class V>
  decltype(auto) apply_visitor(const V& vis) {
    return std::visit(vis, v_);
  }
  int which() const { return (int)v_.index(); }

 private:
  std::variant<Ts...> v_;
};

template <class V, class Visitable>
decltype(auto) apply_visitor(const V& vis, Visitable&& v) {
  return std::forward<Visitable>(v).apply_visitor(vis);
}
}  // namespace boost
#endif
