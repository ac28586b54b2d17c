// Declarations only (CPU oracle build).  boost::numeric::ublas is used by the
// JunkYang wall streamer (lb/streamers/JunkYangFactory.h), which the reference's
// headers always include but which none of the oracle's builds selects, so the
// class template is parsed and never instantiated.  The names below let it
// parse; nothing is defined, so any use that did get instantiated would fail
// to link rather than compute something wrong.
#ifndef HB_REF_SHIM_BOOST_UBLAS_MATRIX_HPP
#define HB_REF_SHIM_BOOST_UBLAS_MATRIX_HPP
#include <cstddef>
#include <iosfwd>
#include <type_traits>
namespace boost {
namespace numeric {
namespace ublas {
struct expression_tag {};
struct expression : expression_tag {};

template <class T>
class vector : public expression_tag {
 public:
  vector();
  explicit vector(std::size_t n);
  template <class E, class = std::enable_if_t<std::is_base_of<expression_tag, E>::value>>
  vector(const E& e);
  template <class E>
  vector& operator=(const E& e);
  void resize(std::size_t n, bool preserve = true);
  std::size_t size() const;
  T& operator[](std::size_t i);
  const T& operator[](std::size_t i) const;
  T& operator()(std::size_t i);
  const T& operator()(std::size_t i) const;
};

template <class T, std::size_t N>
class c_vector : public expression_tag {
 public:
  c_vector();
  template <class E, class = std::enable_if_t<std::is_base_of<expression_tag, E>::value>>
  c_vector(const E& e);
  template <class E>
  c_vector& operator=(const E& e);
  std::size_t size() const;
  T& operator[](std::size_t i);
  const T& operator[](std::size_t i) const;
  T& operator()(std::size_t i);
  const T& operator()(std::size_t i) const;
};

template <class T>
class matrix : public expression_tag {
 public:
  matrix();
  matrix(std::size_t rows, std::size_t cols);
  template <class E, class = std::enable_if_t<std::is_base_of<expression_tag, E>::value>>
  matrix(const E& e);
  template <class E>
  matrix& operator=(const E& e);
  void resize(std::size_t rows, std::size_t cols, bool preserve = true);
  std::size_t size1() const;
  std::size_t size2() const;
  T& operator()(std::size_t i, std::size_t j);
  const T& operator()(std::size_t i, std::size_t j) const;
};

template <class T>
class identity_matrix : public expression_tag {
 public:
  explicit identity_matrix(std::size_t n);
};

template <class T>
class permutation_matrix {
 public:
  explicit permutation_matrix(std::size_t n);
};

template <class A, class B>
using either_expression = std::enable_if_t<std::is_base_of<expression_tag, A>::value ||
                                               std::is_base_of<expression_tag, B>::value,
                                           expression>;
template <class A, class B>
either_expression<A, B> operator+(const A& a, const B& b);
template <class A, class B>
either_expression<A, B> operator-(const A& a, const B& b);
template <class A, class B>
either_expression<A, B> operator*(const A& a, const B& b);

template <class M>
expression subrange(const M& m, std::size_t r0, std::size_t r1, std::size_t c0, std::size_t c1);
template <class A, class B>
expression prod(const A& a, const B& b);
}  // namespace ublas
}  // namespace numeric
}  // namespace boost
#endif
