// Declarations only (CPU oracle build): see matrix.hpp.
#ifndef HB_REF_SHIM_BOOST_UBLAS_LU_HPP
#define HB_REF_SHIM_BOOST_UBLAS_LU_HPP
#include "boost/numeric/ublas/matrix.hpp"
namespace boost {
namespace numeric {
namespace ublas {
template <class M, class P>
int lu_factorize(M& m, P& pm);
template <class M, class P, class V>
void lu_substitute(const M& m, const P& pm, V& v);
}  // namespace ublas
}  // namespace numeric
}  // namespace boost
#endif
