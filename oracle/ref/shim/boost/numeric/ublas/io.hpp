// Declarations only (CPU oracle build): see matrix.hpp.
#ifndef HB_REF_SHIM_BOOST_UBLAS_IO_HPP
#define HB_REF_SHIM_BOOST_UBLAS_IO_HPP
#include "boost/numeric/ublas/matrix.hpp"
#endif
