// The real MPI C++ bindings and boost headers bring the common standard library
// headers with them, and some reference headers rely on that (std::map and assert are used
// without their headers in lb/iolets/InOutLetFileVelocity.h, net/MpiCommunicator.cc and
// geometry/decomposition/OptimisedDecomposition.h).
#ifndef HB_REF_SHIM_STD_HEADERS_H
#define HB_REF_SHIM_STD_HEADERS_H
#include <algorithm>
#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <cstddef>
#include <cstring>
#include <iosfwd>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>
#endif
