// Project-written stand-in for boost::math::pow<N>(x), the integer power the mdelast core
// uses (N = 2 on the EAM path; 6 and 12 in the Lennard-Jones potential). Test
// infrastructure only (oracle/_ref). Evaluated by repeated squaring; for N = 2 it is x*x.
#ifndef MDELAST_ORACLE_BOOST_POW_SHIM_
#define MDELAST_ORACLE_BOOST_POW_SHIM_

#include <cassert> // the real header pulls this in, and barostat.cpp relies on it

namespace boost {
namespace math {

template <int N, typename T> constexpr T pow(T const x) {
    if constexpr (N == 0) {
        return T(1);
    } else if constexpr (N == 1) {
        return x;
    } else if constexpr (N % 2 == 0) {
        T const h = pow<N / 2>(x);
        return h * h;
    } else {
        return x * pow<N - 1>(x);
    }
}

} // namespace math
} // namespace boost

#endif
