// Project-written stand-in for boost::math::interpolators::cardinal_cubic_b_spline, so
// that the reference's poly_table.hpp compiles without Boost. Test infrastructure only
// (oracle/_ref); the product's "bspline" tables are separate code.
//
// Method (the textbook clamped cubic B-spline interpolant on a uniform grid, as in de Boor,
// "A Practical Guide to Splines", ch. IX): s(x) = sum_k b_k B((x - x_k)/h) over k = -1..n,
// B the centred cubic B-spline; s(x_i) = f_i for the n nodes and s'(x_0), s'(x_{n-1}) fixed.
// When the caller gives no endpoint derivatives (as mdelast does) they are estimated by the
// second-order one-sided difference (-3 f_0 + 4 f_1 - f_2) / (2h) and its mirror image. The
// library this stands in for also estimates them by a finite difference, whose exact form
// is not known here, so values within a few intervals of either end may differ from it.
#ifndef MDELAST_ORACLE_BOOST_CUBIC_BSPLINE_SHIM_
#define MDELAST_ORACLE_BOOST_CUBIC_BSPLINE_SHIM_

#include <cmath>
#include <cstddef>
#include <iterator>
#include <limits>
#include <vector>

namespace boost {
namespace math {
namespace interpolators {

template <class Real> class cardinal_cubic_b_spline {
  public:
    template <class It>
    cardinal_cubic_b_spline(It f_begin, It f_end, Real left_endpoint, Real step_size,
                            Real left_endpoint_derivative = std::numeric_limits<Real>::quiet_NaN(),
                            Real right_endpoint_derivative = std::numeric_limits<Real>::quiet_NaN())
        : a_(left_endpoint), h_(step_size), inv_h_(Real(1) / step_size) {
        std::vector<Real> f(f_begin, f_end);
        std::size_t const n = f.size();
        n_ = n;
        if (n < 3) {
            b_.assign(n + 2, n ? f[0] : Real(0));
            return;
        }
        Real d0 = left_endpoint_derivative, d1 = right_endpoint_derivative;
        if (std::isnan(d0))
            d0 = (-3 * f[0] + 4 * f[1] - f[2]) * inv_h_ / 2;
        if (std::isnan(d1))
            d1 = (3 * f[n - 1] - 4 * f[n - 2] + f[n - 3]) * inv_h_ / 2;
        // unknowns b_0..b_{n-1}; b_{-1} and b_n eliminated with the derivative conditions
        std::vector<Real> lo(n, 1), di(n, 4), up(n, 1), rhs(n);
        for (std::size_t i = 0; i < n; ++i)
            rhs[i] = 6 * f[i];
        up[0] = 2;
        rhs[0] += 2 * h_ * d0;
        lo[n - 1] = 2;
        rhs[n - 1] -= 2 * h_ * d1;
        // Thomas algorithm
        for (std::size_t i = 1; i < n; ++i) {
            Real const m = lo[i] / di[i - 1];
            di[i] -= m * up[i - 1];
            rhs[i] -= m * rhs[i - 1];
        }
        std::vector<Real> b(n);
        b[n - 1] = rhs[n - 1] / di[n - 1];
        for (std::size_t i = n - 1; i-- > 0;)
            b[i] = (rhs[i] - up[i] * b[i + 1]) / di[i];
        b_.resize(n + 2);
        for (std::size_t i = 0; i < n; ++i)
            b_[i + 1] = b[i];
        b_[0] = b[1] - 2 * h_ * d0;
        b_[n + 1] = b[n - 2] + 2 * h_ * d1;
    }

    Real operator()(Real x) const {
        if (n_ < 3)
            return b_.empty() ? Real(0) : b_[0];
        Real const u = (x - a_) * inv_h_;
        long k = static_cast<long>(std::floor(u));
        if (!(u == u))
            return u;
        if (k < 0)
            k = 0;
        if (k > static_cast<long>(n_) - 2)
            k = static_cast<long>(n_) - 2;
        Real s = 0;
        for (long j = k - 1; j <= k + 2; ++j) {
            Real const t = std::fabs(u - static_cast<Real>(j));
            Real w;
            if (t < 1)
                w = Real(2) / 3 - t * t + t * t * t / 2;
            else if (t < 2)
                w = (2 - t) * (2 - t) * (2 - t) / 6;
            else
                w = 0;
            s += w * b_[static_cast<std::size_t>(j + 1)];
        }
        return s;
    }

  private:
    Real a_, h_, inv_h_;
    std::size_t n_ = 0;
    std::vector<Real> b_; // b_{-1} .. b_{n}
};

} // namespace interpolators
} // namespace math
} // namespace boost

#endif
