// Host-side objects behind the mdelast_pair / mdelast_eam handles of include/mdelast.h,
// and the error plumbing shared by the library's host code.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "mdelast.h"

namespace mdelast {

// Thread-local error message; returns code for "return fail(...)" use.
int fail(int code, char const *fmt, ...);
void clear_error();
char const *last_error();

// Piecewise quintic table on x_i = i h (poly_table.hpp:21-115): 6 coefficients per
// interval in t = (x - x_i)/h, built in long double, evaluated by Horner.
struct QuinticTable {
    double h = 0, inv_h = 0, inv_h2 = 0;
    int n = 0; // intervals
    std::vector<double> coef; // 6 n

    // "bspline" tables (poly_table.hpp:117-135): three independent cardinal cubic
    // B-splines through the node values of f, f', f'' (coefficients b_-1..b_n of each), and
    // per interval the three cubics in t they reduce to (12 n: f, f', f'' pieces)
    int bspline = 0;
    std::vector<double> bs[3];
    std::vector<double> cub;

    int build(double h_, int64_t n_nodes, double const *f, double const *f1, double const *f2);
    int build_bspline(double const *f, double const *f1, double const *f2);
    // f, f', f'' at x (poly_table.hpp:71-114, or the three splines' values)
    void eval(double x, double out[3]) const;
};

enum PairKind { PAIR_TABLE = 0, PAIR_MORSE = 1, PAIR_LJ = 2 };

} // namespace mdelast

struct mdelast_pair_s {
    int kind = mdelast::PAIR_TABLE;
    int interpolation = MDELAST_QUINTIC;
    double rcut = 0, rmin_fatal = 0;
    mdelast::QuinticTable table;
    double p0 = 0, p1 = 0, p2 = 0; // Morse D, alpha, r0 ; LJ epsilon, sigma, vcut
};

struct mdelast_eam_s {
    int interpolation = MDELAST_QUINTIC;
    double rcut = 0, rhomax_fatal = 0;
    mdelast::QuinticTable rho, F;
};
