// Tabulated and analytic pair functions and EAM functions on the host: construction of the
// quintic coefficients and the scalar evaluators behind Potential.calculate(), EAM.rho()
// and friends. The MD step never calls these; drivers upload the coefficients.
#include "host_tables.h"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <new>

namespace mdelast {

namespace {
thread_local std::string g_error;
}

int fail(int code, char const *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

void clear_error() { g_error.clear(); }

char const *last_error() { return g_error.c_str(); }

// poly_table.hpp:35-63. With node values f, slopes f' and curvatures f'' at both ends of
// an interval, the quintic Hermite polynomial in t has
//   a0 = f0, a1 = h f0', a2 = h^2 f0''/2 and a3..a5 from the three end conditions.
// a3..a5 come from cancelling O(h f') terms and are formed in long double.
int QuinticTable::build(double h_, int64_t n_nodes, double const *f, double const *f1,
                        double const *f2) {
    if (n_nodes < 2 || !(h_ > 0.))
        return fail(MDELAST_ERR_ARGUMENT,
                    "FATAL: QuinticTable needs >= 2 nodes, equal array sizes, and h > 0 "
                    "(nodes %lld, h %g)",
                    static_cast<long long>(n_nodes), h_);
    h = h_;
    inv_h = 1. / h_;
    inv_h2 = 1. / (h_ * h_);
    n = static_cast<int>(n_nodes - 1);
    coef.assign(6 * static_cast<size_t>(n), 0.);
    using ld = long double;
    ld const hl = static_cast<ld>(h_);
    for (int i = 0; i < n; ++i) {
        ld const dy = static_cast<ld>(f[i + 1]) - static_cast<ld>(f[i]);
        ld const d0 = hl * static_cast<ld>(f1[i]), d1 = hl * static_cast<ld>(f1[i + 1]);
        ld const s0 = hl * hl * static_cast<ld>(f2[i]), s1 = hl * hl * static_cast<ld>(f2[i + 1]);
        double *c = coef.data() + 6 * static_cast<size_t>(i);
        c[0] = f[i];
        c[1] = static_cast<double>(d0);
        c[2] = static_cast<double>(0.5L * s0);
        c[3] = static_cast<double>(10.L * dy - 6.L * d0 - 4.L * d1 - 0.5L * (3.L * s0 - s1));
        c[4] = static_cast<double>(-15.L * dy + 8.L * d0 + 7.L * d1 +
                                   0.5L * (3.L * s0 - 2.L * s1));
        c[5] = static_cast<double>(6.L * dy - 3.L * (d0 + d1) - 0.5L * (s0 - s1));
    }
    return MDELAST_OK;
}

namespace {

// Cardinal cubic B-spline through f_0..f_{m-1} on x_i = i h (the Boost 1.84
// cardinal_cubic_b_spline the reference's BSplineTable uses, restated from the textbook
// clamped interpolant, de Boor ch. IX): s(x) = sum_k b_k B((x - x_k) / h), k = -1..m, B the
// centred cubic B-spline, s(x_i) = f_i, end slopes from the second-order one-sided
// differences, the tridiagonal system solved by the Thomas algorithm. Returns b_-1..b_m.
std::vector<double> bspline_fit(double h, int m, double const *f) {
    std::vector<double> out(static_cast<size_t>(m) + 2, m ? f[0] : 0.);
    if (m < 3)
        return out;
    double const inv_h = 1. / h;
    double const d0 = (-3 * f[0] + 4 * f[1] - f[2]) * inv_h / 2;
    double const d1 = (3 * f[m - 1] - 4 * f[m - 2] + f[m - 3]) * inv_h / 2;
    std::vector<double> lo(m, 1.), di(m, 4.), up(m, 1.), rhs(m), b(m);
    for (int i = 0; i < m; ++i)
        rhs[i] = 6 * f[i];
    up[0] = 2;
    rhs[0] += 2 * h * d0;
    lo[m - 1] = 2;
    rhs[m - 1] -= 2 * h * d1;
    for (int i = 1; i < m; ++i) {
        double const q = lo[i] / di[i - 1];
        di[i] -= q * up[i - 1];
        rhs[i] -= q * rhs[i - 1];
    }
    b[m - 1] = rhs[m - 1] / di[m - 1];
    for (int i = m - 1; i-- > 0;)
        b[i] = (rhs[i] - up[i] * b[i + 1]) / di[i];
    for (int i = 0; i < m; ++i)
        out[static_cast<size_t>(i) + 1] = b[i];
    out[0] = b[1] - 2 * h * d0;
    out[static_cast<size_t>(m) + 1] = b[m - 2] + 2 * h * d1;
    return out;
}

// the spline's value: the weights of the four nearest coefficients
double bspline_value(std::vector<double> const &bb, int m, double inv_h, double x) {
    if (m < 3)
        return bb[0];
    double const u = x * inv_h;
    if (!(u == u))
        return u;
    long k = static_cast<long>(std::floor(u));
    if (k < 0)
        k = 0;
    if (k > m - 2)
        k = m - 2;
    double s = 0;
    for (long j = k - 1; j <= k + 2; ++j) {
        double const t = std::fabs(u - static_cast<double>(j));
        double w;
        if (t < 1)
            w = 2. / 3 - t * t + t * t * t / 2;
        else if (t < 2)
            w = (2 - t) * (2 - t) * (2 - t) / 6;
        else
            w = 0;
        s += w * bb[static_cast<size_t>(j + 1)];
    }
    return s;
}

} // namespace

int QuinticTable::build_bspline(double const *f, double const *f1, double const *f2) {
    int const m = n + 1; // nodes
    double const *src[3] = {f, f1, f2};
    for (int q = 0; q < 3; ++q)
        bs[q] = bspline_fit(h, m, src[q]);
    // on interval k (t in [0,1)) the spline is the cubic
    //   ((b_{k-1} + 4 b_k + b_{k+1}) + 3 (b_{k+1} - b_{k-1}) t
    //    + 3 (b_{k-1} - 2 b_k + b_{k+1}) t^2 + (b_{k+2} - b_{k-1} + 3 (b_k - b_{k+1})) t^3) / 6
    cub.assign(12 * static_cast<size_t>(n), 0.);
    using ld = long double;
    for (int k = 0; k < n; ++k)
        for (int q = 0; q < 3; ++q) {
            std::vector<double> const &b = bs[q];
            ld const bm = b[k], b0 = b[k + 1], b1 = b[k + 2], b2 = b[k + 3];
            double *c = cub.data() + 12 * static_cast<size_t>(k) + 4 * q;
            if (m < 3) {
                c[0] = b[0];
                continue;
            }
            c[0] = static_cast<double>((bm + 4.L * b0 + b1) / 6.L);
            c[1] = static_cast<double>((b1 - bm) / 2.L);
            c[2] = static_cast<double>((bm - 2.L * b0 + b1) / 2.L);
            c[3] = static_cast<double>((b2 - bm + 3.L * (b0 - b1)) / 6.L);
        }
    bspline = 1;
    return MDELAST_OK;
}

// poly_table.hpp:71-114: interval index clamped to [0, n-1] with the range test done in
// floating point (a NaN argument takes interval 0 and gives NaN).
void QuinticTable::eval(double x, double out[3]) const {
    if (bspline) {
        for (int q = 0; q < 3; ++q)
            out[q] = bspline_value(bs[q], n + 1, inv_h, x);
        return;
    }
    double const u = x * inv_h;
    int i = 0;
    if (u >= static_cast<double>(n))
        i = n - 1;
    else if (u > 0.)
        i = static_cast<int>(u);
    double const t = u - static_cast<double>(i);
    double const *c = coef.data() + 6 * static_cast<size_t>(i);
    out[0] = c[0] + t * (c[1] + t * (c[2] + t * (c[3] + t * (c[4] + t * c[5]))));
    out[1] = (c[1] + t * (2. * c[2] + t * (3. * c[3] + t * (4. * c[4] + t * 5. * c[5])))) * inv_h;
    out[2] = (2. * c[2] + t * (6. * c[3] + t * (12. * c[4] + t * 20. * c[5]))) * inv_h2;
}

} // namespace mdelast

using namespace mdelast;

namespace {

int check_interp(int interpolation) {
    if (interpolation == MDELAST_QUINTIC || interpolation == MDELAST_BSPLINE)
        return MDELAST_OK;
    return fail(MDELAST_ERR_ARGUMENT,
                "FATAL: unknown table interpolation %d (use 'quintic' or 'bspline')",
                interpolation);
}

} // namespace

extern "C" {

int mdelast_pair_table_create(double rcut, double rmin_fatal, double dr, int64_t n_nodes,
                              const double *v, const double *dv, const double *d2v,
                              int interpolation, mdelast_pair **out) {
    clear_error();
    if (!out || !v || !dv || !d2v)
        return fail(MDELAST_ERR_ARGUMENT, "null argument");
    if (int rc = check_interp(interpolation))
        return rc;
    auto *p = new (std::nothrow) mdelast_pair_s();
    if (!p)
        return fail(MDELAST_ERR_ARGUMENT, "out of host memory");
    p->kind = PAIR_TABLE;
    p->interpolation = interpolation;
    p->rcut = rcut;
    p->rmin_fatal = rmin_fatal;
    int rc = p->table.build(dr, n_nodes, v, dv, d2v);
    if (!rc && interpolation == MDELAST_BSPLINE)
        rc = p->table.build_bspline(v, dv, d2v);
    if (rc) {
        delete p;
        return rc;
    }
    *out = p;
    return MDELAST_OK;
}

int mdelast_pair_morse_create(double rcut, double D, double alpha, double r0,
                              mdelast_pair **out) {
    clear_error();
    if (!out)
        return fail(MDELAST_ERR_ARGUMENT, "null argument");
    auto *p = new mdelast_pair_s();
    p->kind = PAIR_MORSE;
    p->rcut = rcut;
    p->p0 = D;
    p->p1 = alpha;
    p->p2 = r0;
    *out = p;
    return MDELAST_OK;
}

int mdelast_pair_lj_create(double rcut, double epsilon, double sigma, mdelast_pair **out) {
    clear_error();
    if (!out)
        return fail(MDELAST_ERR_ARGUMENT, "null argument");
    auto *p = new mdelast_pair_s();
    p->kind = PAIR_LJ;
    p->rcut = rcut;
    p->p0 = epsilon;
    p->p1 = sigma;
    // potential.hpp:60-63: the energy is shifted by V(rcut)
    double const s6 = std::pow(sigma / rcut, 6);
    p->p2 = 4. * epsilon * (s6 * s6 - s6);
    *out = p;
    return MDELAST_OK;
}

int mdelast_pair_eval(const mdelast_pair *p, double r, double out[3]) {
    if (!p || !out)
        return fail(MDELAST_ERR_ARGUMENT, "null argument");
    if (r > p->rcut) { // potential.hpp:40-43, 64-66, 95-98
        out[0] = out[1] = out[2] = 0.;
        return MDELAST_OK;
    }
    switch (p->kind) {
    case PAIR_TABLE:
        p->table.eval(r, out);
        break;
    case PAIR_MORSE: { // potential.hpp:40-50
        double const e1 = std::exp(-p->p1 * (r - p->p2)), e2 = e1 * e1;
        out[0] = p->p0 * (e2 - 2. * e1);
        out[1] = -2. * p->p0 * p->p1 * (e2 - e1);
        out[2] = 2. * p->p1 * p->p1 * p->p0 * (2. * e2 - e1);
        break;
    }
    default: { // potential.hpp:64-74
        double const s = p->p1 / r, s2 = s * s, v6 = s2 * s2 * s2, v12 = v6 * v6;
        out[0] = 4. * p->p0 * (v12 - v6) - p->p2;
        out[1] = 24. * p->p0 * (v6 - 2. * v12) / r;
        out[2] = 24. * p->p0 * (26. * v12 - 7. * v6) / (r * r);
        break;
    }
    }
    return MDELAST_OK;
}

int mdelast_pair_info(const mdelast_pair *p, double *rcut, int *kind, int *interpolation) {
    if (!p)
        return fail(MDELAST_ERR_ARGUMENT, "null argument");
    if (rcut)
        *rcut = p->rcut;
    if (kind)
        *kind = p->kind;
    if (interpolation)
        *interpolation = p->interpolation;
    return MDELAST_OK;
}

void mdelast_pair_destroy(mdelast_pair *p) { delete p; }

int mdelast_eam_create(double rcut, double rhomax_fatal, double dr, double drho, int64_t n_r,
                       const double *rho, const double *drho_dr, const double *d2rho_dr2,
                       int64_t n_rho, const double *F, const double *dF, const double *d2F,
                       int interpolation, mdelast_eam **out) {
    clear_error();
    if (!out || !rho || !drho_dr || !d2rho_dr2 || !F || !dF || !d2F)
        return fail(MDELAST_ERR_ARGUMENT, "null argument");
    if (int rc = check_interp(interpolation))
        return rc;
    auto *e = new mdelast_eam_s();
    e->interpolation = interpolation;
    e->rcut = rcut;
    e->rhomax_fatal = rhomax_fatal;
    int rc = e->rho.build(dr, n_r, rho, drho_dr, d2rho_dr2);
    if (!rc)
        rc = e->F.build(drho, n_rho, F, dF, d2F);
    if (!rc && interpolation == MDELAST_BSPLINE)
        rc = e->rho.build_bspline(rho, drho_dr, d2rho_dr2);
    if (!rc && interpolation == MDELAST_BSPLINE)
        rc = e->F.build_bspline(F, dF, d2F);
    if (rc) {
        delete e;
        return rc;
    }
    *out = e;
    return MDELAST_OK;
}

int mdelast_eam_eval(const mdelast_eam *e, int what, double x, double *out) {
    if (!e || !out || what < 0 || what > 5)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    double v[3];
    if (what < 3) { // eam.hpp:30-46
        if (x > e->rcut) {
            *out = 0.;
            return MDELAST_OK;
        }
        e->rho.eval(x, v);
        *out = v[what];
        return MDELAST_OK;
    }
    if (x > e->rhomax_fatal) { // eam.hpp:48-70
        static char const *names[3] = {"F", "dFdrho", "d2Fdrho2"};
        return fail(MDELAST_ERR_FATAL, "FATAL: EAM %s rho >rhomax_fatal %g %g", names[what - 3],
                    x, e->rhomax_fatal);
    }
    e->F.eval(x, v);
    *out = v[what - 3];
    return MDELAST_OK;
}

int mdelast_eam_info(const mdelast_eam *e, double *rcut, double *rhomax_fatal,
                     int *interpolation) {
    if (!e)
        return fail(MDELAST_ERR_ARGUMENT, "null argument");
    if (rcut)
        *rcut = e->rcut;
    if (rhomax_fatal)
        *rhomax_fatal = e->rhomax_fatal;
    if (interpolation)
        *interpolation = e->interpolation;
    return MDELAST_OK;
}

void mdelast_eam_destroy(mdelast_eam *e) { delete e; }

int mdelast_abi_version(void) { return MDELAST_ABI_VERSION; }

const char *mdelast_last_error(void) { return mdelast::last_error(); }

} // extern "C"
