// The elastic-constant estimator of molecular_dynamics.py:776-824 and 826-958 evaluated on
// the host from the production-window sums the device keeps (mdelast_fluct): the same
// terms as the reference's per-sample formula, written with means and population
// co-moments instead of sample arrays.
//
//   C_ij = <C^B_ij> - <V>/kT cov(s'_i, s'_j) + c_ij <N/V> kT + K [NPT, i, j < 3]
//
// with c_ij = 2 (i = j < 3), 1 (i = j >= 3), 0 otherwise (the ideal-gas term, :921-930),
// s' = sigma^B in NVT and sigma^B - (N kT / V) delta in NPT (:852-863), so that in NPT
//   cov(s'_i, s'_j) = cov(sB_i, sB_j) - kT [j<3] cov(sB_i, rho) - kT [i<3] cov(rho, sB_j)
//                     + kT^2 [i<3][j<3] var(rho),  rho = N / V;
// K = <V> kT / var(V) (:776-795) and the volumetric thermal expansion
// (N cov(V, e_tot) + P var(V)) / (<V> k T^2) (:797-824). All co-moments are population
// ones (divided by n), as the reference's get_mean_std and window means.
#include <cmath>

#include "host_tables.h"
#include "mdelast.h"

using mdelast::clear_error;
using mdelast::fail;

namespace {

constexpr double kBoltz = 1.38064852e-16; // units.hpp:6

// index of (a, b), a <= b, in the row-by-row upper triangle of an m x m matrix
int upper(int a, int b, int m) {
    if (a > b) {
        int const t = a;
        a = b;
        b = t;
    }
    return a * m - a * (a - 1) / 2 + (b - a);
}

} // namespace

extern "C" int mdelast_elastic_constants(const mdelast_fluct *f, int32_t ensemble,
                                         double T_thermostat, double P_barostat, double *C,
                                         double *summary) {
    clear_error();
    if (!f || !C || !(T_thermostat > 0.))
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    if (!(f->n >= 2.))
        return fail(MDELAST_ERR_ARGUMENT, "the estimator needs at least 2 samples (%g given)",
                    f->n);
    double const n = f->n;
    double const kT = kBoltz * T_thermostat;
    auto cov = [&](int a, int b) { return f->comoment[upper(a, b, 9)] / n; };
    bool const npt = ensemble == MDELAST_NPT;
    double const Vm = f->mean[7], rho_m = f->mean[6];
    double const varV = cov(7, 7);
    double K = 0., compressibility = 0., expansion = 0.;
    if (npt) {
        compressibility = varV / (Vm * kT);
        K = 1. / compressibility;
        expansion = (f->n_atoms * cov(7, 8) + P_barostat * varV) /
                    (Vm * kBoltz * T_thermostat * T_thermostat);
    }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = cov(i, j);
            if (npt) {
                if (j < 3)
                    s -= kT * cov(i, 6);
                if (i < 3)
                    s -= kT * cov(6, j);
                if (i < 3 && j < 3)
                    s += kT * kT * cov(6, 6);
            }
            double const born = i <= j ? f->born_el_mean[upper(i, j, 6)] : 0.;
            double const ideal = i == j ? (i < 3 ? 2. : 1.) * rho_m * kT : 0.;
            double const bulk = npt && i < 3 && j < 3 ? K : 0.;
            C[6 * i + j] = born - Vm / kT * s + ideal + bulk;
        }
    if (summary) {
        summary[0] = (C[0] + C[7] + C[14]) / 3.;
        summary[1] = (C[1] + C[2] + C[8]) / 3.;
        summary[2] = (C[21] + C[28] + C[35]) / 3.;
        summary[3] = K;
        summary[4] = compressibility;
        summary[5] = expansion;
    }
    return MDELAST_OK;
}
