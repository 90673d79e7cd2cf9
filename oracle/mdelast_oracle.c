/* CPU restatement of mdelast's EAM force-and-stress step: the test oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see mdelast_oracle.h). Every function restates the reference
 * code named in its comment, in the reference's operation order, with the data held in
 * flat C arrays (xyz interleaved per atom) instead of the reference's C++ objects.
 * References are to the mdelast sources (src/...).
 */
#include "mdelast_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* src/units.hpp:6-24 */
static const double K_BOLTZ = 1.38064852e-16;

/* src/numerics.hpp:22-27, Suzuki-Yoshida 7-stage weights (Tuckerman eq. 4.11.12) */
static const double WSY7[7] = {
    0.784513610477560, 0.235573213359357, -1.17767998417887,
    1. - 2. * (0.784513610477560 + 0.235573213359357 - 1.17767998417887),
    -1.17767998417887, 0.235573213359357, 0.784513610477560};

/* Voigt order xx yy zz yz xz xy, src/md_driver.hpp:23-24 */
static const int VA[6] = {0, 1, 2, 1, 0, 0};
static const int VB[6] = {0, 1, 2, 2, 2, 1};

/* ------------------------------------------------------------------------------------ */
/* quintic table: src/poly_table.hpp:33-115                                               */

typedef struct {
    double h, inv_h, inv_h2;
    int n; /* intervals */
    double *c; /* 6 per interval */
    /* "bspline" (poly_table.hpp:117-135): three cardinal cubic B-splines through the node
     * values of f, f', f''; coefficients b_{-1}..b_{n_nodes} of each, NULL for quintic */
    double *bs[3];
    int nodes;
} qtab;

/* Cardinal cubic B-spline on nodes x_i = i h, i < n (Boost 1.84
 * cardinal_cubic_b_spline, which the reference uses for its "bspline" tables; restated
 * here, and in the project's shim oracle/shim/boost/.../cardinal_cubic_b_spline.hpp, from
 * the textbook clamped interpolant, de Boor ch. IX): s(x) = sum_k b_k B((x - x_k) / h),
 * k = -1..n, B the centred cubic B-spline, s(x_i) = f_i, and the end slopes estimated by the
 * second-order one-sided differences. Same operations, in the same order, as the shim. */
static void bspline_fit(double h, int n, double const *f, double *b_out /* n + 2 */) {
    double const inv_h = 1. / h;
    if (n < 3) {
        for (int i = 0; i < n + 2; ++i)
            b_out[i] = n ? f[0] : 0.;
        return;
    }
    double const d0 = (-3 * f[0] + 4 * f[1] - f[2]) * inv_h / 2;
    double const d1 = (3 * f[n - 1] - 4 * f[n - 2] + f[n - 3]) * inv_h / 2;
    double *lo = (double *)malloc(sizeof(double) * (size_t)n);
    double *di = (double *)malloc(sizeof(double) * (size_t)n);
    double *up = (double *)malloc(sizeof(double) * (size_t)n);
    double *rhs = (double *)malloc(sizeof(double) * (size_t)n);
    double *b = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        lo[i] = 1;
        di[i] = 4;
        up[i] = 1;
        rhs[i] = 6 * f[i];
    }
    up[0] = 2;
    rhs[0] += 2 * h * d0;
    lo[n - 1] = 2;
    rhs[n - 1] -= 2 * h * d1;
    for (int i = 1; i < n; ++i) {
        double const m = lo[i] / di[i - 1];
        di[i] -= m * up[i - 1];
        rhs[i] -= m * rhs[i - 1];
    }
    b[n - 1] = rhs[n - 1] / di[n - 1];
    for (int i = n - 1; i-- > 0;)
        b[i] = (rhs[i] - up[i] * b[i + 1]) / di[i];
    for (int i = 0; i < n; ++i)
        b_out[i + 1] = b[i];
    b_out[0] = b[1] - 2 * h * d0;
    b_out[n + 1] = b[n - 2] + 2 * h * d1;
    free(lo);
    free(di);
    free(up);
    free(rhs);
    free(b);
}

static double bspline_eval(double const *bb, int n, double inv_h, double x) {
    if (n < 3)
        return bb[0];
    double const u = (x - 0.) * inv_h;
    long k = (long)floor(u);
    if (!(u == u))
        return u;
    if (k < 0)
        k = 0;
    if (k > (long)n - 2)
        k = (long)n - 2;
    double s = 0;
    for (long j = k - 1; j <= k + 2; ++j) {
        double const t = fabs(u - (double)j);
        double w;
        if (t < 1)
            w = 2. / 3 - t * t + t * t * t / 2;
        else if (t < 2)
            w = (2 - t) * (2 - t) * (2 - t) / 6;
        else
            w = 0;
        s += w * bb[j + 1];
    }
    return s;
}

/* the spline through f_0..f_{n-1} (spacing h) evaluated at x: a test entry point */
double orc_bspline_value(double h, int n, double const *f, double x) {
    double *b = (double *)malloc(sizeof(double) * ((size_t)n + 2));
    bspline_fit(h, n, f, b);
    double const v = bspline_eval(b, n, 1. / h, x);
    free(b);
    return v;
}

int orc_quintic_coefficients(double h, int n_nodes, double const *f, double const *f1,
                             double const *f2, double *coef) {
    /* poly_table.hpp:35-63: per interval the quintic Hermite polynomial in t in [0,1]
     * fixed by f, h f', h^2 f'' at both nodes; a3..a5 formed in long double */
    if (n_nodes < 2 || !(h > 0.))
        return -1;
    typedef long double ld;
    ld const hl = (ld)h;
    for (int i = 0; i < n_nodes - 1; ++i) {
        int const a = i, b = i + 1;
        ld const dy = (ld)f[b] - (ld)f[a];
        ld const D0 = hl * (ld)f1[a], D1 = hl * (ld)f1[b];
        ld const S0 = hl * hl * (ld)f2[a], S1 = hl * hl * (ld)f2[b];
        double *c = coef + 6 * i;
        c[0] = f[a];
        c[1] = (double)D0;
        c[2] = (double)(0.5L * S0);
        c[3] = (double)(10.L * dy - 6.L * D0 - 4.L * D1 - 0.5L * (3.L * S0 - S1));
        c[4] = (double)(-15.L * dy + 8.L * D0 + 7.L * D1 + 0.5L * (3.L * S0 - 2.L * S1));
        c[5] = (double)(6.L * dy - 3.L * (D0 + D1) - 0.5L * (S0 - S1));
    }
    return 0;
}

static int qtab_init(qtab *t, double h, int n_nodes, double const *f, double const *f1,
                     double const *f2, int bspline) {
    t->h = h;
    t->inv_h = 1. / h;
    t->inv_h2 = 1. / (h * h);
    t->n = n_nodes - 1;
    t->nodes = n_nodes;
    t->c = (double *)malloc(sizeof(double) * 6 * (size_t)(t->n > 0 ? t->n : 1));
    t->bs[0] = t->bs[1] = t->bs[2] = NULL;
    if (bspline) {
        double const *src[3] = {f, f1, f2};
        for (int k = 0; k < 3; ++k) {
            t->bs[k] = (double *)malloc(sizeof(double) * ((size_t)n_nodes + 2));
            bspline_fit(h, n_nodes, src[k], t->bs[k]);
        }
    }
    return orc_quintic_coefficients(h, n_nodes, f, f1, f2, t->c);
}

static void qtab_free(qtab *t) {
    free(t->c);
    for (int k = 0; k < 3; ++k)
        free(t->bs[k]);
}

/* poly_table.hpp:105-114: clamped interval index, NaN-safe */
static double const *qtab_locate(qtab const *T, double x, double *t) {
    double const u = x * T->inv_h;
    int i = 0;
    if (u >= (double)T->n)
        i = T->n - 1;
    else if (u > 0.)
        i = (int)u;
    *t = u - (double)i;
    return T->c + 6 * i;
}

static double qtab_value(qtab const *T, double x) {
    if (T->bs[0])
        return bspline_eval(T->bs[0], T->nodes, T->inv_h, x);
    double t;
    double const *c = qtab_locate(T, x, &t);
    return c[0] + t * (c[1] + t * (c[2] + t * (c[3] + t * (c[4] + t * c[5]))));
}

static double qtab_d1(qtab const *T, double x) {
    if (T->bs[1])
        return bspline_eval(T->bs[1], T->nodes, T->inv_h, x);
    double t;
    double const *c = qtab_locate(T, x, &t);
    return (c[1] + t * (2. * c[2] + t * (3. * c[3] + t * (4. * c[4] + t * 5. * c[5])))) *
           T->inv_h;
}

static double qtab_d2(qtab const *T, double x) {
    if (T->bs[2])
        return bspline_eval(T->bs[2], T->nodes, T->inv_h, x);
    double t;
    double const *c = qtab_locate(T, x, &t);
    return (2. * c[2] + t * (6. * c[3] + t * (12. * c[4] + t * 20. * c[5]))) * T->inv_h2;
}

void orc_quintic_eval(double const *coef, int n_intervals, double h, double x, double *o) {
    qtab T = {h, 1. / h, 1. / (h * h), n_intervals, (double *)coef, {NULL, NULL, NULL},
              n_intervals + 1};
    o[0] = qtab_value(&T, x);
    o[1] = qtab_d1(&T, x);
    o[2] = qtab_d2(&T, x);
}

/* ------------------------------------------------------------------------------------ */
/* system state                                                                          */

typedef struct {
    double T;
    int n;
    double *q, *p_eta, *eta;
    double Nf;
} chain_t; /* src/thermostat.hpp:9-38 */

struct orc_system {
    int N, ntypes, npot, has_eam;
    /* tables: pair slot k (potential.hpp:77-104), EAM per type (eam.hpp:10-71) */
    double pot_rcut, pot_rmin_fatal, eam_rcut, rhomax_fatal;
    qtab *pot, *trho, *tF;
    double *mass;
    unsigned *type;
    /* per atom, xyz interleaved */
    double *pos, *crd, *vel, *frc, *rho, *Fe, *dF, *d2F, *g, *hv, *hsq, *epot, *ekin;
    /* neighbour list (md_driver.hpp:87-90) */
    int neighbors;
    double r_skin, r_cut_sq, r_cutr_skin_sq;
    int *point, *nbr;
    long nbr_cap;
    /* integrator */
    int ensemble, coupling;
    double Nf, alpha, dt, time, fatal_conservation;
    unsigned long long cycle;
    chain_t th;
    double baro_P, baro_w, baro_eps, baro_peps;
    chain_t bth;
    double h[9], h0[9];
    /* observables */
    double epot_eam_atom, epot_atom, ekin_atom, etot_atom, ekin_tot, etot_cons_initial,
        etot_cons, etot_cons_err, virial, total_laplacian, total_force2, temperature_kin,
        temperature_conf_inverse, pressure;
    double born_stress[6], stress[6], born_el[36], mom[3];
    int sample;
    unsigned status;
    /* g(r) */
    int n_rg;
    double *rg, *gr, *grp, drg, rmaxg;
    unsigned *n_per_type;
};

/* md_driver.hpp:48-50 */
static double nint_ref(double x) {
    return (double)(x < 0. ? (int)(x - 0.5) : (int)(x + 0.5));
}

static double volume(double const *h) {
    /* 3x3 determinant, first-row expansion; for the diagonal box h00*(h11*h22) */
    return h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
           h[2] * (h[3] * h[7] - h[4] * h[6]);
}

/* md_driver.cpp:175-185: p = apply_bc(ci - cj) * diag(h) */
static void min_image(orc_system const *s, double const *ci, double const *cj, double *p) {
    double d[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
    d[0] = d[0] - nint_ref(d[0]);
    d[1] = d[1] - nint_ref(d[1]);
    d[2] = d[2] - nint_ref(d[2]);
    p[0] = d[0] * s->h[0];
    p[1] = d[1] * s->h[4];
    p[2] = d[2] * s->h[8];
}

static double len2(double const *p) { return p[0] * p[0] + p[1] * p[1] + p[2] * p[2]; }

/* eam.hpp:30-46 */
static double eam_rho(orc_system const *s, unsigned t, double dr) {
    return dr > s->eam_rcut ? 0. : qtab_value(&s->trho[t], dr);
}
static double eam_drho(orc_system const *s, unsigned t, double dr) {
    return dr > s->eam_rcut ? 0. : qtab_d1(&s->trho[t], dr);
}
static double eam_d2rho(orc_system const *s, unsigned t, double dr) {
    return dr > s->eam_rcut ? 0. : qtab_d2(&s->trho[t], dr);
}
/* eam.hpp:48-70: the reference exits when rho > rhomax_fatal */
static double eam_F(orc_system *s, unsigned t, double r, int k) {
    if (r > s->rhomax_fatal)
        s->status |= ORC_FATAL_RHO_MAX;
    return k == 0 ? qtab_value(&s->tF[t], r) : k == 1 ? qtab_d1(&s->tF[t], r)
                                                       : qtab_d2(&s->tF[t], r);
}

static void nbr_range(orc_system const *s, int i, int *start, int *end) {
    /* md_driver.cpp:187-193 */
    if (s->neighbors) {
        *start = s->point[i];
        *end = s->point[i + 1];
    } else {
        *start = i + 1;
        *end = s->N;
    }
}

/* md_driver.cpp:279-298: O(N^2) half list j > i, |p|^2 <= (rcut r_skin)^2 */
void orc_calculate_neighbors(orc_system *s) {
    long k = 0;
    for (int i = 0; i < s->N; ++i) {
        double const *ci = s->crd + 3 * i;
        s->point[i] = (int)k;
        for (int j = i + 1; j < s->N; ++j) {
            double p[3];
            min_image(s, ci, s->crd + 3 * j, p);
            if (len2(p) > s->r_cutr_skin_sq)
                continue;
            if (k >= s->nbr_cap) {
                s->nbr_cap *= 2;
                s->nbr = (int *)realloc(s->nbr, sizeof(int) * (size_t)s->nbr_cap);
            }
            s->nbr[k] = j;
            k += 1;
        }
    }
    s->point[s->N] = (int)k;
}

/* md_driver.cpp:195-277: densities rho_i, helpers g_i h_i, embedding F F' F'' */
static void calculate_eam(orc_system *s) {
    if (!s->has_eam)
        return;
    int const obs = s->sample;
    int const N = s->N;
    memset(s->rho, 0, sizeof(double) * (size_t)N);
    if (obs) {
        memset(s->hv, 0, sizeof(double) * 3 * (size_t)N);
        memset(s->g, 0, sizeof(double) * 6 * (size_t)N);
    }
    for (int i = 0; i < N; ++i) {
        double const *ci = s->crd + 3 * i;
        unsigned const ti = s->type[i];
        int start, end;
        nbr_range(s, i, &start, &end);
        for (int k = start; k < end; ++k) {
            int const j = s->neighbors ? s->nbr[k] : k;
            unsigned const tj = s->type[j];
            double p[3];
            min_image(s, ci, s->crd + 3 * j, p);
            double const r2 = len2(p);
            if (r2 > s->r_cut_sq)
                continue;
            double const dr = sqrt(r2);
            double const rho_ij = eam_rho(s, tj, dr);
            double const rho_ji = eam_rho(s, ti, dr);
            s->rho[i] += rho_ij;
            s->rho[j] += rho_ji;
            if (!obs)
                continue;
            double const a_ij = eam_drho(s, tj, dr) / dr;
            double const a_ji = eam_drho(s, ti, dr) / dr;
            for (int iv = 0; iv < 6; ++iv) {
                s->g[6 * i + iv] += a_ij * p[VA[iv]] * p[VB[iv]];
                s->g[6 * j + iv] += a_ji * p[VA[iv]] * p[VB[iv]];
            }
            for (int c = 0; c < 3; ++c)
                s->hv[3 * i + c] += a_ij * p[c];
            for (int c = 0; c < 3; ++c)
                s->hv[3 * j + c] -= a_ji * p[c];
        }
    }
    for (int i = 0; i < N; ++i) {
        double const r = s->rho[i];
        unsigned const ti = s->type[i];
        s->Fe[i] = eam_F(s, ti, r, 0);
        s->dF[i] = eam_F(s, ti, r, 1);
        if (obs) {
            s->d2F[i] = eam_F(s, ti, r, 2);
            s->hsq[i] = len2(s->hv + 3 * i);
        }
    }
}

/* md_driver.cpp:300-430: forces, energies, virial, Born stress; on sampled steps the
 * Born elasticity tensor and the configurational-temperature Laplacian */
void orc_calculate_forces(orc_system *s) {
    calculate_eam(s);
    int const obs = s->sample;
    int const N = s->N;
    memset(s->frc, 0, sizeof(double) * 3 * (size_t)N);
    memset(s->epot, 0, sizeof(double) * (size_t)N);
    s->virial = 0.;
    for (int k = 0; k < 6; ++k)
        s->born_stress[k] = 0.;
    if (obs) {
        for (int k = 0; k < 36; ++k)
            s->born_el[k] = 0.;
        s->total_laplacian = 0.;
    }
    for (int i = 0; i < N; ++i) {
        double *fi = s->frc + 3 * i;
        double const *ci = s->crd + 3 * i;
        double const dF_i = s->dF[i];
        double const d2F_i = s->d2F[i];
        unsigned const ti = s->type[i];
        s->epot[i] += s->Fe[i];
        int start, end;
        nbr_range(s, i, &start, &end);
        for (int k = start; k < end; ++k) {
            int const j = s->neighbors ? s->nbr[k] : k;
            unsigned const tj = s->type[j];
            double p[3];
            min_image(s, ci, s->crd + 3 * j, p);
            double const r2 = len2(p);
            if (r2 > s->r_cut_sq)
                continue;
            unsigned const tmax = ti > tj ? ti : tj, tmin = ti < tj ? ti : tj;
            unsigned const slot = tmax * (tmax + 1) / 2 + tmin;
            double const dr = sqrt(r2);
            /* TablePotential::calculate, potential.hpp:92-104 */
            double V = 0., dV = 0., d2V = 0.;
            if (dr < s->pot_rmin_fatal)
                s->status |= ORC_WARN_RMIN;
            if (!(dr > s->pot_rcut)) {
                V = qtab_value(&s->pot[slot], dr);
                dV = qtab_d1(&s->pot[slot], dr);
                d2V = qtab_d2(&s->pot[slot], dr);
            }
            double dedr = dV;
            double X = 0.;
            if (obs) {
                X = d2V - dV / dr;
                s->total_laplacian += 2. * (d2V + 2. * dV / dr);
            }
            if (s->has_eam) {
                double const drho_i = eam_drho(s, ti, dr);
                double const drho_j = eam_drho(s, tj, dr);
                double const dF_j = s->dF[j];
                dedr += dF_i * drho_j + dF_j * drho_i;
                if (obs) {
                    double const d2rho_i = eam_d2rho(s, ti, dr);
                    double const d2rho_j = eam_d2rho(s, tj, dr);
                    s->total_laplacian += 2. * (dF_j * (d2rho_i + 2. * drho_i / dr) +
                                                dF_i * (d2rho_j + 2. * drho_j / dr));
                    s->total_laplacian += d2F_i * (drho_j * drho_j) + s->d2F[j] * (drho_i * drho_i);
                    X += dF_i * (d2rho_j - drho_j / dr) + dF_j * (d2rho_i - drho_i / dr);
                }
            }
            X /= (dr * dr);
            double const sc = -dedr / dr;
            double const df[3] = {sc * p[0], sc * p[1], sc * p[2]};
            fi[0] += df[0];
            fi[1] += df[1];
            fi[2] += df[2];
            s->frc[3 * j] -= df[0];
            s->frc[3 * j + 1] -= df[1];
            s->frc[3 * j + 2] -= df[2];
            s->epot[i] += 0.5 * V;
            s->epot[j] += 0.5 * V;
            s->virial += dr * dedr;
            for (int iv = 0; iv < 6; ++iv) {
                double const num = p[VA[iv]] * p[VB[iv]];
                s->born_stress[iv] += dedr * num / dr;
                if (!obs)
                    continue;
                for (int ivp = iv; ivp < 6; ++ivp) {
                    double const num2 = num * p[VA[ivp]] * p[VB[ivp]];
                    s->born_el[6 * iv + ivp] += num2 * X;
                }
            }
        }
        if (s->has_eam && obs) {
            double const *gi = s->g + 6 * i;
            for (int iv = 0; iv < 6; ++iv)
                for (int ivp = iv; ivp < 6; ++ivp)
                    s->born_el[6 * iv + ivp] += d2F_i * gi[iv] * gi[ivp];
            s->total_laplacian += d2F_i * s->hsq[i];
        }
    }
    s->virial /= -3.;
    double const vir_trace = -(s->born_stress[0] + s->born_stress[1] + s->born_stress[2]);
    if (fabs(s->virial / (vir_trace / 3.) - 1.) > 1e-7)
        s->status |= ORC_WARN_VIRIAL;
}

/* numerics.hpp:11-18 */
static void expx_operator(double x, double *expx, double *op) {
    static const double c1 = -1.0 / 2.0, c2 = 1.0 / 6.0, c3 = -1.0 / 24.0, c4 = 1. / 120.,
                        c5 = -1. / 720.;
    double const e = exp(-x);
    *expx = e;
    *op = fabs(x) > 1e-3 ? (1.0 - e) / x
                         : 1.0 + x * (c1 + x * (c2 + x * (c3 + x * (c4 + x * c5))));
}

/* md_driver.cpp:603-609 */
static void set_kinetic_energies(orc_system *s) {
    for (int i = 0; i < s->N; ++i)
        s->ekin[i] = 0.5 * s->mass[s->type[i]] * len2(s->vel + 3 * i);
    double acc = 0.;
    for (int i = 0; i < s->N; ++i)
        acc = acc + s->ekin[i];
    s->ekin_tot = acc;
    s->ekin_atom = s->ekin_tot / s->N;
}

/* md_driver.cpp:630-646 */
static void calculate_tconf(orc_system *s) {
    if (!s->sample)
        return;
    s->total_force2 = 0.;
    for (int i = 0; i < s->N; ++i)
        s->total_force2 += len2(s->frc + 3 * i);
    if (s->total_force2 != 0. && s->total_laplacian != 0.)
        s->temperature_conf_inverse = K_BOLTZ * s->total_laplacian / s->total_force2;
    else
        s->temperature_conf_inverse = 0.;
}

/* md_driver.cpp:433-452 */
static void U2(orc_system *s, double dt) {
    double c = 1., e = 1.;
    if (s->ensemble == 2) {
        double const x = s->alpha * dt * s->baro_peps / s->baro_w;
        expx_operator(x, &e, &c);
    }
    double const cdt = c * dt;
    for (int i = 0; i < s->N; ++i) {
        double const m = s->mass[s->type[i]];
        double *v = s->vel + 3 * i;
        double const *f = s->frc + 3 * i;
        for (int a = 0; a < 3; ++a)
            v[a] = v[a] * e + cdt * f[a] / m;
    }
    set_kinetic_energies(s);
    calculate_tconf(s);
}

/* md_driver.cpp:454-459 (Yu et al., Chem. Phys. 370 (2010) 294, eq. 31) */
static void U2p(orc_system *s, double dt) {
    double const pv = s->baro_P * volume(s->h);
    s->baro_peps += (2. * s->alpha * s->ekin_tot + 3. * s->virial - 3. * pv) * dt;
}

/* md_driver.cpp:462-499 */
static void U1(orc_system *s, double dt) {
    double cf = 1.;
    if (s->ensemble == 2) {
        double const x = dt * s->baro_peps / s->baro_w;
        s->baro_eps += x;
        double e;
        expx_operator(x, &e, &cf);
    }
    double const a = cf * dt;
    for (int i = 0; i < s->N; ++i) {
        double *c = s->crd + 3 * i;
        double const *v = s->vel + 3 * i;
        double dc[3] = {a * v[0], a * v[1], a * v[2]};
        dc[0] /= s->h[0];
        dc[1] /= s->h[4];
        dc[2] /= s->h[8];
        c[0] += dc[0];
        c[1] += dc[1];
        c[2] += dc[2];
        double d[3] = {c[0] - nint_ref(c[0]), c[1] - nint_ref(c[1]), c[2] - nint_ref(c[2])};
        s->pos[3 * i] = d[0] * s->h[0];
        s->pos[3 * i + 1] = d[1] * s->h[4];
        s->pos[3 * i + 2] = d[2] * s->h[8];
    }
    if (s->ensemble == 2) {
        double const expe = exp(s->baro_eps);
        double const vol_old = volume(s->h);
        for (int k = 0; k < 9; ++k)
            s->h[k] = s->h0[k] * expe;
        if (fabs(volume(s->h) / vol_old - 1.) > 0.05)
            s->status |= ORC_FATAL_VOLUME;
    }
}

/* thermostat.cpp:40-66 (Yu et al. eq. 8; Allen-Tildesley eqs. 3.73-3.74a) */
static void U4_chain(chain_t *t, double dt, double e_couple, int outward) {
    int const dj = outward ? 1 : -1;
    int const j_first = outward ? 0 : t->n - 1;
    int const j_last = outward ? t->n : -1;
    double const kT = K_BOLTZ * t->T;
    int const j_end = t->n - 1;
    for (int j = j_first; j != j_last; j += dj) {
        double const G = j != 0 ? t->p_eta[j - 1] * t->p_eta[j - 1] / t->q[j - 1] - kT
                                : 2. * e_couple - t->Nf * kT;
        if (j != j_end) {
            double const x = dt * t->p_eta[j + 1] / t->q[j + 1];
            double e, op;
            expx_operator(x, &e, &op);
            t->p_eta[j] = t->p_eta[j] * e + dt * G * op;
        } else {
            t->p_eta[j] += dt * G;
        }
    }
}

/* thermostat.hpp:24-35: the factor for the coupled momenta, and the chain positions */
static double U3_chain(chain_t *t, double dt) {
    double const scale = exp(-dt * t->p_eta[0] / t->q[0]);
    for (int j = 0; j < t->n; ++j)
        t->eta[j] += dt * t->p_eta[j] / t->q[j];
    return scale;
}

/* thermostat.cpp:24-37 */
static double chain_etot(chain_t const *t) {
    double e = t->Nf * t->eta[0];
    for (int j = 1; j < t->n; ++j)
        e += t->eta[j];
    e *= K_BOLTZ * t->T;
    for (int j = 0; j < t->n; ++j)
        e += 0.5 * (t->p_eta[j] * t->p_eta[j]) / t->q[j];
    return e;
}

/* md_driver.cpp:512-531 */
static void U4_thermo(orc_system *s, double dt, int outward) {
    double e_couple = s->ekin_tot;
    if (s->coupling != 0 && s->temperature_conf_inverse != 0.) {
        double const econf = (K_BOLTZ / s->temperature_conf_inverse) * s->Nf / 2.;
        e_couple = s->coupling == 1 ? econf : 0.5 * (s->ekin_tot + econf);
    }
    U4_chain(&s->th, dt, e_couple, outward);
}

/* md_driver.cpp:539-549 */
static void U_NHC_thermo(orc_system *s, double dt) {
    for (int k = 0; k < 7; ++k) {
        double const dtw = WSY7[k] * dt;
        U4_thermo(s, 0.5 * dtw, 0);
        double const sc = U3_chain(&s->th, dtw);
        for (int i = 0; i < 3 * s->N; ++i)
            s->vel[i] *= sc;
        set_kinetic_energies(s);
        U4_thermo(s, 0.5 * dtw, 1);
    }
}

/* md_driver.cpp:551-561, 533-537, 507-510 */
static void U_NHC_baro(orc_system *s, double dt) {
    for (int k = 0; k < 7; ++k) {
        double const dtw = WSY7[k] * dt;
        U4_chain(&s->bth, 0.5 * dtw, 0.5 * (s->baro_peps * s->baro_peps) / s->baro_w, 0);
        s->baro_peps *= U3_chain(&s->bth, dtw);
        U4_chain(&s->bth, 0.5 * dtw, 0.5 * (s->baro_peps * s->baro_peps) / s->baro_w, 1);
    }
}

/* md_driver.cpp:611-628 */
static void set_momentum_tot(orc_system *s) {
    s->mom[0] = s->mom[1] = s->mom[2] = 0.;
    for (int i = 0; i < s->N; ++i) {
        double const m = s->mass[s->type[i]];
        for (int a = 0; a < 3; ++a)
            s->mom[a] += s->vel[3 * i + a] * m;
    }
    double const scale2 = 2. * s->mass[0] * s->ekin_tot;
    if (len2(s->mom) / scale2 > 1e-14)
        s->status |= ORC_FATAL_MOMENTUM;
}

/* md_driver.cpp:648-730 */
static void calculate_thermodynamics(orc_system *s) {
    set_momentum_tot(s);
    double acc = 0.;
    for (int i = 0; i < s->N; ++i)
        acc = acc + s->epot[i];
    s->epot_atom = acc / s->N;
    acc = 0.;
    for (int i = 0; i < s->N; ++i)
        acc = acc + s->Fe[i];
    s->epot_eam_atom = acc / s->N;
    s->etot_atom = s->ekin_atom + s->epot_atom;
    double const old = s->etot_cons;
    s->etot_cons = s->etot_atom * s->N;
    if (s->ensemble == 1 || s->ensemble == 2)
        s->etot_cons += chain_etot(&s->th);
    if (s->ensemble == 2)
        s->etot_cons += volume(s->h) * s->baro_P +
                        (0.5 * (s->baro_peps * s->baro_peps) / s->baro_w + chain_etot(&s->bth));
    s->etot_cons_err = fabs(s->etot_cons / s->etot_cons_initial - 1.);
    double const err_current = fabs(s->etot_cons / old - 1.);
    s->temperature_kin = 2. * s->ekin_tot / (K_BOLTZ * s->Nf);
    calculate_tconf(s);
    double const V = volume(s->h);
    s->pressure = (s->ekin_tot * 2. / 3. + s->virial) / V;
    for (int iv = 0; iv < 6; ++iv)
        s->stress[iv] = -s->born_stress[iv];
    for (int i = 0; i < s->N; ++i) {
        double const *v = s->vel + 3 * i;
        double const m = s->mass[s->type[i]];
        for (int iv = 0; iv < 6; ++iv)
            s->stress[iv] += m * v[VA[iv]] * v[VB[iv]];
    }
    for (int iv = 0; iv < 6; ++iv) {
        s->stress[iv] /= V;
        s->born_stress[iv] /= V;
    }
    if (s->sample)
        for (int k = 0; k < 36; ++k)
            s->born_el[k] /= V;
    double const p_trace = s->stress[0] + s->stress[1] + s->stress[2];
    if (fabs(s->pressure / (p_trace / 3.) - 1.) > 1e-5)
        s->status |= ORC_FATAL_PRESSURE;
    if ((s->etot_cons_err > s->fatal_conservation || err_current > s->fatal_conservation) &&
        s->cycle > 0)
        s->status |= ORC_FATAL_CONSERVATION;
}

/* md_driver.cpp:563-601 */
void orc_integrate(orc_system *s, int n_steps) {
    double const dt = s->dt;
    for (int step = 0; step < n_steps; ++step) {
        if (s->ensemble == 2)
            U_NHC_baro(s, 0.5 * dt);
        if (s->ensemble == 1 || s->ensemble == 2)
            U_NHC_thermo(s, 0.5 * dt);
        if (s->ensemble == 2)
            U2p(s, 0.5 * dt);
        U2(s, 0.5 * dt);
        U1(s, dt);
        orc_calculate_forces(s);
        U2(s, 0.5 * dt);
        if (s->ensemble == 2)
            U2p(s, 0.5 * dt);
        if (s->ensemble == 1 || s->ensemble == 2)
            U_NHC_thermo(s, 0.5 * dt);
        if (s->ensemble == 2)
            U_NHC_baro(s, 0.5 * dt);
        calculate_thermodynamics(s);
        s->time += dt;
        ++s->cycle;
    }
}

/* ------------------------------------------------------------------------------------ */
/* construction: md_driver.cpp:16-160                                                     */

static double *dup(double const *p, long n) {
    double *o = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (n > 0)
        memcpy(o, p, sizeof(double) * (size_t)n);
    return o;
}

static void chain_init(chain_t *t, double T, int n, double const *q, double const *p_eta,
                       double Nf) {
    t->T = T;
    t->n = n;
    t->q = dup(q, n);
    t->p_eta = dup(p_eta, n);
    t->eta = (double *)calloc((size_t)n, sizeof(double));
    t->Nf = Nf;
}

orc_system *orc_create(int n_types, char const *interpolation, double rcut, double rmin_fatal,
                       double dr, int n_r, double const *phi, double const *dphi,
                       double const *d2phi, int has_eam, double eam_rcut, double rhomax_fatal,
                       double drho, int n_rho, double const *rho, double const *drho_dr,
                       double const *d2rho_dr2, double const *F, double const *dF,
                       double const *d2F, int n_atoms, double const *pos, double const *vel,
                       unsigned const *types, double const *mass, int ensemble, int coupling,
                       double T, int nchain, double const *q, double const *p_eta,
                       double Nf_th, double P, double w, double p_eps, double Tb,
                       int nchain_b, double const *qb, double const *p_eta_b, double Nf_b,
                       double const *box9, int n_rg, double const *rg, double Nf, double dt,
                       int neighbors, double r_skin, double fatal_conservation) {
    int const bspline = strcmp(interpolation, "bspline") == 0;
    if (!bspline && strcmp(interpolation, "quintic") != 0)
        return NULL;
    orc_system *s = (orc_system *)calloc(1, sizeof(orc_system));
    int const N = n_atoms;
    s->N = N;
    s->ntypes = n_types;
    s->npot = n_types * (n_types + 1) / 2;
    s->has_eam = has_eam;
    s->pot_rcut = rcut;
    s->pot_rmin_fatal = rmin_fatal;
    s->eam_rcut = eam_rcut;
    s->rhomax_fatal = rhomax_fatal;
    s->pot = (qtab *)calloc((size_t)s->npot, sizeof(qtab));
    for (int k = 0; k < s->npot; ++k)
        qtab_init(&s->pot[k], dr, n_r, phi + (long)k * n_r, dphi + (long)k * n_r,
                  d2phi + (long)k * n_r, bspline);
    s->trho = (qtab *)calloc((size_t)n_types, sizeof(qtab));
    s->tF = (qtab *)calloc((size_t)n_types, sizeof(qtab));
    if (has_eam) {
        for (int t = 0; t < n_types; ++t) {
            qtab_init(&s->trho[t], dr, n_r, rho + (long)t * n_r, drho_dr + (long)t * n_r,
                      d2rho_dr2 + (long)t * n_r, bspline);
            qtab_init(&s->tF[t], drho, n_rho, F + (long)t * n_rho, dF + (long)t * n_rho,
                      d2F + (long)t * n_rho, bspline);
        }
    }
    s->mass = dup(mass, n_types);
    s->type = (unsigned *)malloc(sizeof(unsigned) * (size_t)N);
    memcpy(s->type, types, sizeof(unsigned) * (size_t)N);
    s->pos = dup(pos, 3L * N);
    s->vel = dup(vel, 3L * N);
    s->crd = (double *)calloc(3 * (size_t)N, sizeof(double));
    s->frc = (double *)calloc(3 * (size_t)N, sizeof(double));
    s->rho = (double *)calloc((size_t)N, sizeof(double));
    s->Fe = (double *)calloc((size_t)N, sizeof(double));
    s->dF = (double *)calloc((size_t)N, sizeof(double));
    s->d2F = (double *)calloc((size_t)N, sizeof(double));
    s->g = (double *)calloc(6 * (size_t)N, sizeof(double));
    s->hv = (double *)calloc(3 * (size_t)N, sizeof(double));
    s->hsq = (double *)calloc((size_t)N, sizeof(double));
    s->epot = (double *)calloc((size_t)N, sizeof(double));
    s->ekin = (double *)calloc((size_t)N, sizeof(double));
    s->neighbors = neighbors;
    s->r_skin = r_skin;
    s->r_cut_sq = rcut * rcut;
    s->r_cutr_skin_sq = (rcut * r_skin) * (rcut * r_skin);
    s->point = (int *)calloc((size_t)N + 1, sizeof(int));
    s->nbr_cap = 40L * N > 0 ? 40L * N : 1;
    s->nbr = (int *)calloc((size_t)s->nbr_cap, sizeof(int));
    s->ensemble = ensemble;
    s->coupling = coupling;
    s->Nf = Nf;
    s->alpha = 1. + 3. / Nf;
    s->dt = dt;
    s->fatal_conservation = fatal_conservation;
    chain_init(&s->th, T, nchain, q, p_eta, Nf_th);
    s->baro_P = P;
    s->baro_w = w;
    s->baro_eps = 0.;
    s->baro_peps = p_eps;
    chain_init(&s->bth, Tb, nchain_b, qb, p_eta_b, Nf_b);
    memcpy(s->h, box9, sizeof(double) * 9);
    memcpy(s->h0, box9, sizeof(double) * 9);
    s->sample = 1;
    s->n_rg = n_rg;
    s->rg = dup(rg, n_rg);
    s->gr = (double *)calloc((size_t)n_rg, sizeof(double));
    s->grp = (double *)calloc((size_t)s->npot * (size_t)n_rg, sizeof(double));
    s->drg = rg[1] - rg[0];
    s->rmaxg = rg[n_rg - 1] + 0.5 * (rg[1] - rg[0]);
    s->n_per_type = (unsigned *)calloc((size_t)n_types, sizeof(unsigned));
    /* md_driver.cpp:91-106: scaled coordinates c = apply_bc(p / diag(h)) */
    for (int i = 0; i < N; ++i) {
        double const *p = pos + 3 * i;
        double u[3] = {p[0] / s->h[0], p[1] / s->h[4], p[2] / s->h[8]};
        for (int a = 0; a < 3; ++a)
            s->crd[3 * i + a] = u[a] - nint_ref(u[a]);
        if (types[i] < (unsigned)n_types)
            s->n_per_type[types[i]] += 1;
    }
    /* md_driver.cpp:112-118 */
    if (neighbors)
        orc_calculate_neighbors(s);
    orc_calculate_forces(s);
    set_kinetic_energies(s);
    calculate_thermodynamics(s);
    s->etot_cons_initial = s->etot_cons;
    return s;
}

static void chain_free(chain_t *t) {
    free(t->q);
    free(t->p_eta);
    free(t->eta);
}

void orc_destroy(orc_system *s) {
    if (!s)
        return;
    for (int k = 0; k < s->npot; ++k)
        qtab_free(&s->pot[k]);
    for (int t = 0; t < s->ntypes; ++t) {
        qtab_free(&s->trho[t]);
        qtab_free(&s->tF[t]);
    }
    free(s->pot);
    free(s->trho);
    free(s->tF);
    double *arrs[] = {s->mass, s->pos, s->vel, s->crd, s->frc, s->rho, s->Fe, s->dF, s->d2F,
                      s->g, s->hv, s->hsq, s->epot, s->ekin, s->rg, s->gr, s->grp};
    for (size_t k = 0; k < sizeof(arrs) / sizeof(arrs[0]); ++k)
        free(arrs[k]);
    free(s->type);
    free(s->point);
    free(s->nbr);
    free(s->n_per_type);
    chain_free(&s->th);
    chain_free(&s->bth);
    free(s);
}

void orc_set_sample_observables(orc_system *s, int flag) { s->sample = flag != 0; }
unsigned orc_status(orc_system const *s) { return s->status; }

void orc_scalars(orc_system const *s, double *o) {
    double const v[16] = {s->epot_eam_atom, s->epot_atom, s->ekin_atom, s->etot_atom,
                          s->ekin_tot, s->etot_cons_initial, s->etot_cons, s->etot_cons_err,
                          s->virial, s->total_laplacian, s->total_force2, s->temperature_kin,
                          s->temperature_conf_inverse, s->pressure, s->time, (double)s->cycle};
    memcpy(o, v, sizeof(v));
    memcpy(o + 16, s->born_stress, sizeof(double) * 6);
    memcpy(o + 22, s->stress, sizeof(double) * 6);
    memcpy(o + 28, s->born_el, sizeof(double) * 36);
    memcpy(o + 64, s->h, sizeof(double) * 9);
    o[73] = s->baro_eps;
    o[74] = s->baro_peps;
    memcpy(o + 75, s->mom, sizeof(double) * 3);
}

void orc_atoms(orc_system const *s, int which, double *o) {
    double const *src3[4] = {s->pos, s->crd, s->vel, s->frc};
    double const *src1[6] = {s->rho, s->epot, s->ekin, s->Fe, s->dF, s->d2F};
    if (which >= 0 && which < 4)
        memcpy(o, src3[which], sizeof(double) * 3 * (size_t)s->N);
    else if (which >= 4 && which < 10)
        memcpy(o, src1[which - 4], sizeof(double) * (size_t)s->N);
}

int orc_chain(orc_system const *s, int which, double *p_eta, double *eta) {
    chain_t const *t = which == 0 ? &s->th : &s->bth;
    memcpy(p_eta, t->p_eta, sizeof(double) * (size_t)t->n);
    memcpy(eta, t->eta, sizeof(double) * (size_t)t->n);
    return t->n;
}

long orc_neighbors(orc_system const *s, int *point, int *neighbors, long cap) {
    if (!s->neighbors)
        return -1;
    memcpy(point, s->point, sizeof(int) * ((size_t)s->N + 1));
    long const total = s->point[s->N];
    long const n = total < cap ? total : cap;
    memcpy(neighbors, s->nbr, sizeof(int) * (size_t)n);
    return total;
}

/* md_driver.cpp:732-862 */
void orc_pair_correlation(orc_system *s, int mode) {
    int const total = mode == 0 || mode == 1, partial = mode == 1 || mode == 2;
    int const N = s->N, nrg = s->n_rg;
    if (total)
        memset(s->gr, 0, sizeof(double) * (size_t)nrg);
    if (partial)
        memset(s->grp, 0, sizeof(double) * (size_t)s->npot * (size_t)nrg);
    for (int i = 0; i < N; ++i) {
        double const *ci = s->crd + 3 * i;
        for (int j = i + 1; j < N; ++j) {
            double p[3];
            min_image(s, ci, s->crd + 3 * j, p);
            double const dr = sqrt(len2(p));
            if (dr < s->rmaxg) {
                int const k = (int)floor(dr / s->drg);
                if (total)
                    s->gr[k] += 1.;
                if (partial) {
                    unsigned const ti = s->type[i], tj = s->type[j];
                    unsigned const tmax = ti > tj ? ti : tj, tmin = ti < tj ? ti : tj;
                    s->grp[(long)(tmax * (tmax + 1) / 2 + tmin) * nrg + k] += 1.;
                }
            }
        }
    }
    double const V = volume(s->h);
    if (total)
        for (int k = 0; k < nrg; ++k)
            s->gr[k] *= V / (2. * M_PI * N * N * s->rg[k] * s->rg[k] * s->drg);
    if (partial) {
        int slot = 0;
        for (int b = 0; b < s->ntypes; ++b) {
            for (int a = 0; a <= b; ++a) {
                double const Na = (double)s->n_per_type[a], Nb = (double)s->n_per_type[b];
                double pc = 0.;
                if (a == b) {
                    if (Na > 1)
                        pc = Na * (Na - 1.) / 2.;
                } else {
                    pc = Na * Nb;
                }
                double *g = s->grp + (long)slot * nrg;
                if (pc > 0.) {
                    double const pref = V / (4. * M_PI * pc * s->drg);
                    for (int k = 0; k < nrg; ++k)
                        g[k] *= pref / (s->rg[k] * s->rg[k]);
                } else {
                    memset(g, 0, sizeof(double) * (size_t)nrg);
                }
                slot += 1;
            }
        }
    }
}

void orc_gr(orc_system const *s, double *gr, double *gr_partial) {
    memcpy(gr, s->gr, sizeof(double) * (size_t)s->n_rg);
    memcpy(gr_partial, s->grp, sizeof(double) * (size_t)s->npot * (size_t)s->n_rg);
}
