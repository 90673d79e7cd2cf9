/* CPU restatement of mdelast's EAM force-and-stress step (the test oracle).
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, the smoke check and the CPU-baseline leg of
 * bench.py load this library, and only as a checker; the product path never does.
 *
 * Each function states the reference file:line it restates. Arithmetic follows the
 * reference's operation order in IEEE double without FMA contraction (built with
 * -ffp-contract=off), so on x86-64 it reproduces the reference build bit for bit.
 * Fatal conditions the reference ends the process on (exit(1)) set a bit in
 * orc_status() instead.
 */
#ifndef MDELAST_ORACLE_H_
#define MDELAST_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_system orc_system;

/* Argument list identical to mref_create of oracle/ref_capi.cpp (which follows the
 * md_driver_module constructor, md_driver_module.cpp:95-102). interpolation must be
 * "quintic". */
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
                       int neighbors, double r_skin, double fatal_conservation);
void orc_destroy(orc_system *s);

void orc_integrate(orc_system *s, int n_steps);
void orc_calculate_neighbors(orc_system *s);
void orc_calculate_forces(orc_system *s);
void orc_set_sample_observables(orc_system *s, int flag);
unsigned orc_status(orc_system const *s);

/* Readouts in the layouts of oracle/ref_capi.cpp (mref_scalars, mref_atoms, ...). */
void orc_scalars(orc_system const *s, double *out78);
void orc_atoms(orc_system const *s, int which, double *out);
int orc_chain(orc_system const *s, int which, double *p_eta, double *eta);
long orc_neighbors(orc_system const *s, int *point, int *neighbors, long cap);
void orc_pair_correlation(orc_system *s, int mode);
void orc_gr(orc_system const *s, double *gr, double *gr_partial);

/* Stand-alone quintic table (poly_table.hpp:33-115): coefficients of n_nodes - 1
 * intervals, 6 per interval, built in long double. */
int orc_quintic_coefficients(double h, int n_nodes, double const *f, double const *f1,
                             double const *f2, double *coef_out);
double orc_bspline_value(double h, int n, double const *f, double x);
void orc_quintic_eval(double const *coef, int n_intervals, double h, double x, double *out3);

/* status bits, the same meaning as the MDELAST_STATUS_* bits of include/mdelast.h */
#define ORC_FATAL_RHO_MAX 0x1u
#define ORC_FATAL_VOLUME 0x2u
#define ORC_FATAL_MOMENTUM 0x4u
#define ORC_FATAL_PRESSURE 0x8u
#define ORC_FATAL_CONSERVATION 0x10u
#define ORC_WARN_VIRIAL 0x100u
#define ORC_WARN_RMIN 0x200u

#ifdef __cplusplus
}
#endif
#endif
