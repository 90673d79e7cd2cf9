/* mdelast B200 path: C-ABI of libmdelast_cuda.so.
 *
 * This is the boundary that replaces the C++ force-and-integrator core behind mdelast's
 * pybind11 module md_driver_module (src/md_driver_module.cpp:16-224). Every entry point
 * takes plain pointers and sizes, returns an int status (MDELAST_OK or a negative
 * MDELAST_ERR_*), and reports details through mdelast_last_error(). Quantities crossing
 * this boundary are in the reference's CGS units (src/units.hpp:6-24): cm, g, s, erg,
 * dyn, erg/cm^3; Voigt order xx yy zz yz xz xy (src/md_driver.hpp:23-24).
 *
 * The compute path runs on the GPU (sm_100a). A call that needs the GPU fails with
 * MDELAST_ERR_NO_DEVICE when no CUDA device is usable; there is no CPU fallback.
 */
#ifndef MDELAST_H_
#define MDELAST_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDELAST_ABI_VERSION 1

/* return codes */
#define MDELAST_OK 0
#define MDELAST_ERR_ARGUMENT (-1)    /* invalid argument: message in mdelast_last_error() */
#define MDELAST_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define MDELAST_ERR_NO_DEVICE (-3)   /* no usable CUDA device */
#define MDELAST_ERR_FATAL (-4)       /* a physics check the reference ends the run on */
#define MDELAST_ERR_UNSUPPORTED (-5) /* valid in the reference but not on this path */
#define MDELAST_ERR_CAPACITY (-6)    /* a fixed capacity (neighbour slots, cell size) hit */

/* Status bits of a driver (mdelast_observables.status). FATAL bits correspond to the
 * reference's printf + exit(1) sites; WARN bits to its print-only sites. */
#define MDELAST_FATAL_RHO_MAX 0x1u       /* eam.hpp:48-70: rho > rhomax_fatal */
#define MDELAST_FATAL_VOLUME 0x2u        /* md_driver.cpp:493-497: volume jump > 5 % */
#define MDELAST_FATAL_MOMENTUM 0x4u      /* md_driver.cpp:623-627 */
#define MDELAST_FATAL_PRESSURE 0x8u      /* md_driver.cpp:693-698 */
#define MDELAST_FATAL_CONSERVATION 0x10u /* md_driver.cpp:700-726 */
#define MDELAST_ERR_LIST_OVERFLOW 0x20u  /* neighbour slots per atom exceeded */
#define MDELAST_ERR_CELL_OVERFLOW 0x40u  /* atoms per cell exceeded */
#define MDELAST_FATAL_MASK 0xffu
#define MDELAST_WARN_VIRIAL 0x100u       /* md_driver.cpp:424-429 "FATAL VIRIALS" print */
#define MDELAST_WARN_RMIN 0x200u         /* potential.hpp:93-95 r < rmin_fatal print */
#define MDELAST_WARN_TCONF_ZERO 0x400u   /* md_driver.cpp:518-519 */

/* enums of md_driver.hpp:20-21 */
#define MDELAST_NVE 0
#define MDELAST_NVT 1
#define MDELAST_NPT 2
#define MDELAST_NPT_FLEX 3
#define MDELAST_THERMOSTAT_KINETIC 0
#define MDELAST_THERMOSTAT_CONFIGURATIONAL 1
#define MDELAST_THERMOSTAT_AVERAGE 2

/* table interpolation (poly_table.hpp:137-176) */
#define MDELAST_QUINTIC 0
#define MDELAST_BSPLINE 1

/* arithmetic of the pair kernels */
#define MDELAST_PRECISION_FP64 0  /* FP64 throughout, CGS, the reference's formulas */
#define MDELAST_PRECISION_MIXED 1 /* FP32 pair and table math, FP64 sums and integrator */

const char *mdelast_last_error(void);
int mdelast_abi_version(void);
/* 1 when a CUDA device is usable, 0 otherwise (no error). */
int mdelast_device_available(void);
/* Drivers take their device buffers from a stream-ordered memory pool of the library's
 * own (one per device; the device's default pool is not touched), which keeps freed memory
 * for the next driver, and stage their atom uploads in a pinned host buffer kept for the
 * next creation; this hands the unused part of the pool back to the device and frees the
 * pinned buffer. No reference counterpart (the reference holds host memory only). */
int mdelast_release_cached_memory(int32_t device);

/* ---------------------------------------------------------------------------------
 * Tabulated functions.
 * mdelast_pair_table_create replaces the TablePotential constructor
 * (potential.hpp:77-104, bound at md_driver_module.cpp:58-66); mdelast_eam_create the
 * EAM constructor (eam.hpp:10-28, md_driver_module.cpp:68-85). Node arrays f, f', f''
 * at x_i = i*h, i = 0..n-1, exactly as get_potential.py passes them. Coefficients are
 * built once on the host in extended precision (poly_table.hpp:35-63) and uploaded when
 * a driver is created. The host evaluators below serve the scalar calculate()/rho()/F()
 * methods of the binding; the step itself never calls them.
 * ------------------------------------------------------------------------------- */
typedef struct mdelast_pair_s mdelast_pair;
typedef struct mdelast_eam_s mdelast_eam;

int mdelast_pair_table_create(double rcut, double rmin_fatal, double dr, int64_t n_nodes,
                              const double *v, const double *dv, const double *d2v,
                              int interpolation, mdelast_pair **out);
/* Analytic pair potentials of potential.hpp:29-75 (Morse, LennardJones): host
 * evaluation only; a driver given one returns MDELAST_ERR_UNSUPPORTED. */
int mdelast_pair_morse_create(double rcut, double D, double alpha, double r0,
                              mdelast_pair **out);
int mdelast_pair_lj_create(double rcut, double epsilon, double sigma, mdelast_pair **out);
/* Potential::calculate(r) (potential.hpp:16-26): out = {V, dV/dr, d2V/dr2}. */
int mdelast_pair_eval(const mdelast_pair *p, double r, double out[3]);
/* Parameters: rcut, rmin_fatal (tables), kind (0 table, 1 Morse, 2 LJ), interpolation */
int mdelast_pair_info(const mdelast_pair *p, double *rcut, int *kind, int *interpolation);
void mdelast_pair_destroy(mdelast_pair *p);

int mdelast_eam_create(double rcut, double rhomax_fatal, double dr, double drho,
                       int64_t n_r, const double *rho, const double *drho_dr,
                       const double *d2rho_dr2, int64_t n_rho, const double *F,
                       const double *dF, const double *d2F, int interpolation,
                       mdelast_eam **out);
/* EAM::rho, drhodr, d2rhodr2, F, dFdrho, d2Fdrho2 (eam.hpp:30-70) for what = 0..5.
 * F-family calls with rho > rhomax_fatal return MDELAST_ERR_FATAL (the reference exits). */
int mdelast_eam_eval(const mdelast_eam *e, int what, double x, double *out);
int mdelast_eam_info(const mdelast_eam *e, double *rcut, double *rhomax_fatal,
                     int *interpolation);
void mdelast_eam_destroy(mdelast_eam *e);

/* Evaluate a table on the GPU at n points (host arrays in and out; out is n x 3).
 * which: 0 pair V/dV/d2V ; 1 rho/drho/d2rho ; 2 F/dF/d2F. Used to check the device
 * table code against the host and the oracle. */
int mdelast_table_eval_device(const mdelast_pair *p, const mdelast_eam *e, int which,
                              const double *x, int64_t n, double *out);

/* ---------------------------------------------------------------------------------
 * Driver: one periodic cell, the state MDDriver holds (md_driver.hpp:18-168).
 * mdelast_driver_create replaces the 17-argument MDDriver constructor
 * (md_driver.cpp:16-160, md_driver_module.cpp:95-102) and, like it, builds the
 * neighbour list (if enabled), computes forces, kinetic energies and thermodynamics.
 * ------------------------------------------------------------------------------- */
typedef struct mdelast_driver_s mdelast_driver;

typedef struct {
    int32_t n_atoms;
    int32_t n_types;
    const double *positions;  /* n_atoms x 3 [cm], |x| < box/2 (md_driver.cpp:91-97) */
    const double *velocities; /* n_atoms x 3 [cm/s] */
    const uint32_t *types;    /* n_atoms, < n_types */
    const double *mass;       /* n_types [g] */
    const mdelast_pair *const *pair; /* n_types (n_types+1)/2, slot j(j+1)/2 + i, i <= j */
    const mdelast_eam *const *eam;   /* n_eam entries (0 or n_types) */
    int32_t n_eam;
    int32_t ensemble;         /* MDELAST_NVE .. */
    int32_t coupling;         /* MDELAST_THERMOSTAT_* */
    /* Thermostat(T, q, p_eta, Nf) (thermostat.hpp:9-38) */
    double thermo_T;
    int32_t thermo_nchain;
    const double *thermo_q;
    const double *thermo_p_eta;
    double thermo_Nf;
    /* Barostat(P, w, p_eps, Thermostat) (barostat.hpp:6-17) */
    double baro_P;
    double baro_w;
    double baro_p_eps;
    double baro_thermo_T;
    int32_t baro_nchain;
    const double *baro_q;
    const double *baro_p_eta;
    double baro_Nf;
    double box[9];            /* Box.h, row major; must be diagonal */
    int32_t n_rg;             /* g(r) bin centres (evenly spaced, rg[0] > 0) */
    const double *rg;
    double Nf;
    double dt;
    int32_t neighbors;        /* 1: Verlet list rebuilt by mdelast_driver_calculate_neighbors;
                                 0: all pairs within the cutoff every force call */
    double r_skin;            /* >= 1 */
    double fatal_conservation;
    int32_t precision;        /* MDELAST_PRECISION_* */
    int32_t device;           /* CUDA device ordinal */
} mdelast_driver_config;

/* Scalar state and observables after the last step: the read-only attributes of
 * MDDriver (md_driver_module.cpp:103-140). born_elasticity_tensor holds the upper
 * triangle with zeros below the diagonal, as the reference stores it. */
typedef struct {
    double epot_eam_atom, epot_atom, ekin_atom, etot_atom;
    double ekin_tot, etot_cons_initial, etot_cons, etot_cons_err;
    double virial, total_laplacian, total_force2;
    double temperature_kin, temperature_conf_inverse, pressure;
    double time;
    double cycle;
    double born_stress_tensor[6];
    double stress_tensor[6];
    double born_elasticity_tensor[36];
    double box[9];
    double baro_epsilon, baro_p_epsilon;
    double momentum_tot[3];
    uint32_t status;
    uint32_t sample_observables;
} mdelast_observables;

int mdelast_driver_create(const mdelast_driver_config *cfg, mdelast_driver **out);
void mdelast_driver_destroy(mdelast_driver *d);

/* MDDriver::integrate() (md_driver.cpp:563-601), n_steps times. Asynchronous: a FATAL
 * condition raised by a step is returned by the next call that reads results, as
 * MDELAST_ERR_FATAL with the reference's message in mdelast_last_error(). */
int mdelast_driver_integrate(mdelast_driver *d, int32_t n_steps);
/* MDDriver::calculate_neighbors() (md_driver.cpp:279-298) */
int mdelast_driver_calculate_neighbors(mdelast_driver *d);
/* n_steps of the run loop of molecular_dynamics.py:1240-1254 without its Python: before the
 * step that starts at cycle c the list is rebuilt when rebuild_every > 0 and
 * c % rebuild_every == 0 (drivers with neighbors=1), and the step samples the Born tensor
 * and Laplacian when sample_every > 0 and (c + 1) % sample_every == 0. The rebuilds run on
 * the device inside the step graph; one that outgrows the neighbour capacity stops the
 * remaining steps, and the next wait for results grows the capacity and runs them
 * (mdelast_driver_list_capacity). If device_ms is not NULL the call waits for the steps and
 * stores their duration measured with CUDA events on the driver's stream. */
int mdelast_driver_run(mdelast_driver *d, int32_t n_steps, int32_t rebuild_every,
                       int32_t sample_every, float *device_ms);
/* Diagnostics: run n_steps sampled steps with a CUDA event between consecutive kernels
 * and store the mean device time per launch, in ms, of each kernel of the step:
 * [0] opening scalar work, [1] kick + drift, [2] density pass, [3] force pass + kick,
 * [4] closing scalar work, [5] neighbour-list build. */
#define MDELAST_N_KERNEL_TIMES 6
int mdelast_driver_kernel_times(mdelast_driver *d, int32_t n_steps, double *ms_out);
/* the sample_observables flag (md_driver.hpp:163-167) */
int mdelast_driver_set_sample_observables(mdelast_driver *d, int32_t flag);
int mdelast_driver_get_sample_observables(const mdelast_driver *d, int32_t *flag);
/* wait for queued work; returns MDELAST_ERR_FATAL if a step raised a FATAL bit */
int mdelast_driver_synchronize(mdelast_driver *d);

int mdelast_driver_get_observables(mdelast_driver *d, mdelast_observables *out);

/* per-atom arrays (md_driver_module.cpp:103-109) */
#define MDELAST_ATOM_POSITIONS 0   /* n x 3 */
#define MDELAST_ATOM_COORDINATES 1 /* n x 3, scaled, not wrapped (md_driver.cpp:483-485) */
#define MDELAST_ATOM_VELOCITIES 2  /* n x 3 */
#define MDELAST_ATOM_FORCES 3      /* n x 3 */
#define MDELAST_ATOM_RHO 4         /* n */
#define MDELAST_ATOM_EPOT 5        /* n */
#define MDELAST_ATOM_EKIN 6        /* n */
int mdelast_driver_get_atoms(mdelast_driver *d, int32_t field, double *out);

/* Thermostat chains (thermostat.hpp:9-38): which 0 particle thermostat, 1 barostat's.
 * Writes nchain values to each non-NULL array. */
int mdelast_driver_get_chain(mdelast_driver *d, int32_t which, double *q, double *p_eta,
                             double *eta, int32_t *nchain);

/* The half list in the reference's CSR form (md_driver.hpp:87-90): point[n+1] and, for
 * each atom i, its partners j > i in ascending order. Copies at most cap entries and
 * returns the total in *n_entries. MDELAST_ERR_UNSUPPORTED when lists are disabled. */
int mdelast_driver_get_neighbors(mdelast_driver *d, int32_t *point, int32_t *neighbors,
                                 int64_t cap, int64_t *n_entries);

/* ---------------------------------------------------------------------------------
 * Batches: many independent replicas (cells of any size, composition, temperature,
 * ensemble and seed) that share one potential, advanced together - every kernel of a
 * step covers all replicas, and the scalar NHC/barostat work of the replicas runs side
 * by side. The reference runs such replicas as separate processes
 * (benchmarks/slurm_example.sh:6-24). A batch is a driver handle: mdelast_driver_run,
 * _integrate, _calculate_neighbors, _set_sample_observables, _synchronize,
 * _kernel_times and _destroy act on all its replicas; the readouts below take a replica
 * index (the mdelast_driver_get_* functions read replica 0).
 * ------------------------------------------------------------------------------- */
/* cfgs[k] describes replica k; all must give the same pair/EAM handles and masses, the
 * same neighbors, r_skin, precision and device. */
int mdelast_batch_create(const mdelast_driver_config *cfgs, int32_t n_replicas,
                         mdelast_driver **out);
int mdelast_batch_size(const mdelast_driver *d, int32_t *n_replicas, int64_t *n_atoms);
int mdelast_batch_get_observables(mdelast_driver *d, int32_t replica, mdelast_observables *out);
int mdelast_batch_get_atoms(mdelast_driver *d, int32_t replica, int32_t field, double *out);
int mdelast_batch_get_chain(mdelast_driver *d, int32_t replica, int32_t which, double *q,
                            double *p_eta, double *eta, int32_t *nchain);
int mdelast_batch_get_neighbors(mdelast_driver *d, int32_t replica, int32_t *point,
                                int32_t *neighbors, int64_t cap, int64_t *n_entries);
/* Status word of every replica (MDELAST_FATAL_* / MDELAST_ERR_* / MDELAST_WARN_* bits)
 * after the queued steps, into status[n_replicas]. Unlike the readouts above it succeeds
 * after a FATAL bit has stopped the batch, so a caller can tell which replica raised it. */
int mdelast_batch_get_status(mdelast_driver *d, uint32_t *status);

/* Pair correlation (md_driver.cpp:732-862): mode 0 calculate_pair_correlation,
 * 1 calculate_pair_correlations, 2 calculate_partial_pair_correlation. gr has n_rg
 * values, gr_partial n_types(n_types+1)/2 x n_rg. */
int mdelast_driver_pair_correlation(mdelast_driver *d, int32_t mode);
/* Copies the last results: gr (n_rg) and gr_partial (n_types(n_types+1)/2 rows of n_rg,
 * row a + b(b+1)/2 for types a <= b); either may be NULL. Before any calculation, and for
 * the part a mode did not compute, the previous values (initially zeros), as the
 * reference's gr / gr_partial attributes. */
int mdelast_driver_get_gr(mdelast_driver *d, double *gr, double *gr_partial);
/* The same for replica `replica` of a batch, with that replica's rg. */
int mdelast_batch_pair_correlation(mdelast_driver *d, int32_t replica, int32_t mode);
int mdelast_batch_get_gr(mdelast_driver *d, int32_t replica, double *gr, double *gr_partial);

/* Launch shapes of the two pair passes. No counterpart in the reference (its loops are
 * serial). autotune times the density and the force pass (sampled-step variants when the
 * driver samples observables, else the plain ones) on the current positions for every
 * lanes-per-atom value in {1, 4, 8, 16} and block target in {8, 16, 32, 64} x 148, n_repeat
 * launches each, and where the tables are staged (below) also the staged force pass with
 * 4, 8 or 16 lanes per atom and {1, 2, 4} x 148 blocks of 512 threads; it keeps the fastest
 * for each pass and recomputes the per-atom state with it; the state does not advance.
 * choice (4 values, may be NULL): lanes per atom of the density and force passes, block
 * targets of the density and force passes; ms_out (2, may be NULL): their mean times in
 * ms. set_launch sets a shape directly (keeping the force-pass variant). Both drop the
 * captured step graphs (recaptured on the next step). */
int mdelast_driver_autotune(mdelast_driver *d, int32_t n_repeat, int32_t *choice,
                            double *ms_out);
int mdelast_driver_set_launch(mdelast_driver *d, int32_t tpa_density, int32_t tpa_force,
                              int32_t blocks_density, int32_t blocks_force);
/* The same choice made on real steps: each candidate shape runs n_steps sampled steps of
 * run(n, rebuild_every, 1) (the state advances: use it as part of a warm-up), and the
 * passes are timed in the cache state a step leaves them, which repeated passes on a fixed
 * state (autotune) do not reproduce. The density pass is tuned first over lanes per atom
 * {1, 4, 8, 16} x {16, 32, 64} x 148 blocks, then the force pass over {1, 4, 8, 16} x
 * {8, 16, 32} x 148 and, where tables are staged, the staged pass at {4, 8} x {4, 8} x 148.
 * About 30 n_steps steps in all. choice and ms_out as for autotune. */
int mdelast_driver_autotune_steps(mdelast_driver *d, int32_t n_steps, int32_t rebuild_every,
                                  int32_t *choice, double *ms_out);
/* The staged force pass. No counterpart in the reference. In mixed precision with quintic
 * EAM tables, a driver keeps an FP32 copy of the top intervals of every phi_ab and rho_a
 * (those up to the largest cutoff, at most 184 KB; each function once), and the staged
 * force pass copies it into each block's shared memory and reads the tables there instead
 * of through the L1 (a two-element alloy's tables fit down to r of about 1.6 A; shorter
 * pairs read the global tables). Per-atom results are bit for bit those of the other
 * force pass. set: on (1) or off (0), with the current lanes per atom (4, 8 or 16 when on)
 * and block target; MDELAST_ERR_UNSUPPORTED when no staged copy exists. get: *on the
 * variant in use, *available whether a staged copy exists (either may be NULL). */
int mdelast_driver_set_force_staging(mdelast_driver *d, int32_t on);
/* Neighbour-list capacity per atom (*maxn) and how many step launches were resumed after
 * an in-step list rebuild outgrew it (*regrowths); either may be NULL. The reference grows
 * its list whenever it needs to (md_driver.cpp:288-292); here an in-step rebuild that
 * overflows stops the launch's remaining steps on the device (their kernels return without
 * work), and the next wait for results grows the capacity and runs those steps again, so
 * run()/integrate_n() continue instead of failing. MDELAST_LIST_HEADROOM (default 0.5)
 * sets the headroom h of a new capacity: (1 + h) x the largest count, + 32 when h > 0. */
int mdelast_driver_list_capacity(mdelast_driver *d, int32_t *maxn, int32_t *regrowths);
int mdelast_driver_get_force_staging(mdelast_driver *d, int32_t *on, int32_t *available);
/* The list the pair passes walk. No counterpart in the reference (its passes walk the
 * neighbour list, whose pairs beyond r_cut they skip). factor > 1: the neighbour list's
 * pairs within factor * r_cut (FP64 min-image, the same test from both atoms), rebuilt after
 * every neighbour-list rebuild and whenever some atom has moved by more than
 * (factor - 1) r_cut / 2 since the last refresh, so every pair within r_cut is kept and the
 * results do not change; factor 0: the neighbour list itself. Drivers start at 1.06 when
 * they keep a neighbour list with r_skin above it (the environment variable
 * MDELAST_PAIR_LIST sets another start value). */
int mdelast_driver_set_pair_list(mdelast_driver *d, double factor);

/* ---- Samples and fluctuation sums (molecular_dynamics.py:1218-1238, 663-1000) ----
 *
 * Every step that samples observables (sample_observables set, or the sampled steps of
 * mdelast_driver_run) appends one record of what the reference's append_sample reads
 * after that step (molecular_dynamics.py:1218-1238) to a ring on the device, one ring per
 * replica. The host drains it when it wants the series, so a run needs no per-step
 * readout. */
typedef struct mdelast_sample {
    double time, cycle;
    double temperature_kin, temperature_conf_inverse, total_laplacian, total_force2;
    double pressure;
    double stress_tensor[6];
    double etot_atom, epot_atom, epot_eam_atom, ekin_atom, etot_cons, etot_cons_err;
    double born_stress_tensor[6];
    double born_elasticity_tensor[21]; /* upper triangle, row by row (C11 C12 .. C16 C22 ..) */
    double volume;                     /* box volume after the step */
    double status;                     /* the status word after the step */
} mdelast_sample;

#define MDELAST_DEFAULT_SAMPLE_RING 1024
/* (Re)allocate every replica's ring with room for `capacity` records (0: no ring);
 * records not yet drained are dropped. A driver starts with MDELAST_DEFAULT_SAMPLE_RING. */
int mdelast_driver_set_sample_ring(mdelast_driver *d, int32_t capacity);
/* Copy the records written since the last drain, oldest first, at most `cap`; *n_out gets
 * the number copied and *n_lost the number overwritten before they were drained. Records
 * beyond `cap` stay for the next drain. */
int mdelast_driver_drain_samples(mdelast_driver *d, mdelast_sample *out, int64_t cap,
                                 int64_t *n_out, int64_t *n_lost);
int mdelast_batch_drain_samples(mdelast_driver *d, int32_t replica, mdelast_sample *out,
                                int64_t cap, int64_t *n_out, int64_t *n_lost);

/* Running sums of the production window for the fluctuation formula of the elastic
 * constants (molecular_dynamics.py:826-958), bulk modulus and thermal expansion
 * (:776-824), updated on the device at every sampled step once started (Welford's
 * updates in FP64). x = (born_stress_tensor[6], N/V, V, etot_atom). */
typedef struct mdelast_fluct {
    double n;                 /* samples accumulated */
    double n_atoms;
    double mean[9];           /* means of x */
    double comoment[45];      /* sum (x_a - mean_a)(x_b - mean_b), a <= b, row by row */
    double born_el_mean[21];  /* mean of born_elasticity_tensor (upper triangle) */
} mdelast_fluct;
/* Clear the sums of every replica and start accumulating from the next sampled step
 * (the reference's samples_thermalization cut). */
int mdelast_driver_fluct_start(mdelast_driver *d);
int mdelast_driver_get_fluct(mdelast_driver *d, mdelast_fluct *out);
int mdelast_batch_get_fluct(mdelast_driver *d, int32_t replica, mdelast_fluct *out);
/* The reference's estimator (molecular_dynamics.py:776-824, 826-958) from the sums, on the
 * host: C (6 x 6) = <C^B> - <V>/kT cov(s', s') + ideal-gas term (+ bulk modulus in the
 * upper-left block for NPT), s' = sigma^B - (N kT / V) delta in NPT; kT = k_B T_thermostat.
 * summary (6 values, may be NULL): C11, C12, C44 (component averages), bulk modulus,
 * isothermal compressibility, volumetric thermal expansion (the last three 0 unless NPT).
 * Needs at least 2 samples. */
int mdelast_elastic_constants(const mdelast_fluct *f, int32_t ensemble, double T_thermostat,
                              double P_barostat, double *C, double *summary);

/* ---- Learned warm start: a small MLP trained and evaluated on the device ----
 * No counterpart in the reference (its runs start from a guessed lattice constant and
 * equilibrate by NPT). Fully connected layers of the given widths, GELU between layers,
 * linear output, FP32; loss = mean squared error over all outputs; Adam (lr, beta 0.9 /
 * 0.999, eps 1e-8), full batch. Parameters: per layer W (in x out, row-major) then b (out).
 * Training is deterministic (fixed-order sums, no atomics). */
typedef struct mdelast_mlp_s mdelast_mlp;
#define MDELAST_MLP_MAX_LAYERS 8
/* widths: n_layers + 1 values (inputs, hidden widths, outputs). Glorot-normal weights and
 * zero biases drawn from `seed`. */
int mdelast_mlp_create(int32_t n_layers, const int32_t *widths, uint64_t seed, int32_t device,
                       mdelast_mlp **out);
void mdelast_mlp_destroy(mdelast_mlp *m);
int mdelast_mlp_n_params(const mdelast_mlp *m, int64_t *n);
int mdelast_mlp_get_params(mdelast_mlp *m, float *out);
/* also resets the optimiser state */
int mdelast_mlp_set_params(mdelast_mlp *m, const float *in);
/* y (n x outputs) = f(x (n x inputs)); host arrays */
int mdelast_mlp_forward(mdelast_mlp *m, const float *x, int32_t n, float *y);
/* loss and its gradient with respect to every parameter (host arrays; either output may
 * be NULL), without changing the parameters */
int mdelast_mlp_gradients(mdelast_mlp *m, const float *x, const float *y, int32_t n,
                          float *loss, float *grad);
/* `steps` Adam steps on (x, y); *loss (may be NULL) = the loss after the last step */
int mdelast_mlp_train(mdelast_mlp *m, const float *x, const float *y, int32_t n,
                      int32_t steps, float lr, float *loss);

/* g(r) that allocates nothing. No counterpart in the reference: it exists for callers
 * that may not allocate device memory when they sample g(r), for example an application
 * whose allocator owns all device memory and forbids third-party cudaMalloc/cudaFree, or
 * a sampling loop that cannot take the device-wide synchronisation of a cudaFree.
 *
 * Same counting and normalisation as mdelast_driver_pair_correlation (md_driver.cpp:
 * 732-862) and bit-identical results on the same coordinates, but on arrays the caller
 * holds on the current device: coordinates (n_atoms x 3 scaled coordinates, as the
 * MDELAST_ATOM_COORDINATES readout), types (n_atoms values; an atom whose type is not in
 * [0, n_types) takes no part: it is in no pair count and not in the N of the
 * normalisations), rg (n_rg evenly spaced bin centres, rg[0] > 0), and the outputs
 * gr (n_rg, written for modes 0 and 1) and gr_partial (n_types(n_types+1)/2 rows of n_rg,
 * written for modes 1 and 2; the other may be NULL). box: 3 edges of the diagonal box, in
 * host memory. The work is queued on `stream` (a cudaStream_t; NULL is the default stream)
 * and the call returns without waiting for it.
 *
 * Scratch: a fixed array in the library's device image holding
 * (1 + n_types(n_types+1)/2) x n_rg 64-bit counters, at most MDELAST_GR_STATIC_MAX_SLOTS
 * (512 KB), and n_types <= 8; larger requests return MDELAST_ERR_CAPACITY with the sizes
 * in mdelast_last_error(). Nothing needs to start at zero: each call clears the counters it
 * uses on `stream` before counting.
 *
 * The first call on a device does set-up (it loads the library's kernels on that device
 * and looks up the scratch address with cudaGetSymbolAddress, with that device current);
 * make it before any stream capture begins. The address is kept for the life of the
 * process: after a cudaDeviceReset of that device it is stale, and this entry point must
 * not be used on that device again in the same process. There is ONE scratch array per
 * device: calls
 * that overlap on the same device (different streams, or different host threads, without
 * ordering between them) race on it and give wrong counts; order them on one stream or
 * with events. */
#define MDELAST_GR_STATIC_MAX_SLOTS 65536
int mdelast_pair_correlation_static(const double *coordinates, const uint32_t *types,
                                    int32_t n_atoms, int32_t n_types, const double *box,
                                    const double *rg, int32_t n_rg, int32_t mode, double *gr,
                                    double *gr_partial, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MDELAST_H_ */
