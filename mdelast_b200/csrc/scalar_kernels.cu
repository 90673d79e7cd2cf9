// Per-replica scalar work of a step: the Nose-Hoover-chain thermostat and barostat
// propagators (thermostat.cpp:40-66, md_driver.cpp:454-561), the coefficients of the
// kick and drift, the deterministic reduction of the atom kernels' block sums, and the
// thermodynamics with the reference's fatal checks (md_driver.cpp:603-730).
//
// One block per replica. The particle thermostat chain and the barostat chain are
// independent within a half step and run side by side on the first threads of two warps.
#include "kernels.cuh"

namespace mdelast {

namespace {

__constant__ double c_wsy7[7] = {
    0.784513610477560, 0.235573213359357, -1.17767998417887,
    1. - 2. * (0.784513610477560 + 0.235573213359357 - 1.17767998417887),
    -1.17767998417887, 0.235573213359357, 0.784513610477560}; // numerics.hpp:22-27

constexpr double kBoltz = 1.38064852e-16; // units.hpp:7

// exp(-x) and op(x) = (1 - exp(-x))/x of numerics.hpp:11-18.
//
// expx_exact is the reference's formula: the library exp, then op = (1 - e)/x, or for
// |x| <= 1e-3 the reference's own 5th-order Taylor polynomial of op.
//
// expx_series evaluates op from its Taylor series op(x) = sum (-x)^k/(k+1)! to degree 23
// by Estrin's scheme, and exp(-x) = 1 - x op(x) with one FMA. For |x| <= 2 the first omitted
// term, x^24/25!, is below 3e-18 relative; measured against long-double references over
// [-2, 2], op is within 4 ulp and exp(-x) within 22 ulp (at x = 2, where 1 - x op = 0.135
// loses three bits). It has no branch. Thermostat arguments are x = dt p_eta/Q: ~dt/tau
// at equilibrium (0.02 for tau = 50 fs, dt = 2 fs), but in the first few hundred steps from
// a lattice start the upper links of a 13,500-atom cell's chain reach 1.24 (half of the
// arguments above 1/16, 6 % above 1/2).
__device__ __forceinline__ void expx_exact(double x, double &expx, double &op) {
    double const c1 = -1.0 / 2.0, c2 = 1.0 / 6.0, c3 = -1.0 / 24.0, c4 = 1. / 120.,
                 c5 = -1. / 720.;
    double const e = exp(-x);
    expx = e;
    op = fabs(x) > 1e-3 ? (1.0 - e) / x
                        : 1.0 + x * (c1 + x * (c2 + x * (c3 + x * (c4 + x * c5))));
}

constexpr double kSeriesMax = 2.0;

__device__ __forceinline__ void expx_series(double x, double &expx, double &op) {
    double const y = -x, y2 = y * y, y4 = y2 * y2, y8 = y4 * y4, y16 = y8 * y8;
    double const b0 = fma(y, 1.0 / 2.0, 1.0), b1 = fma(y, 1.0 / 24.0, 1.0 / 6.0),
                 b2 = fma(y, 1.0 / 720.0, 1.0 / 120.0), b3 = fma(y, 1.0 / 40320.0, 1.0 / 5040.0),
                 b4 = fma(y, 1.0 / 3628800.0, 1.0 / 362880.0),
                 b5 = fma(y, 1.0 / 479001600.0, 1.0 / 39916800.0),
                 b6 = fma(y, 1.0 / 87178291200.0, 1.0 / 6227020800.0),
                 b7 = fma(y, 1.0 / 20922789888000.0, 1.0 / 1307674368000.0),
                 b8 = fma(y, 1.0 / 6402373705728000.0, 1.0 / 355687428096000.0),
                 b9 = fma(y, 1.0 / 2432902008176640000.0, 1.0 / 121645100408832000.0),
                 b10 = fma(y, 1.0 / 1124000727777607680000.0, 1.0 / 51090942171709440000.0),
                 b11 = fma(y, 1.0 / 620448401733239439360000.0, 1.0 / 25852016738884976640000.0);
    double const t0 = fma(y2, b1, b0), t1 = fma(y2, b3, b2), t2 = fma(y2, b5, b4),
                 t3 = fma(y2, b7, b6), t4 = fma(y2, b9, b8), t5 = fma(y2, b11, b10);
    double const u0 = fma(y4, t1, t0), u1 = fma(y4, t3, t2), u2 = fma(y4, t5, t4);
    op = fma(y16, u2, fma(y8, u1, u0));
    expx = fma(-x, op, 1.0);
}

// The series outside its range falls back to the exact form.
__device__ __forceinline__ void expx_operator(double x, double &expx, double &op) {
    expx_series(x, expx, op);
    if (fabs(x) > kSeriesMax)
        expx_exact(x, expx, op);
}

// In a chain sweep: EXACT = false takes the series alone and only notes an argument beyond
// its range in `large`; a half step that saw one is redone from its start with EXACT = true,
// which falls back to the exact form per exponential. A branch per exponential, even one
// never taken, doubled the time of a 10-link half step (27,600 against 13,500 cycles).
template <bool EXACT>
__device__ __forceinline__ void expx_sweep(double x, double &expx, double &op, bool &large) {
    if (EXACT) {
        expx_operator(x, expx, op);
    } else {
        expx_series(x, expx, op);
        large |= fabs(x) > kSeriesMax;
    }
}

__device__ __forceinline__ double volume(const double h[3]) { return h[0] * (h[1] * h[2]); }

// A chain of NC links held in registers while it is propagated: NC is a template
// parameter (dispatched from the runtime chain length), so the loops unroll exactly and no
// predicated-off link sits on the sequential critical path of a sweep.
template <int NC> struct ChainR {
    double p[NC], iq[NC], eta[NC];
    double kT, Nf;
};

template <int NC> __device__ __forceinline__ void chain_load(Chain const &c, ChainR<NC> &r) {
    r.Nf = c.Nf;
    r.kT = kBoltz * c.T;
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        r.p[j] = c.p_eta[j];
        r.iq[j] = c.inv_q[j];
        r.eta[j] = c.eta[j];
    }
}

template <int NC> __device__ __forceinline__ void chain_store(ChainR<NC> const &r, Chain &c) {
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        c.p_eta[j] = r.p[j];
        c.eta[j] = r.eta[j];
    }
}

// thermostat.cpp:40-66 (Yu et al., Chem. Phys. 370 (2010) 294, eq. 8; Allen-Tildesley
// eqs. 3.73-3.74a): one sweep of the chain. Inward (top link first) each link needs the
// updated link above it, so its exponential is on the critical path; outward every
// exponential uses the not-yet-updated link above and all are formed up front.
template <int NC, bool EXACT>
__device__ __forceinline__ void U4_in(ChainR<NC> &c, double dt, double ec, bool &large) {
#pragma unroll
    for (int j = NC - 1; j >= 0; --j) {
        double G;
        if (j != 0)
            G = c.p[j - 1] * c.p[j - 1] * c.iq[j - 1] - c.kT;
        else
            G = 2. * ec - c.Nf * c.kT;
        if (j == NC - 1) {
            c.p[j] += dt * G;
        } else {
            double e, op;
            expx_sweep<EXACT>(dt * c.p[j + 1] * c.iq[j + 1], e, op, large);
            c.p[j] = c.p[j] * e + dt * G * op;
        }
    }
}

template <int NC, bool EXACT>
__device__ __forceinline__ void U4_out(ChainR<NC> &c, double dt, double ec, bool &large) {
    double e[NC], op[NC];
#pragma unroll
    for (int j = 0; j < NC - 1; ++j)
        expx_sweep<EXACT>(dt * c.p[j + 1] * c.iq[j + 1], e[j], op[j], large);
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        double G;
        if (j != 0)
            G = c.p[j - 1] * c.p[j - 1] * c.iq[j - 1] - c.kT;
        else
            G = 2. * ec - c.Nf * c.kT;
        if (j == NC - 1)
            c.p[j] += dt * G;
        else
            c.p[j] = c.p[j] * e[j] + dt * G * op[j];
    }
}

// thermostat.hpp:24-35: factor exp(-dt p_eta[0]/Q[0]) for the coupled momenta; advances
// the chain positions
template <int NC, bool EXACT> __device__ __forceinline__ double U3(ChainR<NC> &c, double dt,
                                                                  bool &large) {
    double s, op;
    expx_sweep<EXACT>(dt * c.p[0] * c.iq[0], s, op, large);
#pragma unroll
    for (int j = 0; j < NC; ++j)
        c.eta[j] += dt * c.p[j] * c.iq[j];
    return s;
}

// thermostat.cpp:24-37
__device__ double chain_etot(Chain const &c) {
    double e = c.Nf * c.eta[0];
    for (int j = 1; j < c.n; ++j)
        e += c.eta[j];
    e *= kBoltz * c.T;
    for (int j = 0; j < c.n; ++j)
        e += 0.5 * (c.p_eta[j] * c.p_eta[j]) / c.q[j];
    return e;
}

// One Suzuki-Yoshida sub-step of the particle thermostat (md_driver.cpp:539-549 with the U4
// coupling of md_driver.cpp:512-531): returns the U3 factor; the kinetic energy follows it
// as ekin * s^2.
template <int NC, bool EXACT>
__device__ __forceinline__ double thermo_substep(ChainR<NC> &c, double dtw, double &ekin,
                                                 bool conf, bool average, double econf,
                                                 bool &large) {
    U4_in<NC, EXACT>(c, 0.5 * dtw, !conf ? ekin : (average ? 0.5 * (ekin + econf) : econf),
                     large);
    double const s = U3<NC, EXACT>(c, dtw, large);
    ekin = ekin * s * s;
    U4_out<NC, EXACT>(c, 0.5 * dtw, !conf ? ekin : (average ? 0.5 * (ekin + econf) : econf),
                      large);
    return s;
}

// The particle thermostat's half step (md_driver.cpp:539-549). The velocities are not
// touched: the product of the seven U3 factors is returned and applied by the next atom
// kernel. The chain in memory is written only by a half step that completes.
template <int NC, bool EXACT>
__device__ __forceinline__ double thermo_half(Chain &gc, double dt, double &ekin, bool conf,
                                              bool average, double econf, bool &large) {
    ChainR<NC> c;
    chain_load<NC>(gc, c);
    double S = 1.;
#pragma unroll 1
    for (int k = 0; k < 7; ++k)
        S *= thermo_substep<NC, EXACT>(c, c_wsy7[k] * dt, ekin, conf, average, econf, large);
    if (EXACT || !large)
        chain_store<NC>(c, gc);
    return S;
}

template <int NC>
__device__ __noinline__ double thermo_half_exact(Chain &gc, double dt, double &ekin, bool conf,
                                                 bool average, double econf) {
    bool large = false;
    return thermo_half<NC, true>(gc, dt, ekin, conf, average, econf, large);
}

template <int NC>
__device__ double nhc_thermo_n(Chain &gc, double dt, double &ekin, bool conf, bool average,
                               double econf) {
    double e = ekin;
    bool large = false;
    double S = thermo_half<NC, false>(gc, dt, e, conf, average, econf, large);
    if (large) {
        e = ekin;
        S = thermo_half_exact<NC>(gc, dt, e, conf, average, econf);
    }
    ekin = e;
    return S;
}

// One sub-step of the barostat's chain (md_driver.cpp:551-561, 533-537, 507-510) acting on
// the barostat momentum p.
template <int NC, bool EXACT>
__device__ __forceinline__ double baro_substep(ChainR<NC> &c, double dtw, double p, double iw,
                                               bool &large) {
    U4_in<NC, EXACT>(c, 0.5 * dtw, 0.5 * (p * p) * iw, large);
    p *= U3<NC, EXACT>(c, dtw, large);
    U4_out<NC, EXACT>(c, 0.5 * dtw, 0.5 * (p * p) * iw, large);
    return p;
}

template <int NC, bool EXACT>
__device__ __forceinline__ double baro_half(Chain &gc, double dt, double p, double iw,
                                            bool &large) {
    ChainR<NC> c;
    chain_load<NC>(gc, c);
#pragma unroll 1
    for (int k = 0; k < 7; ++k)
        p = baro_substep<NC, EXACT>(c, c_wsy7[k] * dt, p, iw, large);
    if (EXACT || !large)
        chain_store<NC>(c, gc);
    return p;
}

template <int NC>
__device__ __noinline__ double baro_half_exact(Chain &gc, double dt, double p, double iw) {
    bool large = false;
    return baro_half<NC, true>(gc, dt, p, iw, large);
}

template <int NC> __device__ double nhc_baro_n(Chain &gc, double dt, double p, double iw) {
    bool large = false;
    double const q = baro_half<NC, false>(gc, dt, p, iw, large);
    return large ? baro_half_exact<NC>(gc, dt, p, iw) : q;
}

#define MDELAST_CHAIN_CASES(F)                                                                \
    F(1) F(2) F(3) F(4) F(5) F(6) F(7) F(8) F(9) F(10) F(11) F(12) F(13) F(14) F(15) F(16)

__device__ double nhc_thermo(Replica *R, Chain &gc, double dt, double &ekin) {
    double const tci = R->obs.temperature_conf_inverse;
    bool const conf = R->coupling != MDELAST_THERMOSTAT_KINETIC && tci != 0.;
    if (R->coupling != MDELAST_THERMOSTAT_KINETIC && tci == 0.)
        atomicOr(&R->obs.status, MDELAST_WARN_TCONF_ZERO);
    double const econf = conf ? (kBoltz / tci) * R->Nf / 2. : 0.;
    bool const average = R->coupling == MDELAST_THERMOSTAT_AVERAGE;
    switch (gc.n) {
#define F(N)                                                                                  \
    case N:                                                                                   \
        return nhc_thermo_n<N>(gc, dt, ekin, conf, average, econf);
        MDELAST_CHAIN_CASES(F)
#undef F
    default:
        return 1.;
    }
}

__device__ void nhc_baro(Replica *R, Chain &gc, double dt) {
    double const iw = 1. / R->baro_w;
    double p = R->p_eps;
    switch (gc.n) {
#define F(N)                                                                                  \
    case N:                                                                                   \
        p = nhc_baro_n<N>(gc, dt, p, iw);                                                     \
        break;
        MDELAST_CHAIN_CASES(F)
#undef F
    default:
        break;
    }
    R->p_eps = p;
}

// md_driver.cpp:454-459 (Yu et al. eq. 31)
__device__ void U2p(Replica *R, double dt, double ekin, double virial) {
    double const pv = R->baro_P * volume(R->h);
    R->p_eps += (2. * R->alpha * ekin + 3. * virial - 3. * pv) * dt;
}

__device__ int monomial_index(int iv, int ivp) {
    constexpr int VA[6] = {0, 1, 2, 1, 0, 0}, VB[6] = {0, 1, 2, 2, 2, 1};
    // exponents (x, y, z) of the monomials in the order the force kernel accumulates them
    constexpr int EX[15][3] = {{4, 0, 0}, {0, 4, 0}, {0, 0, 4}, {3, 1, 0}, {3, 0, 1},
                               {1, 3, 0}, {0, 3, 1}, {1, 0, 3}, {0, 1, 3}, {2, 2, 0},
                               {2, 0, 2}, {0, 2, 2}, {2, 1, 1}, {1, 2, 1}, {1, 1, 2}};
    int e[3] = {0, 0, 0};
    e[VA[iv]]++;
    e[VB[iv]]++;
    e[VA[ivp]]++;
    e[VB[ivp]]++;
    for (int m = 0; m < 15; ++m)
        if (EX[m][0] == e[0] && EX[m][1] == e[1] && EX[m][2] == e[2])
            return m;
    return 0;
}

// The replica state in shared memory for k_post: one thread works through a long chain of
// dependent updates of it (the thermodynamics), and reading and writing it in global
// memory on that chain costs a round trip to L2 per access. Copied in and out by the
// whole block.
__device__ __forceinline__ void replica_load(Replica const *g, Replica *s) {
    static_assert(sizeof(Replica) % sizeof(double) == 0, "Replica is copied as doubles");
    const double *src = reinterpret_cast<const double *>(g);
    double *dst = reinterpret_cast<double *>(s);
    for (int k = threadIdx.x; k < static_cast<int>(sizeof(Replica) / sizeof(double));
         k += blockDim.x)
        dst[k] = src[k];
    __syncthreads();
}

__device__ __forceinline__ void replica_store(Replica const *s, Replica *g) {
    __syncthreads();
    const double *src = reinterpret_cast<const double *>(s);
    double *dst = reinterpret_cast<double *>(g);
    for (int k = threadIdx.x; k < static_cast<int>(sizeof(Replica) / sizeof(double));
         k += blockDim.x)
        dst[k] = src[k];
}

} // namespace

// Opening scalar work of integrate() (md_driver.cpp:567-581): barostat and particle NHC
// half steps, U2p, and the coefficients of the opening kick and of the drift, with the
// NPT box update of U1 (md_driver.cpp:488-498).
__global__ void k_pre(AtomsView A) {
    if (*A.halt) // a list build ran out of capacity: nothing until the host regrows
        return;
    Replica *R = A.rep + blockIdx.x;
    __shared__ double s_S, s_ekin;
    int const ens = R->ensemble;
    double const dt = R->dt;
    if (threadIdx.x == 0) {
        R->sub_d2 = 0.; // k_kick_drift takes this step's largest displacement
        double ekin = R->obs.ekin_tot;
        double S = 1.;
        if (ens == MDELAST_NVT || ens == MDELAST_NPT) {
            S = nhc_thermo(R, R->th, 0.5 * dt, ekin);
        }
        s_S = S;
        s_ekin = ekin;
    } else if (threadIdx.x == 32 && ens == MDELAST_NPT) {
        nhc_baro(R, R->bth, 0.5 * dt);
    }
    __syncthreads();
    if (threadIdx.x != 0)
        return;
    double const ekin = s_ekin;
    R->obs.ekin_tot = ekin;
    double e = 1., c = 1.;
    if (ens == MDELAST_NPT) {
        U2p(R, 0.5 * dt, ekin, R->obs.virial);
        double const x = R->alpha * (0.5 * dt) * R->p_eps / R->baro_w;
        expx_operator(x, e, c);
    }
    R->s_kick = R->vscale * s_S;
    R->vscale = 1.;
    R->e_kick = e;
    R->cdt_kick = c * (0.5 * dt);
    // U1 (md_driver.cpp:464-470, 488-498)
    double cf = 1.;
    if (ens == MDELAST_NPT) {
        double const x = dt * R->p_eps / R->baro_w;
        R->eps += x;
        double ee;
        expx_operator(x, ee, cf);
    }
    R->cfdt = cf * dt;
    for (int a = 0; a < 3; ++a)
        R->h_pos[a] = R->h[a];
    if (ens == MDELAST_NPT) {
        double const expe = exp(R->eps);
        double const vol_old = volume(R->h);
        for (int a = 0; a < 3; ++a)
            R->h[a] = R->h0[a] * expe;
        if (fabs(volume(R->h) / vol_old - 1.) > 0.05)
            atomicOr(&R->obs.status, MDELAST_FATAL_VOLUME);
    }
}

// Closing scalar work: reduce the block sums of the density and force passes, finish
// calculate_forces (md_driver.cpp:410-429), the tail of U2 (set_kinetic_energies,
// calculate_configurational_temperature), U2p and the NHC half steps (md_driver.cpp:
// 583-595), and calculate_thermodynamics (md_driver.cpp:648-730). POST_INIT does the
// part of the constructor after calculate_forces (md_driver.cpp:114-118).
// Block sums of the density and force passes folded in chunks of kChunk blocks: block
// (c, r) adds blocks [c kChunk, (c+1) kChunk) of replica r for every slot, in a fixed
// order, spreading the reduction over many SMs (k_post then adds the chunk sums).
__global__ void k_reduce(AtomsView A) {
    if (*A.halt) // a list build ran out of capacity: nothing until the host regrows
        return;
    Replica const *R = A.rep + blockIdx.y;
    int const c = blockIdx.x;
    int const g = threadIdx.x >> 6, q = threadIdx.x & 63;
    __shared__ double part[4][64];
    double a = 0.;
    if (q < F_NSUM + D_NSUM) {
        bool const fpass = q < F_NSUM;
        int const ns = fpass ? F_NSUM : D_NSUM;
        int const col = fpass ? q : q - F_NSUM;
        double const *P = fpass ? A.pf : A.pd;
        long const b0 = fpass ? R->fblk_begin : R->dblk_begin;
        int const nb = fpass ? R->fblk_n : R->dblk_n;
        int const lo = c * kChunk, hi = lo + kChunk < nb ? lo + kChunk : nb;
#pragma unroll
        for (int k = 0; k < kChunk / 4; ++k) {
            int const b = lo + g + 4 * k;
            if (b < hi)
                a += P[(b0 + b) * ns + col];
        }
    }
    part[g][q] = a;
    __syncthreads();
    if (threadIdx.x < 64)
        A.red[(static_cast<size_t>(blockIdx.y) * A.max_chunks + c) * 64 + q] =
            (part[0][q] + part[1][q]) + (part[2][q] + part[3][q]);
}

// Row a and column b (a <= b) of entry q of the upper triangle of an n x n matrix stored
// row by row.
__device__ __forceinline__ void upper_pair(int q, int n, int &a, int &b) {
    a = 0;
    while (q >= n - a) {
        q -= n - a;
        ++a;
    }
    b = a + q;
}

// One sampled step: append what molecular_dynamics.py:1218-1238 reads to the replica's
// ring, and, while accumulating, fold x = (sigma^B[6], N/V, V, etot_atom) and C^B into the
// running means and co-moments (Welford's updates; the production-window sums behind
// molecular_dynamics.py:776-958). Called by every thread of the block: each entry is one
// thread's, with the same operations in the same order as a serial update.
__device__ void record_sample(AtomsView const &A, int r, Replica *R, double V) {
    __shared__ double s_d0[9], s_d1[9];
    int const t = threadIdx.x;
    mdelast_observables const &o = R->obs;
    bool const ring = A.ring && A.ring_cap > 0;
    if (ring) {
        long const slot = static_cast<long>(R->n_samples) % A.ring_cap;
        mdelast_sample &s = A.ring[static_cast<size_t>(r) * A.ring_cap + slot];
        if (t == 0) {
            s.time = o.time;
            s.cycle = o.cycle;
            s.temperature_kin = o.temperature_kin;
            s.temperature_conf_inverse = o.temperature_conf_inverse;
            s.total_laplacian = o.total_laplacian;
            s.total_force2 = o.total_force2;
            s.pressure = o.pressure;
            s.etot_atom = o.etot_atom;
            s.epot_atom = o.epot_atom;
            s.epot_eam_atom = o.epot_eam_atom;
            s.ekin_atom = o.ekin_atom;
            s.etot_cons = o.etot_cons;
            s.etot_cons_err = o.etot_cons_err;
            s.volume = V;
            s.status = static_cast<double>(o.status);
        } else if (t >= 32 && t < 38) {
            s.stress_tensor[t - 32] = o.stress_tensor[t - 32];
            s.born_stress_tensor[t - 32] = o.born_stress_tensor[t - 32];
        } else if (t >= 64 && t < 85) {
            int a, b;
            upper_pair(t - 64, 6, a, b);
            s.born_elasticity_tensor[t - 64] = o.born_elasticity_tensor[6 * a + b];
        }
    }
    bool const acc = R->acc_on;
    mdelast_fluct &f = R->acc;
    double const n1 = f.n + 1.;
    double const inv_n = 1. / n1;
    if (acc && t < 9) {
        double const x = t < 6    ? o.born_stress_tensor[t]
                         : t == 6 ? R->n_atoms / V
                         : t == 7 ? V
                                  : o.etot_atom;
        double const d0 = x - f.mean[t];
        double const m = f.mean[t] + d0 * inv_n;
        s_d0[t] = d0;
        s_d1[t] = x - m;
        f.mean[t] = m;
    }
    __syncthreads();
    if (t == 0) {
        if (ring)
            R->n_samples += 1.;
        if (acc)
            f.n = n1;
    }
    if (!acc)
        return;
    if (t < 45) {
        int a, b;
        upper_pair(t, 9, a, b);
        f.comoment[t] += s_d0[a] * s_d1[b];
    } else if (t >= 64 && t < 85) {
        int a, b;
        upper_pair(t - 64, 6, a, b);
        f.born_el_mean[t - 64] += (o.born_elasticity_tensor[6 * a + b] - f.born_el_mean[t - 64]) * inv_n;
    }
}

// what & 1: empty every replica's sample ring; what & 2: clear the fluctuation sums and
// start accumulating.
__global__ void k_samples_reset(AtomsView A, int what) {
    int const r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n_rep)
        return;
    Replica *R = A.rep + r;
    if (what & 1)
        R->n_samples = 0.;
    if (what & 2) {
        mdelast_fluct &f = R->acc;
        f.n = 0.;
        f.n_atoms = R->n_atoms;
        for (int k = 0; k < 9; ++k)
            f.mean[k] = 0.;
        for (int k = 0; k < 45; ++k)
            f.comoment[k] = 0.;
        for (int k = 0; k < 21; ++k)
            f.born_el_mean[k] = 0.;
        R->acc_on = 1;
    }
}

__device__ void thermodynamics(Replica *R, int mode, int obs, const double *sf, const double *sd,
                               double S, double ekin, double virial);

__global__ void k_post(AtomsView A, int mode, int obs) {
    if (*A.halt) // a list build ran out of capacity: nothing until the host regrows
        return;
    __shared__ Replica sR;
    __shared__ double sf[F_NSUM], sd[D_NSUM];
    __shared__ double s_part[4][F_NSUM + D_NSUM];
    __shared__ double s_S, s_ekin, s_virial;
    replica_load(A.rep + blockIdx.x, &sR);
    Replica *R = &sR;
    int const t = threadIdx.x;
    // Chunk sums of the two passes (k_reduce): 4 groups of 64 threads, thread (g, q) adds
    // slot q over chunks g, g+4, ...; the group totals are then added in a fixed order, so
    // the result does not depend on timing.
    {
        int const g = t >> 6, q = t & 63;
        int const nslot = F_NSUM + D_NSUM;
        if (q < nslot) {
            int const nb = R->fblk_n > R->dblk_n ? R->fblk_n : R->dblk_n;
            int const nc = (nb + kChunk - 1) / kChunk;
            double const *P = A.red + static_cast<size_t>(blockIdx.x) * A.max_chunks * 64;
            double a0 = 0., a1 = 0.;
            int c = g;
            for (; c + 4 < nc; c += 8) {
                a0 += P[c * 64 + q];
                a1 += P[(c + 4) * 64 + q];
            }
            for (; c < nc; c += 4)
                a0 += P[c * 64 + q];
            s_part[g][q] = a0 + a1;
        }
        __syncthreads();
        if (t < nslot) {
            double const v = (s_part[0][t] + s_part[1][t]) + (s_part[2][t] + s_part[3][t]);
            if (t < F_NSUM)
                sf[t] = v;
            else
                sd[t - F_NSUM] = v;
        }
    }
    __syncthreads();
    int const ens = R->ensemble;
    double const dt = R->dt;
    mdelast_observables &o = R->obs;
    // The box does not change in k_post: the volume of the thermodynamics (md_driver.cpp:
    // 648-730), which divides the Born tensor, one entry per thread (zeros below the
    // diagonal, as the reference stores it).
    double const V = volume(R->h);
    if (obs && t < 36) {
        int const a = t / 6, b = t % 6;
        o.born_elasticity_tensor[t] =
            b < a ? 0. : (sf[F_CB + monomial_index(a, b)] + sd[D_CB + a * (11 - a) / 2 + b]) / V;
    }
    if (t == 0) {
        double const virial = sf[F_VIRIAL] / -3.;
        s_virial = virial;
        o.virial = virial;
        double const vir_trace = -(sf[F_SIGMA] + sf[F_SIGMA + 1] + sf[F_SIGMA + 2]);
        if (fabs(virial / (vir_trace / 3.) - 1.) > 1e-7)
            atomicOr(&o.status, MDELAST_WARN_VIRIAL);
        if (obs)
            o.total_laplacian = sf[F_LAP] + sd[D_LAP];
        double ekin = sf[F_EKIN];
        if (mode == POST_STEP) {
            if (obs) {
                double const f2 = sf[F_F2];
                o.total_force2 = f2;
                o.temperature_conf_inverse =
                    (f2 != 0. && o.total_laplacian != 0.) ? kBoltz * o.total_laplacian / f2 : 0.;
            }
            if (ens == MDELAST_NPT)
                U2p(R, 0.5 * dt, ekin, virial);
        }
        s_ekin = ekin;
    }
    __syncthreads();
    if (mode == POST_STEP) {
        if (t == 0) {
            double ekin = s_ekin, S = 1.;
            if (ens == MDELAST_NVT || ens == MDELAST_NPT) {
                S = nhc_thermo(R, R->th, 0.5 * dt, ekin);
            }
            s_S = S;
            s_ekin = ekin;
        } else if (t == 32 && ens == MDELAST_NPT) {
            nhc_baro(R, R->bth, 0.5 * dt);
        }
    } else if (t == 0) {
        s_S = 1.;
    }
    __syncthreads();
    if (t == 0)
        thermodynamics(R, mode, obs, sf, sd, s_S, s_ekin, s_virial);
    if (mode == POST_STEP && obs) {
        __syncthreads();
        record_sample(A, static_cast<int>(blockIdx.x), R, V);
    }
    replica_store(&sR, A.rep + blockIdx.x);
}

// calculate_thermodynamics (md_driver.cpp:648-730) on the replica's shared copy, one thread;
// k_post spreads the Born tensor's division by the volume and the sample record over the
// block.
__device__ void thermodynamics(Replica *R, int mode, int obs,
                               const double *sf, const double *sd, double S, double ekin,
                               double virial) {
    mdelast_observables &o = R->obs;
    double const dt = R->dt;
    int const ens = R->ensemble;
    int const N = R->n_atoms;
    R->vscale = S;
    o.ekin_tot = ekin;
    o.ekin_atom = ekin / N;
    double mom2 = 0.;
    for (int a = 0; a < 3; ++a) {
        o.momentum_tot[a] = S * sf[F_MV + a];
        mom2 += o.momentum_tot[a] * o.momentum_tot[a];
    }
    if (mom2 / (2. * R->mass0 * ekin) > 1e-14)
        atomicOr(&o.status, MDELAST_FATAL_MOMENTUM);
    o.epot_atom = sf[F_EPOT] / N;
    o.epot_eam_atom = sd[D_FSUM] / N;
    o.etot_atom = o.ekin_atom + o.epot_atom;
    double const old = o.etot_cons;
    double etot = o.etot_atom * N;
    if (ens == MDELAST_NVT || ens == MDELAST_NPT)
        etot += chain_etot(R->th);
    double const V = volume(R->h);
    if (ens == MDELAST_NPT)
        etot += V * R->baro_P + (0.5 * (R->p_eps * R->p_eps) / R->baro_w + chain_etot(R->bth));
    o.etot_cons = etot;
    double const e0 = mode == POST_INIT ? 0. : R->etot_cons_initial;
    o.etot_cons_err = fabs(etot / e0 - 1.);
    double const err_current = fabs(etot / old - 1.);
    o.temperature_kin = 2. * ekin / (kBoltz * R->Nf);
    if (obs) {
        double const f2 = sf[F_F2];
        o.total_force2 = f2;
        o.temperature_conf_inverse =
            (f2 != 0. && o.total_laplacian != 0.) ? kBoltz * o.total_laplacian / f2 : 0.;
    }
    o.pressure = (ekin * 2. / 3. + virial) / V;
    double const S2 = S * S;
    for (int k = 0; k < 6; ++k) {
        o.stress_tensor[k] = (-sf[F_SIGMA + k] + S2 * sf[F_MVV + k]) / V;
        o.born_stress_tensor[k] = sf[F_SIGMA + k] / V;
    }
    double const p_trace = o.stress_tensor[0] + o.stress_tensor[1] + o.stress_tensor[2];
    if (fabs(o.pressure / (p_trace / 3.) - 1.) > 1e-5)
        atomicOr(&o.status, MDELAST_FATAL_PRESSURE);
    if ((o.etot_cons_err > R->fatal_conservation || err_current > R->fatal_conservation) &&
        R->cycle > 0.)
        atomicOr(&o.status, MDELAST_FATAL_CONSERVATION);
    if (mode == POST_STEP) {
        R->time += dt;
        R->cycle += 1.;
    } else {
        R->etot_cons_initial = etot;
        o.etot_cons_initial = etot;
    }
    o.etot_cons_initial = R->etot_cons_initial;
    o.time = R->time;
    o.cycle = R->cycle;
    for (int a = 0; a < 3; ++a) {
        for (int b = 0; b < 3; ++b)
            o.box[3 * a + b] = a == b ? R->h[a] : 0.;
    }
    o.baro_epsilon = R->eps;
    o.baro_p_epsilon = R->p_eps;
    o.sample_observables = obs;
    R->sub_force = 0; // a forced pair-list refresh has run by now
}

} // namespace mdelast
