// Device-side layout of the mdelast B200 path: per-replica state, the atom arrays in HBM,
// and the inline helpers shared by the kernels.
//
// Layout (all arrays padded so that every replica starts on a multiple of kTile slots and
// no thread block straddles two replicas):
//   crd   double4[n_pad]   scaled coordinates (not wrapped, as md_driver.cpp:483-485 keeps
//                          them) and the type in .w - the one record a pair gather reads
//   vel   double[3][n_pad] velocities (SoA), times Replica::vscale (deferred NHC factor)
//   frc   double[3][n_pad] forces
//   rho, Fe, epot double[n_pad]; dF2 double2[n_pad] = (F'(rho), F''(rho))
//   nbr   int[n_pad][maxn] full neighbour list, atom-major (one contiguous row per atom,
//                          read by the atom's TPA lanes together): partners j > i from
//                          slot 0 up (n_up), j < i from slot maxn-1 down (n_dn)
//   rb    double[npot][nri][18] r-table bundle of each type pair (a <= b):
//                          phi_ab | rho_a | rho_b quintic coefficients of one interval
//   Ft    double[ntypes][nfi][6] embedding-function coefficients
#pragma once

#include <cstdint>

#include "mdelast.h"

namespace mdelast {

constexpr int kMaxChain = 16;
constexpr int kTile = 256;  // replica atom ranges start on multiples of kTile slots
constexpr int kBlock = 128; // threads per block of the atom kernels (divides kTile)
constexpr int kMaxTypes = 8;
constexpr int kChunk = 32;  // block sums folded per k_reduce block

// Slots of the per-block partial sums of the force pass.
enum FSlot : int {
    F_VIRIAL = 0,  // sum dr * dE/dr over pairs
    F_SIGMA = 1,   // 6 Born-stress components
    F_CB = 7,      // 15 degree-4 monomials of X_ij dp (pair part of the Born tensor)
    F_LAP = 22,    // pair part of the Laplacian
    F_F2 = 23,     // sum |F_i|^2
    F_EKIN = 24,   // sum m v^2 / 2 after the closing kick
    F_MVV = 25,    // 6 components of sum m v_a v_b
    F_MV = 31,     // 3 components of sum m v
    F_EPOT = 34,   // sum of per-atom potential energies
    F_NSUM = 35
};
// Slots of the per-block partial sums of the density pass.
enum DSlot : int {
    D_FSUM = 0, // sum of embedding energies F(rho_i)
    D_CB = 1,   // 21 upper-triangle entries of F''_i g_i g_i^T
    D_LAP = 22, // sum F''_i |h_i|^2
    D_NSUM = 23
};

struct Chain {
    double T, Nf;
    int n, pad;
    double q[kMaxChain], inv_q[kMaxChain], p_eta[kMaxChain], eta[kMaxChain];
};

struct Replica {
    // set at creation
    int atom_begin, n_atoms, block_begin, n_blocks; // slots [atom_begin, + n_blocks*kBlock)
    int dblk_begin, dblk_n, fblk_begin, fblk_n;     // blocks of the density / force pass
    int ensemble, coupling;
    int cell_begin, nc[3]; // cells per dimension for the list build (nc[0] == 0: all pairs)
    double Nf, alpha, dt, fatal_conservation, mass0;
    double baro_P, baro_w;
    double h0[3];
    // evolving scalar state
    double h[3];      // current box diagonal
    double h_pos[3];  // box the positions array refers to (before the last U1 box update)
    double eps, p_eps;
    double vscale;    // pending uniform factor of the stored velocities
    double s_kick, e_kick, cdt_kick, cfdt; // coefficients of this step's kick and drift
    double etot_cons_initial;
    double time, cycle;
    Chain th, bth;
    mdelast_observables obs;
    int initialised, pad2;
    // samples: records appended to the ring so far; fluctuation sums while acc_on
    double n_samples;
    int acc_on, pad3;
    mdelast_fluct acc;
    // pair list of the pair passes: largest squared displacement this step since its last
    // refresh, and a forced refresh (after a neighbour-list rebuild)
    double sub_d2;
    int sub_force, pad4;
};

struct TablesView {
    const double *rb; // [npot][nri][18]
    int nri, npot;
    double inv_hr, inv_hr2;
    const double *Ft; // [ntypes][nfi][6]
    int nfi, ntypes;
    double inv_hf, inv_hf2;
    int has_eam, interp; // interp: MDELAST_QUINTIC or MDELAST_BSPLINE (bundle layout)
    double r_cut_sq; // pow<2>(pot[0]->rcut), md_driver.cpp:42
    double pot_rcut[kMaxTypes * (kMaxTypes + 1) / 2];
    double pot_rmin[kMaxTypes * (kMaxTypes + 1) / 2];
    double eam_rcut[kMaxTypes];
    double rhomax[kMaxTypes];
    double mass[kMaxTypes];
    // mixed precision: the r tables in FP32 with lengths in angstrom and values in eV
    // (phi) or angstrom^-3 (rho). rbf: per type pair (a <= b) and interval one record of
    // TabFmt<IP>::kB floats holding phi_ab, rho_a, rho_b at strides of kFb (the force
    // pass reads all three at one r, from one place); rrf: per type and interval one
    // record of kFf floats holding rho (the density pass reads one function per pair).
    // Cutoffs in angstrom.
    const float *rbf, *rrf;
    float finv_hr, finv_hr2, fr_cut_sq, fpad;
    // Staged copy for the shared-memory force pass (quintic only): the intervals
    // [st_lo, st_lo + st_n) of every phi_ab (slot s at s * st_n) followed by every rho_a
    // (type a at (npot + a) * st_n), 6 floats each, de-duplicated (each rho once, not once
    // per type pair). st_n == 0: no staged copy. st_bytes: its size (a multiple of 16).
    const float *stf;
    int st_lo, st_n, st_bytes;
    // fuc: every function's FP32 cutoff is at least the pair cutoff, so no per-function
    // cutoff applies to a pair within it; the mixed passes then skip those tests. uc64: the
    // same in FP64, exactly: every cutoff is at least sqrt(r_cut_sq), the largest distance
    // the FP64 passes compute for a pair with r^2 <= r_cut_sq (sqrt is correctly rounded)
    int fuc, uc64;
    float fpot_rcut[kMaxTypes * (kMaxTypes + 1) / 2];
    float fpot_rmin[kMaxTypes * (kMaxTypes + 1) / 2];
    float feam_rcut[kMaxTypes];
};

// cgs <-> the angstrom / eV units of the mixed-precision kernels (units.hpp:6-24)
constexpr double kEv = 1.6021773e-12;
constexpr double kAng = 1e-8;

struct AtomsView {
    int n_pad, n_rep;
    Replica *rep;
    const int *rep_of; // replica of each slot, -1 for padding
    double4 *crd;
    double *vel, *frc; // [3][n_pad]
    double *rho, *Fe, *epot;
    double2 *dF2;
    float4 *posf; // mixed precision: wrapped positions [angstrom], type in .w (or null)
    float2 *dF2f; // mixed precision: F' [eV A^3], F'' [eV A^6]
    int *nbr, *n_up, *n_dn;
    int maxn;
    double *pd, *pf; // per-block partial sums [n_blocks][D_NSUM], [n_blocks][F_NSUM]
    double *red;     // chunk sums of pf/pd [n_rep][max_chunks][64] (k_reduce)
    int max_chunks, pad_red;
    const int *dblk_rep, *fblk_rep; // replica of each block of the density / force pass
    // cell list (list builds)
    int *cell_count, *cell_atoms;
    const int *cell_rep; // replica of each cell
    int cell_cap, n_cells;
    double r_list_sq;
    int *max_count; // [2]: largest neighbour count, largest cell count of the last build
    mdelast_sample *ring; // [n_rep][ring_cap] records of sampled steps (or null)
    int ring_cap, pad_ring;
    // The list the pair passes read: the neighbour list itself, or its pairs within
    // sub_r2 (squared radius, cm^2) kept since the coordinates crd_ref; refreshed once some
    // atom has moved by more than half the radius margin (sub_half2 = that half, squared).
    // pnbr16 (when not null) holds the pair list instead of pnbr, each entry the partner's
    // offset from its replica's first slot in 16 bits (replicas of at most 65,536 atoms):
    // half the bytes the pair passes read per pair.
    int *pnbr, *pn_up, *pn_dn;
    uint16_t *pnbr16;
    int pmaxn, pad_p;
    // Set (to 1) by a list build that ran out of neighbour or cell capacity. Every kernel
    // of a step returns at once while it is set, so the steps of a launch after an
    // overflowing in-step rebuild change nothing; the host grows the capacity and resumes
    // from the last completed step.
    int *halt;
    double4 *crd_ref;     // null: the pair passes read the neighbour list
    double sub_r2, sub_half2;
};

// md_driver.hpp:48-50: round half away from zero through a truncating int conversion
__device__ __forceinline__ double nint_ref(double x) {
    return static_cast<double>(x < 0. ? static_cast<int>(__dadd_rn(x, -0.5))
                                      : static_cast<int>(__dadd_rn(x, 0.5)));
}

// md_driver.cpp:175-185 with the reference's exact operations (no contraction):
// p = (d - nint(d)) * h for d = ci - cj, and r2 = (px*px + py*py) + pz*pz.
__device__ __forceinline__ double min_image_r2(double4 ci, double4 cj, double hx, double hy,
                                               double hz, double &px, double &py, double &pz) {
    double dx = __dadd_rn(ci.x, -cj.x), dy = __dadd_rn(ci.y, -cj.y), dz = __dadd_rn(ci.z, -cj.z);
    dx = __dadd_rn(dx, -nint_ref(dx));
    dy = __dadd_rn(dy, -nint_ref(dy));
    dz = __dadd_rn(dz, -nint_ref(dz));
    px = __dmul_rn(dx, hx);
    py = __dmul_rn(dy, hy);
    pz = __dmul_rn(dz, hz);
    return __dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)), __dmul_rn(pz, pz));
}

// Row i of the pair list in either entry width: at(k) is the atom slot of list slot k
// (partners j > i from slot 0 up, j < i from slot pmaxn - 1 down). IX = int: slots as stored;
// IX = uint16_t: offsets from the replica's first slot `base`. Loads stream (evict first):
// each row is read once per pass.
template <typename IX> struct PairRow {
    const IX *p;
    int base;
    __device__ __forceinline__ int at(int k) const {
        if constexpr (sizeof(IX) == 2)
            return base + static_cast<int>(__ldcs(p + k));
        else
            return __ldcs(p + k);
    }
};
template <typename IX>
__device__ __forceinline__ PairRow<IX> pair_row(AtomsView const &A, int i, int base) {
    const IX *p;
    if constexpr (sizeof(IX) == 2)
        p = A.pnbr16;
    else
        p = A.pnbr;
    return PairRow<IX>{p + static_cast<size_t>(i) * A.pmaxn, base};
}

__host__ __device__ __forceinline__ int pair_slot(int a, int b) {
    int const hi = a > b ? a : b, lo = a > b ? b : a;
    return hi * (hi + 1) / 2 + lo;
}

// poly_table.hpp:105-114: interval index clamped in floating point, local coordinate t.
__device__ __forceinline__ int tab_locate(double x, double inv_h, int n, double &t) {
    double const u = __dmul_rn(x, inv_h);
    int i = 0;
    if (u >= static_cast<double>(n))
        i = n - 1;
    else if (u > 0.)
        i = static_cast<int>(u);
    t = __dadd_rn(u, -static_cast<double>(i));
    return i;
}

// Horner forms of poly_table.hpp:71-97 on the 6 coefficients c of one interval.
__device__ __forceinline__ double tab_v(const double *c, double t) {
    return c[0] + t * (c[1] + t * (c[2] + t * (c[3] + t * (c[4] + t * c[5]))));
}
__device__ __forceinline__ double tab_d1(const double *c, double t, double inv_h) {
    return (c[1] + t * (2. * c[2] + t * (3. * c[3] + t * (4. * c[4] + t * 5. * c[5])))) * inv_h;
}
__device__ __forceinline__ double tab_d2(const double *c, double t, double inv_h2) {
    return (2. * c[2] + t * (6. * c[3] + t * (12. * c[4] + t * 20. * c[5]))) * inv_h2;
}

// load the 6 coefficients of one interval (16-byte aligned) through the read-only path
__device__ __forceinline__ void ld6(const double *p, double c[6]) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = __ldg(q), b = __ldg(q + 1), d = __ldg(q + 2);
    c[0] = a.x;
    c[1] = a.y;
    c[2] = b.x;
    c[3] = b.y;
    c[4] = d.x;
    c[5] = d.y;
}

// Interval data of one tabulated function in the two interpolation schemes
// (poly_table.hpp:137-176): QUINTIC, the 6 coefficients of the quintic in t from which
// value and derivatives all come (poly_table.hpp:71-97); BSPLINE, 12 = three cubics in t,
// the pieces of the three independent cubic B-splines through the node values of f, f'
// and f'' (poly_table.hpp:117-135), evaluated as values. kF is the per-function stride;
// a pair-table bundle holds three functions (phi_ab, rho_a, rho_b).
template <int IP> struct TabFmt {
    static constexpr int kF = IP == MDELAST_BSPLINE ? 12 : 6;
    // FP32 records of the mixed-precision tables, packed (a quintic's 6 coefficients in 24
    // bytes, 3 x 24 = 72 bytes per pair bundle): the pair passes are limited by how much of
    // the tables the L1 cache holds (measured: 96- and 128-byte bundles make the force pass
    // 7 % and 19 % slower; 32-byte rho records make the density pass 4.5 % slower).
    static constexpr int kFf = IP == MDELAST_BSPLINE ? 12 : 6;
    static constexpr int kFb = IP == MDELAST_BSPLINE ? 12 : 6;
    static constexpr int kB = 3 * kFb;
};

__device__ __forceinline__ double cubic_at(const double *p, double t) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 const a = __ldg(q), b = __ldg(q + 1);
    return a.x + t * (a.y + t * (b.x + t * b.y));
}

// value (NV), first (ND1) and second (ND2) derivative of the function whose interval data
// start at p; inv_h, inv_h2 scale the quintic's derivatives
template <int IP, bool NV, bool ND1, bool ND2>
__device__ __forceinline__ void tab_eval(const double *p, double t, double inv_h, double inv_h2,
                                         double &v, double &d1, double &d2) {
    if constexpr (IP == MDELAST_BSPLINE) {
        if (NV)
            v = cubic_at(p, t);
        if (ND1)
            d1 = cubic_at(p + 4, t);
        if (ND2)
            d2 = cubic_at(p + 8, t);
    } else {
        double c[6];
        ld6(p, c);
        if (NV)
            v = tab_v(c, t);
        if (ND1)
            d1 = tab_d1(c, t, inv_h);
        if (ND2)
            d2 = tab_d2(c, t, inv_h2);
    }
}

} // namespace mdelast
