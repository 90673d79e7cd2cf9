// Mixed-precision pair passes: pair geometry and table evaluation in FP32, in angstrom and
// eV, with every sum over pairs (per-atom densities, forces and energies, the virial, Born
// stress, Born tensor and Laplacian) accumulated in FP64 and converted to cgs at the end;
// the per-atom helpers g_i and h_i of the density pass are summed in FP32 along the row.
//
// Pair forces stay exactly antisymmetric: dp_ij = -dp_ji bit for bit (IEEE subtraction and
// round-to-nearest-even are odd functions), every other pair quantity depends on r only,
// and the two EAM cross terms of dE/dr are rounded separately and added commutatively.
// With the per-atom sums in FP64 the total momentum is conserved as in the FP64 path.
//
// The neighbour list, the embedding function and the integrator are shared with the FP64
// path (FP64, cgs): the list comes from the FP64 coordinates, and k_kick_drift refreshes
// the FP32 positions posf after every drift.
#include "kernels.cuh"
#include "pair_common.cuh"

namespace mdelast {

namespace {

__device__ __forceinline__ int tab_locate_f(float x, float inv_h, int n, float &t) {
    float const u = __fmul_rn(x, inv_h);
    int i = 0;
    if (u >= static_cast<float>(n))
        i = n - 1;
    else if (u > 0.f)
        i = static_cast<int>(u);
    t = __fsub_rn(u, static_cast<float>(i));
    return i;
}

// the 6 quintic coefficients of a packed (8-byte aligned) record
__device__ __forceinline__ void ld6f(const float *p, float c[6]) {
    const float2 *q = reinterpret_cast<const float2 *>(p);
    float2 const a = __ldg(q), b = __ldg(q + 1), d = __ldg(q + 2);
    c[0] = a.x;
    c[1] = a.y;
    c[2] = b.x;
    c[3] = b.y;
    c[4] = d.x;
    c[5] = d.y;
}

// The pair force is evaluated from both of its atoms, in different code paths of the
// force pass; its arithmetic is written with explicit rounding (no contraction left to
// the compiler) so that both evaluations give the same bits.
__device__ __forceinline__ float tabf_v(const float *c, float t) {
    return c[0] + t * (c[1] + t * (c[2] + t * (c[3] + t * (c[4] + t * c[5]))));
}
__device__ __forceinline__ float tabf_d1(const float *c, float t, float inv_h) {
    float p = __fmul_rn(5.f, c[5]);
    p = __fmaf_rn(t, p, __fmul_rn(4.f, c[4]));
    p = __fmaf_rn(t, p, __fmul_rn(3.f, c[3]));
    p = __fmaf_rn(t, p, __fmul_rn(2.f, c[2]));
    p = __fmaf_rn(t, p, c[1]);
    return __fmul_rn(p, inv_h);
}
__device__ __forceinline__ float tabf_d2(const float *c, float t, float inv_h2) {
    return (2.f * c[2] + t * (6.f * c[3] + t * (12.f * c[4] + t * 20.f * c[5]))) * inv_h2;
}

// FP32 counterpart of tab_eval (device.cuh): QUINTIC interval data are the 6 quintic
// coefficients, BSPLINE data three cubics (values of the splines of f, f', f''); both with
// explicit rounding.
__device__ __forceinline__ float cubicf_at(const float *p, float t) {
    float4 const a = __ldg(reinterpret_cast<const float4 *>(p));
    return __fmaf_rn(t, __fmaf_rn(t, __fmaf_rn(t, a.w, a.z), a.y), a.x);
}

template <int IP, bool NV, bool ND1, bool ND2>
__device__ __forceinline__ void tabf_eval(const float *p, float t, float inv_h, float inv_h2,
                                          float &v, float &d1, float &d2) {
    if constexpr (IP == MDELAST_BSPLINE) {
        if (NV)
            v = cubicf_at(p, t);
        if (ND1)
            d1 = cubicf_at(p + 4, t);
        if (ND2)
            d2 = cubicf_at(p + 8, t);
    } else {
        float c[6];
        ld6f(p, c);
        if (NV)
            v = tabf_v(c, t);
        if (ND1)
            d1 = tabf_d1(c, t, inv_h);
        if (ND2)
            d2 = tabf_d2(c, t, inv_h2);
    }
}

} // namespace

// FP32 wrapped positions of every atom from the FP64 coordinates and the current box.
__global__ void k_posf(AtomsView A) {
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n_pad)
        return;
    int const r = A.rep_of[i];
    if (r < 0)
        return;
    Replica const *R = A.rep + r;
    double4 const c = A.crd[i];
    A.posf[i] = make_float4(static_cast<float>((c.x - nint_ref(c.x)) * R->h[0] / kAng),
                            static_cast<float>((c.y - nint_ref(c.y)) * R->h[1] / kAng),
                            static_cast<float>((c.z - nint_ref(c.z)) * R->h[2] / kAng),
                            static_cast<float>(c.w));
}

// One lane's share of an atom row in the density pass: branch-free body, two entries per
// unrolled pass, as in the force pass; an entry beyond the cutoff adds zeros. UC: every
// density cutoff is at least the pair cutoff (no per-type test).
template <bool OBS, int TPA, int IP, typename IX, bool UC>
__device__ __forceinline__ void dens_loop(AtomsView const &A, TablesView const &T, float4 pi,
                                          float3 L, float3 iL, PairRow<IX> const &row, int nu,
                                          int ntot, int sub, double &rho, float (&g)[6],
                                          float (&hv)[3]) {
    // the next partner's record and the list entry after it are loaded ahead, so the
    // entry's load does not delay the record's
    float4 pn = A.posf[sub < ntot ? row.at(list_slot(sub, nu, A.pmaxn)) : row.base];
    int jn = sub < ntot ? row.at(list_slot(min(sub + TPA, ntot - 1), nu, A.pmaxn)) : row.base;
#pragma unroll 2
    for (int kk = sub; kk < ntot; kk += TPA) {
        float4 const pj = pn;
        pn = A.posf[jn];
        jn = row.at(list_slot(min(kk + 2 * TPA, ntot - 1), nu, A.pmaxn));
        float dx, dy, dz;
        float const r2 = min_image_f(pi, pj, L, iL, dx, dy, dz);
        float const idr = rsqrtf(r2);
        float const dr = __fmul_rn(r2, idr);
        int const tj = static_cast<int>(pj.w);
        bool const in_cut = !(r2 > T.fr_cut_sq) && (UC || !(dr > T.feam_rcut[tj]));
        float t;
        int const k = tab_locate_f(dr, T.finv_hr, T.nri, t);
        float v = 0.f, d1 = 0.f, d2 = 0.f;
        tabf_eval<IP, true, OBS, false>(
            T.rrf + (static_cast<size_t>(tj) * T.nri + k) * TabFmt<IP>::kFf, t, T.finv_hr,
            T.finv_hr2, v, d1, d2);
        if (!in_cut) {
            v = 0.f;
            d1 = 0.f;
        }
        rho += static_cast<double>(v);
        if (OBS) {
            float const ar = d1 * idr;
            float const ap[3] = {ar * dx, ar * dy, ar * dz};
            g[0] += ap[0] * dx;
            g[1] += ap[1] * dy;
            g[2] += ap[2] * dz;
            g[3] += ap[1] * dz;
            g[4] += ap[0] * dz;
            g[5] += ap[0] * dy;
            hv[0] += ap[0];
            hv[1] += ap[1];
            hv[2] += ap[2];
        }
    }
}

// Density pass of md_driver.cpp:195-277 in mixed precision (see k_density for the roles).
// The block's FP64 sums (embedding energy, the per-atom Born term F''_i g_i g_i^T and
// Laplacian term) are folded warp by warp after each atom group into per-warp shared
// accumulators instead of being carried in registers through the pair loop: the loop then
// runs with about half the registers, so twice the warps per SM hide the latency of the
// partner gathers.
//
// Bounded to 8 blocks of 128 threads per SM (64 registers; the compiler's own choice is 72,
// 7 blocks): a few bytes of spills, and the extra warps hide more of the gather latency
// (0.194 -> 0.182 ms at 16 x 13,500 atoms; 9 and 10 blocks spilled more and ran slower).
template <bool OBS, int TPA, int IP, typename IX>
__global__ void __launch_bounds__(kBlock, 8) k_density_mx(AtomsView A, TablesView T) {
    if (halted(A)) // a list build ran out of capacity: nothing until the host regrows
        return;
    constexpr int kF = TabFmt<IP>::kF;
    __shared__ double sacc[kBlock / 32][D_NSUM];
    int const warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < (kBlock / 32) * D_NSUM; k += kBlock)
        (&sacc[0][0])[k] = 0.;
    __syncthreads();
    int const r = A.dblk_rep[blockIdx.x];
    Replica const *R = A.rep + r;
    int const lb = blockIdx.x - R->dblk_begin, nb = R->dblk_n;
    int const apb = kBlock / TPA, sub = threadIdx.x % TPA;
    int const n_slots = R->n_blocks * kBlock;
    float3 L, iL;
    box_f(R, L, iL);
    double const a3 = kAng * kAng * kAng;
    for (int a0 = lb * apb; a0 < n_slots; a0 += nb * apb) {
        int const a = a0 + static_cast<int>(threadIdx.x) / TPA;
        int const i = R->atom_begin + a;
        bool const valid = a < R->n_atoms && T.has_eam;
        double rho = 0.;
        float g[6] = {0, 0, 0, 0, 0, 0}, hv[3] = {0, 0, 0};
        int ti = 0;
        if (valid) {
            float4 const pi = A.posf[i];
            ti = static_cast<int>(pi.w);
            int const nu = A.pn_up[i], ntot = nu + A.pn_dn[i];
            PairRow<IX> const row = pair_row<IX>(A, i, R->atom_begin);
            // uniform cutoffs (every setfl potential): no per-function cutoff test
            if (T.fuc)
                dens_loop<OBS, TPA, IP, IX, true>(A, T, pi, L, iL, row, nu, ntot, sub, rho, g, hv);
            else
                dens_loop<OBS, TPA, IP, IX, false>(A, T, pi, L, iL, row, nu, ntot, sub, rho, g,
                                                   hv);
        }
        rho = group_sum<TPA>(rho);
        if (OBS) {
#pragma unroll
            for (int u = 0; u < 6; ++u)
                g[u] = group_sum<TPA>(g[u]);
#pragma unroll
            for (int u = 0; u < 3; ++u)
                hv[u] = group_sum<TPA>(hv[u]);
        }
        double F = 0., d2F = 0.;
        bool const own = valid && sub == 0;
        if (own) {
            // the embedding function in FP64 and cgs (eam.hpp:48-70)
            double const rc = rho / a3;
            if (rc > T.rhomax[ti])
                status_or(A.rep + r, MDELAST_FATAL_RHO_MAX);
            double t;
            int const k = tab_locate(rc, T.inv_hf, T.nfi, t);
            double dF = 0.;
            tab_eval<IP, true, true, OBS>(T.Ft + (static_cast<size_t>(ti) * T.nfi + k) * kF, t,
                                          T.inv_hf, T.inv_hf2, F, dF, d2F);
            A.rho[i] = rc;
            A.Fe[i] = F;
            // F' [erg cm^3] -> [eV A^3] and F'' [erg cm^6] -> [eV A^6]
            if (OBS) {
                A.dF2[i] = make_double2(dF, d2F);
                A.dF2f[i] = make_float2(static_cast<float>(dF / (a3 * kEv)),
                                        static_cast<float>(d2F / (a3 * a3 * kEv)));
            } else {
                A.dF2[i].x = dF;
                A.dF2f[i].x = static_cast<float>(dF / (a3 * kEv));
            }
        }
        warp_accumulate(F, &sacc[warp][D_FSUM]);
        if (OBS) {
            // g in cm^-3 and h in cm^-4, as the cgs F'' expects; zero for lanes without an atom
            double gc[6];
#pragma unroll
            for (int u = 0; u < 6; ++u)
                gc[u] = own ? static_cast<double>(g[u]) / a3 : 0.;
            int q = D_CB;
#pragma unroll
            for (int u = 0; u < 6; ++u)
#pragma unroll
                for (int v = u; v < 6; ++v)
                    warp_accumulate(d2F * gc[u] * gc[v], &sacc[warp][q++]);
            double const ha = a3 * kAng;
            double const h0 = hv[0] / ha, h1 = hv[1] / ha, h2 = hv[2] / ha;
            warp_accumulate(own ? d2F * (h0 * h0 + h1 * h1 + h2 * h2) : 0., &sacc[warp][D_LAP]);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < D_NSUM; k += blockDim.x) {
        double s = 0.;
#pragma unroll
        for (int w = 0; w < kBlock / 32; ++w)
            s += sacc[w][k];
        A.pd[static_cast<size_t>(blockIdx.x) * D_NSUM + k] = s;
    }
}

// Sums over the pairs of one lane's share of an atom row, added into the FP64 block
// accumulators once per row. The diagonal Born stress is summed in FP64 pair by pair and
// the virial is taken as its trace (the sum over pairs of dE/dr r equals that of
// dE/dr x_a^2 / r): the reference checks the virial against the stress trace to 1e-7 and
// the pressure against the stress trace to 1e-5 (md_driver.cpp:422-429, 693-698), and near
// zero pressure, where kinetic and virial parts cancel, that holds only if both come from
// the same FP32 pair terms. The off-diagonal stress, Born tensor and Laplacian terms are
// summed in FP32 along the row (at most ~20 FP32 terms, no error beyond the terms' own)
// and in FP64 across rows and atoms.
template <bool OBS> struct PairSums {
    double sig_d[3] = {0., 0., 0.};
    float sig_o[3] = {0, 0, 0};
    float cb[OBS ? 15 : 1] = {};
    float lap = 0.f;
};

// Per-atom inputs of one row of the force pass.
struct RowIn {
    float4 pi;
    float dFi, d2Fi;
    int ti;
    float3 L, iL;
};

// The quintic coefficients of phi_s, rho_ti and rho_tj on interval k: from the staged
// shared-memory copy (STAGED and k staged) or from the global pair bundle. Both hold the
// same FP32 values, so the pair terms do not depend on where they were read.
template <bool STAGED>
__device__ __forceinline__ void pair_coefs(TablesView const &T, const float *stab, int s,
                                           int ti, int tj, int k, float cp[6], float ci[6],
                                           float cj[6]) {
    if (STAGED) {
        unsigned const q = static_cast<unsigned>(k - T.st_lo);
        if (q < static_cast<unsigned>(T.st_n)) {
            int const n6 = 6 * T.st_n;
            const float *b = stab + 6 * q;
            const float2 *pp = reinterpret_cast<const float2 *>(b + s * n6);
            const float2 *pi = reinterpret_cast<const float2 *>(b + (T.npot + ti) * n6);
            const float2 *pj = reinterpret_cast<const float2 *>(b + (T.npot + tj) * n6);
#pragma unroll
            for (int u = 0; u < 3; ++u) {
                float2 const a = pp[u], c = pi[u], d = pj[u];
                cp[2 * u] = a.x;
                cp[2 * u + 1] = a.y;
                ci[2 * u] = c.x;
                ci[2 * u + 1] = c.y;
                cj[2 * u] = d.x;
                cj[2 * u + 1] = d.y;
            }
            return;
        }
    }
    constexpr int kFb = TabFmt<MDELAST_QUINTIC>::kFb;
    const float *bundle = T.rbf + (static_cast<size_t>(s) * T.nri + k) * TabFmt<MDELAST_QUINTIC>::kB;
    // rho_a of the bundle belongs to the smaller type of the pair
    int const oi = (ti <= tj) ? kFb : 2 * kFb, oj = (ti < tj) ? 2 * kFb : kFb;
    ld6f(bundle, cp);
    ld6f(bundle + oi, ci);
    ld6f(bundle + oj, cj);
}

// One lane's walk over list slots [s0, s1) of an atom row (slots of partners j > i when
// UPPER, else of partners j < i, addressed from the end of the row); every pair adds its
// force and half its energy to the atom, and pairs j > i also add to the global sums.
// STAGED: quintic tables read from the staged shared-memory copy `stab` where staged.
template <bool OBS, bool UPPER, int TPA, int IP, bool STAGED, typename IX, bool UC>
__device__ __forceinline__ void force_row_mx(AtomsView const &A, TablesView const &T,
                                             RowIn const &in, PairRow<IX> const &row, int n,
                                             int sub,
                                             double &fx, double &fy, double &fz, double &epot,
                                             PairSums<OBS> &ps, bool &warn_rmin,
                                             const float *stab = nullptr) {
    if (sub >= n)
        return;
    auto slot = [&](int k) { return UPPER ? k : A.pmaxn - 1 - k; };
    // the row's entries are read once per pass: streaming loads (evict first), so that
    // they do not push the table and the partner records out of the L1 (measured: step
    // 1.025 -> 0.987 ms at 16 x 13,500 atoms)
    int jn = row.at(slot(sub));
    float4 pn = A.posf[jn];
    float2 fn = A.dF2f[jn];
    jn = row.at(slot(min(sub + TPA, n - 1)));
    // The body has no branch: a pair beyond the cutoff is evaluated and its terms are
    // replaced by zeros (the sums then gain +0 or -0, which changes no sum), and the next
    // partner is always prefetched (the last one again at the end of the row). Two
    // iterations then form one block of straight-line code, in which the second pair's
    // gathers and table loads overlap the first pair's arithmetic.
#pragma unroll 2
    for (int kk = sub; kk < n; kk += TPA) {
        float4 const pj = pn;
        float2 const dFj2 = fn;
        pn = A.posf[jn];
        fn = A.dF2f[jn];
        jn = row.at(slot(min(kk + 2 * TPA, n - 1)));
        float dx, dy, dz;
        float const r2 = min_image_f(in.pi, pj, in.L, in.iL, dx, dy, dz);
        bool const in_cut = !(r2 > T.fr_cut_sq);
        float const idr = rsqrtf(r2);
        float const dr = __fmul_rn(r2, idr);
        int const tj = static_cast<int>(pj.w);
        int const ti = in.ti;
        int const s = pair_slot(ti, tj);
        float t;
        int const k = tab_locate_f(dr, T.finv_hr, T.nri, t);
        constexpr int kFb = TabFmt<IP>::kFb;
        float V = 0.f, dV = 0.f, d2V = 0.f;
        float drho_i = 0.f, drho_j = 0.f, d2rho_i = 0.f, d2rho_j = 0.f;
        if (in_cut && dr < T.fpot_rmin[s])
            warn_rmin = true;
        bool const eam_i = T.has_eam && (UC || !(dr > T.feam_rcut[ti]));
        bool const eam_j = T.has_eam && (UC || !(dr > T.feam_rcut[tj]));
        if constexpr (IP == MDELAST_QUINTIC) {
            // the three functions' coefficients first (independent loads), then the math
            float cp[6], ci[6], cj[6];
            pair_coefs<STAGED>(T, stab, s, ti, tj, k, cp, ci, cj);
            if (UC || !(dr > T.fpot_rcut[s])) {
                V = tabf_v(cp, t);
                dV = tabf_d1(cp, t, T.finv_hr);
                if (OBS)
                    d2V = tabf_d2(cp, t, T.finv_hr2);
            }
            if (eam_i) {
                drho_i = tabf_d1(ci, t, T.finv_hr);
                if (OBS)
                    d2rho_i = tabf_d2(ci, t, T.finv_hr2);
            }
            if (eam_j) {
                drho_j = tabf_d1(cj, t, T.finv_hr);
                if (OBS)
                    d2rho_j = tabf_d2(cj, t, T.finv_hr2);
            }
        } else {
            const float *bundle = T.rbf + (static_cast<size_t>(s) * T.nri + k) * TabFmt<IP>::kB;
            if (UC || !(dr > T.fpot_rcut[s]))
                tabf_eval<IP, true, true, OBS>(bundle, t, T.finv_hr, T.finv_hr2, V, dV, d2V);
            // rho'_{t_i} and rho'_{t_j} at r: rho_a of the bundle belongs to the smaller type
            int const oi = (ti <= tj) ? kFb : 2 * kFb, oj = (ti < tj) ? 2 * kFb : kFb;
            float unused = 0.f;
            if (eam_i)
                tabf_eval<IP, false, true, OBS>(bundle + oi, t, T.finv_hr, T.finv_hr2, unused,
                                                drho_i, d2rho_i);
            if (eam_j)
                tabf_eval<IP, false, true, OBS>(bundle + oj, t, T.finv_hr, T.finv_hr2, unused,
                                                drho_j, d2rho_j);
        }
        float dedr = dV, X = 0.f, lap = 0.f;
        if (OBS) {
            X = d2V - dV * idr;
            lap = 2.f * (d2V + 2.f * dV * idr);
        }
        if (T.has_eam) {
            float const dFj = dFj2.x, dFi = in.dFi;
            // the two cross terms rounded separately and added commutatively: the pair
            // force is the same, bit for bit, seen from either atom
            dedr = __fadd_rn(dedr, __fadd_rn(__fmul_rn(dFi, drho_j), __fmul_rn(dFj, drho_i)));
            if (OBS && UPPER) {
                float const d2Fj = dFj2.y, d2Fi = in.d2Fi;
                lap += 2.f * (dFj * (d2rho_i + 2.f * drho_i * idr) +
                              dFi * (d2rho_j + 2.f * drho_j * idr));
                lap += d2Fi * (drho_j * drho_j) + d2Fj * (drho_i * drho_i);
                X += dFi * (d2rho_j - drho_j * idr) + dFj * (d2rho_i - drho_i * idr);
            }
        }
        if (!in_cut) {
            dedr = 0.f;
            V = 0.f;
            X = 0.f;
            lap = 0.f;
        }
        float const sc = __fmul_rn(-dedr, idr);
        fx += static_cast<double>(__fmul_rn(sc, dx));
        fy += static_cast<double>(__fmul_rn(sc, dy));
        fz += static_cast<double>(__fmul_rn(sc, dz));
        epot += static_cast<double>(0.5f * V);
        if (UPPER) {
            float const xx = dx * dx, yy = dy * dy, zz = dz * dz;
            float const yz = dy * dz, xz = dx * dz, xy = dx * dy;
            float const w = dedr * idr;
            ps.sig_d[0] += static_cast<double>(w * xx);
            ps.sig_d[1] += static_cast<double>(w * yy);
            ps.sig_d[2] += static_cast<double>(w * zz);
            ps.sig_o[0] += w * yz;
            ps.sig_o[1] += w * xz;
            ps.sig_o[2] += w * xy;
            if (OBS) {
                X *= idr * idr;
                float const Xxx = X * xx, Xyy = X * yy, Xzz = X * zz;
                ps.cb[0] += Xxx * xx;
                ps.cb[1] += Xyy * yy;
                ps.cb[2] += Xzz * zz;
                ps.cb[3] += Xxx * xy;
                ps.cb[4] += Xxx * xz;
                ps.cb[5] += Xyy * xy;
                ps.cb[6] += Xyy * yz;
                ps.cb[7] += Xzz * xz;
                ps.cb[8] += Xzz * yz;
                ps.cb[9] += Xxx * yy;
                ps.cb[10] += Xxx * zz;
                ps.cb[11] += Xyy * zz;
                ps.cb[12] += Xxx * yz;
                ps.cb[13] += Xyy * xz;
                ps.cb[14] += Xzz * xy;
                ps.lap += lap;
            }
        }
    }
}

// Force pass of md_driver.cpp:300-430 (with the closing kick) in mixed precision; see
// k_force for the roles of the terms. Each atom row is walked in two loops, partners j > i
// (which also feed the global sums) and partners j < i, so the lanes of a warp do not
// diverge on the global-sum work. The FP64 block accumulators live in shared memory
// (slot-major), one set per group of TPA lanes: each atom's pair sums are combined across
// its lanes in FP64 first, which keeps the accumulators at 36 slots per group instead of
// per thread (5.6 KB instead of 37 KB per block at 8 lanes per atom) and leaves that
// shared memory to the L1 that caches the tables (measured 2-4 % faster).
//
// STAGED: the block first copies the staged quintic tables (T.stf, T.st_bytes, about 180 KB
// for a two-element alloy) into dynamic shared memory and reads every staged interval from
// there, so table lookups no longer compete with the partner gathers for the L1 and never
// miss to the L2. One such block fills an SM's shared memory, so it is NB = kBlockStaged
// threads wide. Per-atom results equal the unstaged kernel's bit for bit; the global sums
// differ only in the grouping of their FP64 partial sums.
constexpr int kBlockStaged = kStagedBlock;

template <bool OBS, bool KICK, int TPA, int IP, bool STAGED, typename IX,
          int NB = STAGED ? kBlockStaged : kBlock>
__global__ void __launch_bounds__(NB) k_force_mx(AtomsView A, TablesView T) {
    if (halted(A)) // a list build ran out of capacity: nothing until the host regrows
        return;
    constexpr int kG = NB / TPA;
    __shared__ double s_acc[F_NSUM * kG];
    extern __shared__ float4 s_stage[];
    int const tid = threadIdx.x, grp = tid / TPA;
    for (int k = tid; k < F_NSUM * kG; k += NB)
        s_acc[k] = 0.;
    if (STAGED) {
        const float4 *src = reinterpret_cast<const float4 *>(T.stf);
        int const n16 = T.st_bytes / 16;
        for (int k = tid; k < n16; k += NB)
            s_stage[k] = __ldg(src + k);
    }
    __syncthreads();
    const float *stab = reinterpret_cast<const float *>(s_stage);
    int const r = A.fblk_rep[blockIdx.x];
    Replica const *R = A.rep + r;
    int const lb = blockIdx.x - R->fblk_begin, nb = R->fblk_n;
    int const apb = NB / TPA, sub = tid % TPA;
    int const n_slots = R->n_blocks * kBlock;
    RowIn in;
    box_f(R, in.L, in.iL);
    for (int a0 = lb * apb; a0 < n_slots; a0 += nb * apb) {
        int const a = a0 + tid / TPA;
        int const i = R->atom_begin + a;
        bool const valid = a < R->n_atoms;
        double fx = 0., fy = 0., fz = 0., epot = 0.;
        double sums[F_F2]; // this atom's pair sums (virial, Born stress, tensor, Laplacian)
#pragma unroll
        for (int k = 0; k < F_F2; ++k)
            sums[k] = 0.;
        in.ti = 0;
        if (valid) {
            in.pi = A.posf[i];
            in.ti = static_cast<int>(in.pi.w);
            float2 const dFi2 = T.has_eam ? A.dF2f[i] : make_float2(0.f, 0.f);
            in.dFi = dFi2.x;
            in.d2Fi = OBS ? dFi2.y : 0.f;
            int const nu = A.pn_up[i], nd = A.pn_dn[i];
            PairRow<IX> const row = pair_row<IX>(A, i, R->atom_begin);
            bool warn_rmin = false;
            PairSums<OBS> ps;
            // uniform cutoffs (every setfl potential): no per-function cutoff tests
            if (T.fuc) {
                force_row_mx<OBS, true, TPA, IP, STAGED, IX, true>(
                    A, T, in, row, nu, sub, fx, fy, fz, epot, ps, warn_rmin, stab);
                force_row_mx<OBS, false, TPA, IP, STAGED, IX, true>(
                    A, T, in, row, nd, sub, fx, fy, fz, epot, ps, warn_rmin, stab);
            } else {
                force_row_mx<OBS, true, TPA, IP, STAGED, IX, false>(
                    A, T, in, row, nu, sub, fx, fy, fz, epot, ps, warn_rmin, stab);
                force_row_mx<OBS, false, TPA, IP, STAGED, IX, false>(
                    A, T, in, row, nd, sub, fx, fy, fz, epot, ps, warn_rmin, stab);
            }
            if (warn_rmin)
                status_or(A.rep + r, MDELAST_WARN_RMIN);
            sums[F_VIRIAL] = (ps.sig_d[0] + ps.sig_d[1]) + ps.sig_d[2];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sums[F_SIGMA + k] = ps.sig_d[k];
                sums[F_SIGMA + 3 + k] = static_cast<double>(ps.sig_o[k]);
            }
            if (OBS) {
#pragma unroll
                for (int k = 0; k < 15; ++k)
                    sums[F_CB + k] = static_cast<double>(ps.cb[k]);
                sums[F_LAP] = static_cast<double>(ps.lap);
            }
        }
        fx = group_sum<TPA>(fx);
        fy = group_sum<TPA>(fy);
        fz = group_sum<TPA>(fz);
        epot = group_sum<TPA>(epot);
        constexpr int kPair = OBS ? F_F2 : F_CB; // the pair sums this step forms
#pragma unroll
        for (int k = 0; k < kPair; ++k)
            sums[k] = group_sum<TPA>(sums[k]);
        if (sub == 0) {
#pragma unroll
            for (int k = 0; k < kPair; ++k)
                s_acc[k * kG + grp] += sums[k];
        }
        if (valid && sub == 0) {
            double const kf = kEv / kAng; // eV/A -> dyn
            fx *= kf;
            fy *= kf;
            fz *= kf;
            epot *= kEv;
            if (T.has_eam)
                epot += A.Fe[i];
            size_t const np = A.n_pad;
            A.frc[i] = fx;
            A.frc[np + i] = fy;
            A.frc[np + i + np] = fz;
            A.epot[i] = epot;
            double const m = T.mass[in.ti];
            double vx = A.vel[i], vy = A.vel[np + i], vz = A.vel[2 * np + i];
            if (KICK) {
                double const e = R->e_kick, cdt = R->cdt_kick;
                vx = vx * e + cdt * fx / m;
                vy = vy * e + cdt * fy / m;
                vz = vz * e + cdt * fz / m;
                A.vel[i] = vx;
                A.vel[np + i] = vy;
                A.vel[2 * np + i] = vz;
            }
            double *acc = s_acc + grp;
            acc[F_F2 * kG] += fx * fx + fy * fy + fz * fz;
            acc[F_EKIN * kG] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
            acc[(F_MVV + 0) * kG] += m * vx * vx;
            acc[(F_MVV + 1) * kG] += m * vy * vy;
            acc[(F_MVV + 2) * kG] += m * vz * vz;
            acc[(F_MVV + 3) * kG] += m * vy * vz;
            acc[(F_MVV + 4) * kG] += m * vx * vz;
            acc[(F_MVV + 5) * kG] += m * vx * vy;
            acc[(F_MV + 0) * kG] += vx * m;
            acc[(F_MV + 1) * kG] += vy * m;
            acc[(F_MV + 2) * kG] += vz * m;
            acc[F_EPOT * kG] += epot;
        }
    }
    // the groups' slots into the block sums; pair sums from eV (and eV/A^2 for the
    // Laplacian) to cgs
    __syncthreads();
    double acc[F_NSUM];
#pragma unroll
    for (int k = 0; k < F_NSUM; ++k)
        acc[k] = tid < kG ? s_acc[k * kG + tid] : 0.;
    acc[F_VIRIAL] *= kEv;
#pragma unroll
    for (int k = 0; k < 6; ++k)
        acc[F_SIGMA + k] *= kEv;
#pragma unroll
    for (int k = 0; k < 15; ++k)
        acc[F_CB + k] *= kEv;
    acc[F_LAP] *= kEv / (kAng * kAng);
    block_sum_store<F_NSUM, NB>(acc, A.pf + static_cast<size_t>(blockIdx.x) * F_NSUM);
}

namespace {
template <bool OBS, int IP, typename IX>
void density_mx_tpa_ix(int tpa, int grid, cudaStream_t s, AtomsView const &A,
                       TablesView const &T) {
    switch (tpa) {
    case 1: k_density_mx<OBS, 1, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    case 4: k_density_mx<OBS, 4, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    case 8: k_density_mx<OBS, 8, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    default: k_density_mx<OBS, 16, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    }
}
template <bool OBS, int IP>
void density_mx_tpa(int tpa, int grid, cudaStream_t s, AtomsView const &A, TablesView const &T) {
    if (A.pnbr16)
        density_mx_tpa_ix<OBS, IP, uint16_t>(tpa, grid, s, A, T);
    else
        density_mx_tpa_ix<OBS, IP, int>(tpa, grid, s, A, T);
}
template <bool OBS, bool KICK, int IP, typename IX>
void force_mx_tpa_ix(int tpa, int grid, cudaStream_t s, AtomsView const &A,
                     TablesView const &T) {
    switch (tpa) {
    case 1: k_force_mx<OBS, KICK, 1, IP, false, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    case 4: k_force_mx<OBS, KICK, 4, IP, false, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    case 8: k_force_mx<OBS, KICK, 8, IP, false, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    default: k_force_mx<OBS, KICK, 16, IP, false, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    }
}
template <bool OBS, bool KICK, int IP>
void force_mx_tpa(int tpa, int grid, cudaStream_t s, AtomsView const &A, TablesView const &T) {
    if (A.pnbr16)
        force_mx_tpa_ix<OBS, KICK, IP, uint16_t>(tpa, grid, s, A, T);
    else
        force_mx_tpa_ix<OBS, KICK, IP, int>(tpa, grid, s, A, T);
}
// the staged kernels: lanes per atom 4, 8 or 16 (one lane per atom would need 143 KB of
// accumulators beside the tables)
template <bool OBS, bool KICK, typename IX>
void force_mx_staged_ix(int tpa, int grid, cudaStream_t s, AtomsView const &A,
                        TablesView const &T) {
    size_t const smem = static_cast<size_t>(T.st_bytes);
    constexpr int Q = MDELAST_QUINTIC;
    switch (tpa) {
    case 4: k_force_mx<OBS, KICK, 4, Q, true, IX><<<grid, kBlockStaged, smem, s>>>(A, T); break;
    case 8: k_force_mx<OBS, KICK, 8, Q, true, IX><<<grid, kBlockStaged, smem, s>>>(A, T); break;
    default:
        k_force_mx<OBS, KICK, 16, Q, true, IX><<<grid, kBlockStaged, smem, s>>>(A, T);
        break;
    }
}
template <bool OBS, bool KICK>
void force_mx_staged_tpa(int tpa, int grid, cudaStream_t s, AtomsView const &A,
                         TablesView const &T) {
    if (A.pnbr16)
        force_mx_staged_ix<OBS, KICK, uint16_t>(tpa, grid, s, A, T);
    else
        force_mx_staged_ix<OBS, KICK, int>(tpa, grid, s, A, T);
}
template <bool OBS, bool KICK, typename IX> cudaError_t staged_attr_ix(int bytes) {
    constexpr int Q = MDELAST_QUINTIC;
    cudaFuncAttribute const a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaFuncSetAttribute(k_force_mx<OBS, KICK, 4, Q, true, IX>, a, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_force_mx<OBS, KICK, 8, Q, true, IX>, a, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_force_mx<OBS, KICK, 16, Q, true, IX>, a, bytes);
    return e;
}
template <bool OBS, bool KICK> cudaError_t staged_attr(int bytes) {
    cudaError_t e = staged_attr_ix<OBS, KICK, int>(bytes);
    if (e == cudaSuccess)
        e = staged_attr_ix<OBS, KICK, uint16_t>(bytes);
    return e;
}
template <int IP>
void density_mx_ip(bool obs, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                   TablesView const &T) {
    if (obs)
        density_mx_tpa<true, IP>(tpa, grid, s, A, T);
    else
        density_mx_tpa<false, IP>(tpa, grid, s, A, T);
}
template <int IP>
void force_mx_ip(bool obs, bool kick, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                 TablesView const &T) {
    if (obs && kick)
        force_mx_tpa<true, true, IP>(tpa, grid, s, A, T);
    else if (obs)
        force_mx_tpa<true, false, IP>(tpa, grid, s, A, T);
    else if (kick)
        force_mx_tpa<false, true, IP>(tpa, grid, s, A, T);
    else
        force_mx_tpa<false, false, IP>(tpa, grid, s, A, T);
}
} // namespace

void launch_density_mx(bool obs, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                       TablesView const &T) {
    if (T.interp == MDELAST_BSPLINE)
        density_mx_ip<MDELAST_BSPLINE>(obs, tpa, grid, s, A, T);
    else
        density_mx_ip<MDELAST_QUINTIC>(obs, tpa, grid, s, A, T);
}

void launch_force_mx(bool obs, bool kick, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                     TablesView const &T) {
    if (T.interp == MDELAST_BSPLINE)
        force_mx_ip<MDELAST_BSPLINE>(obs, kick, tpa, grid, s, A, T);
    else
        force_mx_ip<MDELAST_QUINTIC>(obs, kick, tpa, grid, s, A, T);
}

void launch_force_mx_staged(bool obs, bool kick, int tpa, int grid, cudaStream_t s,
                            AtomsView const &A, TablesView const &T) {
    if (obs && kick)
        force_mx_staged_tpa<true, true>(tpa, grid, s, A, T);
    else if (obs)
        force_mx_staged_tpa<true, false>(tpa, grid, s, A, T);
    else if (kick)
        force_mx_staged_tpa<false, true>(tpa, grid, s, A, T);
    else
        force_mx_staged_tpa<false, false>(tpa, grid, s, A, T);
}

cudaError_t prepare_force_mx_staged(int smem_bytes) {
    cudaError_t e = staged_attr<true, true>(smem_bytes);
    if (e == cudaSuccess)
        e = staged_attr<true, false>(smem_bytes);
    if (e == cudaSuccess)
        e = staged_attr<false, true>(smem_bytes);
    if (e == cudaSuccess)
        e = staged_attr<false, false>(smem_bytes);
    return e;
}

} // namespace mdelast
