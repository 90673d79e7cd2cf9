// Atom-parallel kernels of one MD step: neighbour-list build, density + embedding pass,
// force + closing-kick pass, opening kick + drift. One thread per atom slot; every
// replica's slots form whole blocks, so a block's partial sums belong to one replica.
// The full neighbour list makes the pair passes gather-only: no atomics, deterministic
// results, and forces that are antisymmetric pair by pair to the last bit.
#include "kernels.cuh"
#include "pair_common.cuh"

namespace mdelast {


// ------------------------------------------------------------------------------------
// neighbour list (md_driver.cpp:279-298): every pair with the reference's min-image
// |p|^2 <= (rcut r_skin)^2, found through a cell list (or all pairs when a replica has
// fewer than 3 list radii along an edge). Atoms are binned into half cells: 2 nc per edge
// for the nc = floor(h / (1.05 r_list)) cells no thinner than the list radius (with a margin
// for the box changes of an NPT run between rebuilds), so the partners of an atom lie in
// the 5 x 5 x 5 half cells around its own. The grid is fixed when a run starts; a barostat
// may shrink the box below it between builds, so each build takes, along every edge, the
// reach k (half cells either side) with k * h / nc >= the list radius in the current box.

// reach along one edge of h with nc (half) cells (2 while two half cells span the list
// radius, as they start)
__device__ __forceinline__ int cell_reach(double h, int nc, double rl2) {
    double const w = h / nc;
    int k = 1;
    while (k < nc && (k * w) * (k * w) < rl2)
        ++k;
    return k;
}

// the distinct cells of one edge the stencil spans from cell idx: count, and the first
// (all nc cells from 0 once 2k + 1 exceeds the edge)
__device__ __forceinline__ void cell_span(int idx, int nc, int k, int &first, int &count) {
    bool const fits = 2 * k + 1 <= nc;
    count = fits ? 2 * k + 1 : nc;
    first = fits ? idx - k : 0;
}

// the box has shrunk so far that two half cells no longer span the list radius (reach > 2
// along some edge; written without divisions, with a relative slack of 1e-12 towards
// calling the cells narrow)
__device__ __forceinline__ bool narrow_cells(Replica const &R, double rl2) {
    bool n = false;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        n = n || (R.nc[a] > 2 && 4. * R.h[a] * R.h[a] <= rl2 * R.nc[a] * R.nc[a] * (1. + 1e-12));
    return n;
}

__global__ void k_cell_bin(AtomsView A) {
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n_pad)
        return;
    int const r = A.rep_of[i];
    if (r < 0)
        return;
    Replica const &R = A.rep[r];
    if (R.nc[0] == 0)
        return;
    double4 const c = A.crd[i];
    double const w[3] = {c.x - nint_ref(c.x), c.y - nint_ref(c.y), c.z - nint_ref(c.z)};
    int idx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int k = static_cast<int>(floor((w[a] + 0.5) * R.nc[a]));
        idx[a] = k < 0 ? 0 : (k >= R.nc[a] ? R.nc[a] - 1 : k);
    }
    int const cell = R.cell_begin + (idx[2] * R.nc[1] + idx[1]) * R.nc[0] + idx[0];
    int const pos = atomicAdd(&A.cell_count[cell], 1);
    if (pos < A.cell_cap)
        A.cell_atoms[static_cast<size_t>(cell) * A.cell_cap + pos] = i;
    else {
        status_or(&A.rep[r], MDELAST_ERR_CELL_OVERFLOW);
        set_halt(A);
    }
}

// Order each cell's members by slot index (rank sort in shared memory), so that the list
// and everything summed over it are deterministic. One warp per half cell (about 8 atoms),
// blockDim.x / 32 cells per block.
__global__ void k_cell_sort(AtomsView A) {
    extern __shared__ int s_mem[];
    __shared__ int s_max; // the block's largest cell count: one global atomic per block
    int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int const cell = blockIdx.x * static_cast<int>(blockDim.x >> 5) + warp;
    if (threadIdx.x == 0)
        s_max = 0;
    __syncthreads();
    int n = cell < A.n_cells ? A.cell_count[cell] : 0;
    if (lane == 0)
        atomicMax(&s_max, n);
    __syncthreads();
    if (threadIdx.x == 0)
        atomicMax(&A.max_count[1], s_max);
    if (cell >= A.n_cells)
        return;
    if (n > A.cell_cap)
        n = A.cell_cap;
    int *src = s_mem + static_cast<size_t>(warp) * A.cell_cap;
    int *dst = A.cell_atoms + static_cast<size_t>(cell) * A.cell_cap;
    for (int k = lane; k < n; k += 32)
        src[k] = dst[k];
    __syncwarp();
    for (int k = lane; k < n; k += 32) {
        int const v = src[k];
        int rank = 0;
        for (int m = 0; m < n; ++m)
            rank += src[m] < v;
        dst[rank] = v;
    }
}

// One batch of up to 32 candidate partners j of atom i (one per lane): lanes with a hit
// store j in the atom's row, j > i from slot 0 up and j < i from slot maxn-1 down, in
// lane order, so the list is deterministic (cell stencil order, then slot order within a
// cell, which k_cell_sort fixed). nu/nd count the stored entries (nu + nd <= maxn, so the
// pair kernels never read an unwritten slot); total counts every partner found.
__device__ __forceinline__ void nb_batch(AtomsView const &A, int i, int j, bool hit,
                                         unsigned lane, int &nu, int &nd, int &total,
                                         bool &full) {
    bool const hu = hit && j > i, hd = hit && j < i;
    unsigned const up = __ballot_sync(0xffffffffu, hu);
    unsigned const dn = __ballot_sync(0xffffffffu, hd);
    int const cu = __popc(up), cd = __popc(dn);
    total += cu + cd;
    if (full || nu + nd + cu + cd > A.maxn) {
        full = true;
        return;
    }
    unsigned const lt = (1u << lane) - 1u;
    size_t const row = static_cast<size_t>(i) * A.maxn;
    if (hu)
        A.nbr[row + nu + __popc(up & lt)] = j;
    if (hd)
        A.nbr[row + (A.maxn - 1 - nd - __popc(dn & lt))] = j;
    nu += cu;
    nd += cd;
}

// Cell-list replicas: one block per group of 2 x 2 x 2 half cells (one cell of the
// coarse grid). The partners of the group's atoms all lie in the 6 x 6 x 6 half cells
// around it (its window), so their records are staged in shared memory once per group
// (in chunks of kStageH, window cells in z, y, x order, members in slot order) and each
// warp tests one atom at a time against them. An atom's partners lie in the 5 x 5 x 5 half
// cells around its own, and of those only the cells its list sphere reaches: per row of
// five half cells along x (fixed z, y) the warp takes the lower bound of the distance from
// the atom to the row, skips rows beyond the radius and trims the row's x range to the
// cells within it; each trimmed row is a contiguous run of staged records. On the 13,500-atom
// Cu-Zn cell that tests about 510 candidates per atom instead of the window's 1,690.
//
// Each candidate is first tested in FP32 on positions in the group's frame with a margin
// that covers the FP32 error, from outside (no pair within the radius is dropped) and from
// inside (a pair well within it needs no further test); the survivors are packed, in
// candidate order, into a per-warp queue, stored 32 at a time, and the few that lie within
// the error margin of the radius get the reference's exact FP64 test first. Rows, runs and
// members come in a fixed order, so the list is deterministic; the pairs kept are exactly
// those of the all-pairs search.
constexpr int kStageH = 2048;
constexpr int kWarpsH = kNbrCellsThreads / 32; // warps per block of k_nbr_cells
constexpr int kWin = 6;    // window edge, half cells
constexpr int kNearEdge = 1 << 30; // queue flag: the candidate needs the FP64 test

// lower bound (in half-cell widths) of the distance along one edge from an atom at
// fraction f of its half cell to the half cell d cells away; a small slack keeps the bound
// below the true distance under the FP32 rounding of f
__device__ __forceinline__ float cell_gap(int d, float f) {
    float const g = d > 0 ? static_cast<float>(d) - f
                          : (d < 0 ? static_cast<float>(-d - 1) + f : 0.f);
    return fmaxf(g - 1e-3f, 0.f);
}

__global__ void __launch_bounds__(kWarpsH * 32, 3) k_nbr_cells(AtomsView A) {
    extern __shared__ unsigned char s_raw[];
    float4 *s_w = reinterpret_cast<float4 *>(s_raw); // wrapped scaled, FP32
    int *s_j = reinterpret_cast<int *>(s_w + kStageH);
    int const cap = A.cell_cap, me_cap = 8 * cap;
    int *s_me = s_j + kStageH; // the group's atoms
    int *s_mq = s_me + me_cap; // ... and the window cell of each
    int *s_cnt = s_mq + me_cap; // [4][me_cap]: nu, nd, total, full of the group's atoms
    __shared__ int s_cell[kWin * kWin * kWin], s_off[kWin * kWin * kWin + 1], s_moff[9];
    __shared__ int s_tmax; // the group's largest neighbour count
    __shared__ int s_queue[kWarpsH][64]; // staged indices that passed the FP32 test
    int const r = A.cell_rep[8 * blockIdx.x];
    Replica const &R = A.rep[r];
    if (narrow_cells(R, A.r_list_sq))
        return;
    int const nx = R.nc[0], ny = R.nc[1], nz = R.nc[2];
    int const grp = blockIdx.x - R.cell_begin / 8;
    int const gx = grp % (nx / 2), gy = (grp / (nx / 2)) % (ny / 2),
              gz = grp / ((nx / 2) * (ny / 2));
    constexpr int kCells = kWin * kWin * kWin;
    for (int q = threadIdx.x; q < kCells; q += blockDim.x) {
        int const u = q % kWin, v = (q / kWin) % kWin, w = q / (kWin * kWin);
        int const cx = (2 * gx - 2 + u + nx) % nx, cy = (2 * gy - 2 + v + ny) % ny,
                  cz = (2 * gz - 2 + w + nz) % nz;
        int const c = R.cell_begin + (cz * ny + cy) * nx + cx;
        s_cell[q] = c;
        s_off[q + 1] = min(A.cell_count[c], cap);
    }
    __syncthreads();
    unsigned const lane = threadIdx.x & 31u;
    int const warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    unsigned const lt = (1u << lane) - 1u;
    if (warp == 0) {
        // exclusive scan of the window cells' counts; the group's 8 cells' counts
        int carry = 0;
        for (int b = 0; b < kCells; b += 32) {
            int const q = b + static_cast<int>(lane);
            int const c = q < kCells ? s_off[q + 1] : 0;
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int const t = __shfl_up_sync(0xffffffffu, incl, o);
                if (static_cast<int>(lane) >= o)
                    incl += t;
            }
            if (q < kCells)
                s_off[q + 1] = carry + incl;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0)
            s_off[0] = 0;
        __syncwarp();
        // the group's cells are the window cells with u, v, w in {2, 3}
        int const k = static_cast<int>(lane) & 7;
        int const q = ((2 + (k >> 2)) * kWin + 2 + ((k >> 1) & 1)) * kWin + 2 + (k & 1);
        int const c = s_off[q + 1] - s_off[q];
        int incl = c;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            int const t = __shfl_up_sync(0xffffffffu, incl, o);
            if ((static_cast<int>(lane) & 7) >= o)
                incl += t;
        }
        if (lane < 8)
            s_moff[k + 1] = incl;
        if (lane == 0) {
            s_moff[0] = 0;
            s_tmax = 0;
        }
    }
    __syncthreads();
    int const n_me = s_moff[8];
    for (int a = threadIdx.x; a < n_me; a += blockDim.x) {
        int k = 0;
        while (s_moff[k + 1] <= a)
            ++k;
        int const q = ((2 + (k >> 2)) * kWin + 2 + ((k >> 1) & 1)) * kWin + 2 + (k & 1);
        s_me[a] = A.cell_atoms[static_cast<size_t>(s_cell[q]) * cap + (a - s_moff[k])];
        s_mq[a] = q;
    }
    int *c_nu = s_cnt, *c_nd = s_cnt + me_cap, *c_tot = s_cnt + 2 * me_cap,
        *c_full = s_cnt + 3 * me_cap;
    for (int a = threadIdx.x; a < n_me; a += blockDim.x)
        c_nu[a] = c_nd[a] = c_tot[a] = c_full[a] = 0;
    int const M = s_off[kCells];
    double const hx = R.h[0], hy = R.h[1], hz = R.h[2];
    double const rl2 = A.r_list_sq;
    // FP32 pre-test on positions in the group's frame: the staged records hold, rounded
    // once to FP32, (w + shift - centre) h, with w the wrapped scaled coordinate, shift
    // the period (-1, 0, 1) that places the record's window cell next to the group and
    // centre the group's centre; every value is at most h/2 in size. Per coordinate the
    // difference of two such values is off by at most 2^-24 h / 2 twice plus 2^-24 of
    // itself; 1e-7 (h_x + h_y + h_z) and a 1e-6 relative widening of the radius cover
    // that and the FP32 products and sums. Window offsets are the minimum image for every
    // pair within the radius (6 or more half cells per edge), so no rint is needed.
    double const ox = (2 * gx + 1.) / nx - 0.5, oy = (2 * gy + 1.) / ny - 0.5,
                 oz = (2 * gz + 1.) / nz - 0.5;
    double const rpre = sqrt(rl2) * (1. + 1e-6) + 1e-7 * (hx + hy + hz);
    float const rpre2 = static_cast<float>(rpre * rpre * (1. + 1e-6));
    // the same bound from inside: below rin2 in FP32 a pair is within the radius in exact
    // arithmetic (and in the reference's FP64 test, whose rounding is far smaller), so only
    // the candidates between rin2 and rpre2 need the FP64 test
    double const rin = sqrt(rl2) * (1. - 1e-6) - 1e-7 * (hx + hy + hz);
    float const rin2 = rin > 0. ? static_cast<float>(rin * rin * (1. - 1e-6)) : 0.f;
    // half-cell widths
    float const wxf = static_cast<float>(hx / nx), wyf = static_cast<float>(hy / ny),
                wzf = static_cast<float>(hz / nz);
    int *queue = s_queue[warp];
    for (int c0 = 0; c0 < M; c0 += kStageH) {
        int const len = min(kStageH, M - c0);
        __syncthreads(); // the previous chunk is done with
        // one staged record per thread at a time: its window cell by bisection of the
        // cells' offsets (the largest q with s_off[q] <= p, a non-empty cell)
        for (int p = c0 + static_cast<int>(threadIdx.x); p < c0 + len;
             p += static_cast<int>(blockDim.x)) {
            int lo = 0, hi = kCells;
            while (hi - lo > 1) {
                int const mid = (lo + hi) >> 1;
                if (s_off[mid] <= p)
                    lo = mid;
                else
                    hi = mid;
            }
            int const q = lo;
            int const u = q % kWin, v = (q / kWin) % kWin, w = q / (kWin * kWin);
            int const ux = 2 * gx - 2 + u, uy = 2 * gy - 2 + v, uz = 2 * gz - 2 + w;
            double const sx = (ux < 0 ? -1. : (ux >= nx ? 1. : 0.)) - ox,
                         sy = (uy < 0 ? -1. : (uy >= ny ? 1. : 0.)) - oy,
                         sz = (uz < 0 ? -1. : (uz >= nz ? 1. : 0.)) - oz;
            int const j = A.cell_atoms[static_cast<size_t>(s_cell[q]) * cap + (p - s_off[q])];
            double4 const c = A.crd[j];
            s_j[p - c0] = j;
            s_w[p - c0] = make_float4(static_cast<float>((c.x - nint_ref(c.x) + sx) * hx),
                                      static_cast<float>((c.y - nint_ref(c.y) + sy) * hy),
                                      static_cast<float>((c.z - nint_ref(c.z) + sz) * hz), 0.f);
        }
        __syncthreads();
        for (int a = warp; a < n_me; a += nwarp) {
            int const i = s_me[a], qa = s_mq[a];
            int const ua = qa % kWin, va = (qa / kWin) % kWin, wa = qa / (kWin * kWin);
            double4 const ci = A.crd[i];
            double const cwx = ci.x - nint_ref(ci.x), cwy = ci.y - nint_ref(ci.y),
                         cwz = ci.z - nint_ref(ci.z);
            // the atom in the group's frame (its own cell is never shifted)
            float const wx = static_cast<float>((cwx - ox) * hx),
                        wy = static_cast<float>((cwy - oy) * hy),
                        wz = static_cast<float>((cwz - oz) * hz);
            // the atom's fraction of its half cell along each edge
            float const fx = fminf(fmaxf(static_cast<float>((cwx + 0.5) * nx - (2 * gx - 2 + ua)), 0.f), 1.f),
                        fy = fminf(fmaxf(static_cast<float>((cwy + 0.5) * ny - (2 * gy - 2 + va)), 0.f), 1.f),
                        fz = fminf(fmaxf(static_cast<float>((cwz + 0.5) * nz - (2 * gz - 2 + wa)), 0.f), 1.f);
            int nu = c_nu[a], nd = c_nd[a], total = c_tot[a];
            bool full = c_full[a] != 0;
            // exact test of the first n (<= 32) queued candidates, one per lane in order
            // (queue entries: the staged index, with kNearEdge set when the FP32 distance
            // lies between rin2 and rpre2)
            auto drain = [&](int n) {
                int const qv = static_cast<int>(lane) < n ? queue[lane] : -1;
                int const k = qv >= 0 ? (qv & ~kNearEdge) : -1;
                int const j = k >= 0 ? s_j[k] : -1;
                bool hit = k >= 0 && j != i; // the atom itself passes the pre-test
                if (hit && (qv & kNearEdge)) {
                    double px, py, pz;
                    hit = min_image_r2(ci, A.crd[j], hx, hy, hz, px, py, pz) <= rl2;
                }
                nb_batch(A, i, j, hit, lane, nu, nd, total, full);
            };
            // The atom's 25 rows of five half cells along x (fixed z, y offsets dw, dv), one
            // per lane: rows whose lower distance bound exceeds the radius are dropped, the
            // others trimmed along x to the cells within it (the bounds grow monotonically
            // away from the atom's own column); each kept row is a run [s0, s1) of staged
            // records, and the warp walks the non-empty runs in row order.
            auto sq = [](float g, float w) { return (g * w) * (g * w); };
            int rs0 = 0, rs1 = 0;
            if (lane < 25) {
                int const dw = static_cast<int>(lane) / 5 - 2, dv = static_cast<int>(lane) % 5 - 2;
                float const ryz = sq(cell_gap(dw, fz), wzf) + sq(cell_gap(dv, fy), wyf);
                if (ryz <= rpre2) {
                    float const rem = rpre2 - ryz;
                    int const ulo = -2 + (sq(cell_gap(-2, fx), wxf) > rem) +
                                    (sq(cell_gap(-1, fx), wxf) > rem);
                    int const uhi = 2 - (sq(cell_gap(2, fx), wxf) > rem) -
                                    (sq(cell_gap(1, fx), wxf) > rem);
                    int const row = ((wa + dw) * kWin + va + dv) * kWin + ua;
                    rs0 = max(s_off[row + ulo], c0) - c0;
                    rs1 = min(s_off[row + uhi + 1], c0 + len) - c0;
                }
            }
            unsigned rows = __ballot_sync(0xffffffffu, rs1 > rs0);
            int pend = 0;
            while (rows) {
                int const rr = __ffs(rows) - 1;
                rows &= rows - 1;
                int const s0 = __shfl_sync(0xffffffffu, rs0, rr),
                          s1 = __shfl_sync(0xffffffffu, rs1, rr);
                for (int base = s0; base < s1; base += 32) {
                    int const k = base + static_cast<int>(lane);
                    bool pass = false, edge = false;
                    if (k < s1) {
                        float4 const w = s_w[k];
                        float const dx = wx - w.x, dy = wy - w.y, dz = wz - w.z;
                        float const r2 = dx * dx + dy * dy + dz * dz;
                        pass = r2 <= rpre2;
                        edge = !(r2 < rin2);
                    }
                    unsigned const bal = __ballot_sync(0xffffffffu, pass);
                    if (pass)
                        queue[pend + __popc(bal & lt)] = edge ? (k | kNearEdge) : k;
                    pend += __popc(bal);
                    __syncwarp();
                    if (pend >= 32) {
                        drain(32);
                        __syncwarp();
                        if (static_cast<int>(lane) < pend - 32)
                            queue[lane] = queue[32 + lane];
                        pend -= 32;
                        __syncwarp();
                    }
                }
            }
            if (pend > 0) {
                drain(pend);
                __syncwarp();
            }
            if (lane == 0) {
                c_nu[a] = nu;
                c_nd[a] = nd;
                c_tot[a] = total;
                c_full[a] = full ? 1 : 0;
            }
        }
    }
    __syncthreads();
    int tmax = 0;
    for (int a = threadIdx.x; a < n_me; a += blockDim.x) {
        int const i = s_me[a];
        A.n_up[i] = c_nu[a];
        A.n_dn[i] = c_nd[a];
        if (c_tot[a] > A.maxn) {
            status_or(&A.rep[r], MDELAST_ERR_LIST_OVERFLOW);
            set_halt(A);
        }
        tmax = max(tmax, c_tot[a]);
    }
    // the block's largest count, then one atomic per block (one per atom on a single
    // address serialises in the L2)
    tmax = __reduce_max_sync(0xffffffffu, tmax);
    if (lane == 0)
        atomicMax(&s_tmax, tmax);
    __syncthreads();
    if (threadIdx.x == 0)
        atomicMax(&A.max_count[0], s_tmax);
}

size_t nbr_cells_smem(int cell_cap) {
    return (sizeof(float4) + sizeof(int)) * kStageH + 8 * 6 * sizeof(int) * cell_cap;
}

// One atom's list by one warp (all pairs, or the cells within the widened reach); the
// lanes test 32 candidates at a time. Atoms of cell-list replicas are left to k_nbr_cells
// when cells_done, unless their cells are narrow.
__device__ __forceinline__ void nbr_build_atom(AtomsView const &A, int i, unsigned lane,
                                               int cells_done) {
    int const r = A.rep_of[i];
    if (r < 0) {
        if (lane == 0) {
            A.n_up[i] = 0;
            A.n_dn[i] = 0;
        }
        return;
    }
    Replica const &R = A.rep[r];
    double const rl2 = A.r_list_sq;
    if (cells_done && R.nc[0] != 0 && !narrow_cells(R, rl2))
        return;
    double4 const ci = A.crd[i];
    double const hx = R.h[0], hy = R.h[1], hz = R.h[2];
    int nu = 0, nd = 0, total = 0;
    bool full = false;
    double px, py, pz;
    if (R.nc[0] == 0) {
        int const b = R.atom_begin, e = R.atom_begin + R.n_atoms;
        for (int base = b; base < e; base += 32) {
            int const j = base + static_cast<int>(lane);
            bool hit = false;
            if (j < e && j != i)
                hit = min_image_r2(ci, A.crd[j], hx, hy, hz, px, py, pz) <= rl2;
            nb_batch(A, i, j, hit, lane, nu, nd, total, full);
        }
    } else {
        double const w[3] = {ci.x - nint_ref(ci.x), ci.y - nint_ref(ci.y), ci.z - nint_ref(ci.z)};
        int idx[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int k = static_cast<int>(floor((w[a] + 0.5) * R.nc[a]));
            idx[a] = k < 0 ? 0 : (k >= R.nc[a] ? R.nc[a] - 1 : k);
        }
        int first[3], count[3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
            cell_span(idx[a], R.nc[a], cell_reach(R.h[a], R.nc[a], rl2), first[a], count[a]);
        for (int dz = 0; dz < count[2]; ++dz) {
            int const cz = (first[2] + dz + R.nc[2]) % R.nc[2];
            for (int dy = 0; dy < count[1]; ++dy) {
                int const cy = (first[1] + dy + R.nc[1]) % R.nc[1];
                for (int dx = 0; dx < count[0]; ++dx) {
                    int const cx = (first[0] + dx + R.nc[0]) % R.nc[0];
                    int const cell = R.cell_begin + (cz * R.nc[1] + cy) * R.nc[0] + cx;
                    int n = A.cell_count[cell];
                    if (n > A.cell_cap)
                        n = A.cell_cap;
                    int const *m = A.cell_atoms + static_cast<size_t>(cell) * A.cell_cap;
                    for (int base = 0; base < n; base += 32) {
                        int const k = base + static_cast<int>(lane);
                        int const j = k < n ? m[k] : -1;
                        bool hit = false;
                        if (k < n && j != i)
                            hit = min_image_r2(ci, A.crd[j], hx, hy, hz, px, py, pz) <= rl2;
                        nb_batch(A, i, j, hit, lane, nu, nd, total, full);
                    }
                }
            }
        }
    }
    if (lane == 0) {
        A.n_up[i] = nu;
        A.n_dn[i] = nd;
        if (total > A.maxn) {
            status_or(&A.rep[r], MDELAST_ERR_LIST_OVERFLOW);
            set_halt(A);
        }
        atomicMax(&A.max_count[0], total);
    }
}

// Grid-striding warps over the atoms of the replicas k_nbr_cells left (all when
// !cells_done); the padding slots keep the zero counts of their allocation.
__global__ void k_nbr_build(AtomsView A, int cells_done) {
    unsigned const lane = threadIdx.x & 31u;
    int const w0 = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    int const n_warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
    for (int r = 0; r < A.n_rep; ++r) {
        Replica const &R = A.rep[r];
        if (cells_done && R.nc[0] != 0 && !narrow_cells(R, A.r_list_sq))
            continue;
        for (int a = w0; a < R.n_atoms; a += n_warps)
            nbr_build_atom(A, R.atom_begin + a, lane, cells_done);
    }
}

// ------------------------------------------------------------------------------------
// Density pass (md_driver.cpp:195-277): rho_i = sum_j rho_{type j}(r_ij); on sampled
// steps g_i = sum_j rho'_{type j}(r)/r p p^T (Voigt) and h_i = sum_j rho'_{type j}(r)/r p,
// then F, F', F'' of rho_i. g and h are only needed in F''_i g_i g_i^T and F''_i |h_i|^2,
// so those per-atom Born and Laplacian terms (md_driver.cpp:410-419) are formed here and
// g, h are never stored.

// The block's FP64 sums (embedding energy, the per-atom Born term F''_i g_i g_i^T and
// Laplacian term) are folded warp by warp after each atom group into per-warp shared
// accumulators, not carried in registers through the pair loop.
template <bool OBS, int TPA, int IP, typename IX>
__global__ void __launch_bounds__(kBlock) k_density(AtomsView A, TablesView T) {
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
    double const hx = R->h[0], hy = R->h[1], hz = R->h[2];
    bool const uc = T.uc64 != 0; // one cutoff for every function: no per-type test
    for (int a0 = lb * apb; a0 < n_slots; a0 += nb * apb) {
        int const a = a0 + static_cast<int>(threadIdx.x) / TPA;
        int const i = R->atom_begin + a;
        bool const valid = a < R->n_atoms && T.has_eam;
        double rho = 0.;
        double g[6] = {0, 0, 0, 0, 0, 0}, hv[3] = {0, 0, 0};
        double4 ci = make_double4(0., 0., 0., 0.);
        if (valid) {
            ci = A.crd[i];
            int const ti = static_cast<int>(ci.w);
            int const nu = A.pn_up[i], ntot = nu + A.pn_dn[i];
            PairRow<IX> const row = pair_row<IX>(A, i, R->atom_begin);
            // the next partner's record is loaded one iteration ahead, its list entry two
            double4 cn = A.crd[sub < ntot ? row.at(list_slot(sub, nu, A.pmaxn)) : i];
            int jn = sub < ntot ? row.at(list_slot(min(sub + TPA, ntot - 1), nu, A.pmaxn)) : i;
            for (int kk = sub; kk < ntot; kk += TPA) {
                double4 const cj = cn;
                if (kk + TPA < ntot) {
                    cn = A.crd[jn];
                    jn = row.at(list_slot(min(kk + 2 * TPA, ntot - 1), nu, A.pmaxn));
                }
                double px, py, pz;
                double const r2 = min_image_r2(ci, cj, hx, hy, hz, px, py, pz);
                if (r2 > T.r_cut_sq)
                    continue;
                double const dr = sqrt(r2);
                int const tj = static_cast<int>(cj.w);
                if (!uc && dr > T.eam_rcut[tj])
                    continue;
                double t;
                int const k = tab_locate(dr, T.inv_hr, T.nri, t);
                int const s = pair_slot(ti, tj);
                int const off = (tj == (ti < tj ? ti : tj)) ? kF : 2 * kF;
                double v = 0., d1 = 0., d2 = 0.;
                tab_eval<IP, true, OBS, false>(
                    T.rb + (static_cast<size_t>(s) * T.nri + k) * 3 * kF + off, t, T.inv_hr,
                    T.inv_hr2, v, d1, d2);
                rho += v;
                if (OBS) {
                    double const ar = d1 / dr;
                    double const ap[3] = {ar * px, ar * py, ar * pz};
                    g[0] += ap[0] * px;
                    g[1] += ap[1] * py;
                    g[2] += ap[2] * pz;
                    g[3] += ap[1] * pz;
                    g[4] += ap[0] * pz;
                    g[5] += ap[0] * py;
                    hv[0] += ap[0];
                    hv[1] += ap[1];
                    hv[2] += ap[2];
                }
            }
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
            int const ti = static_cast<int>(ci.w);
            // embedding function (eam.hpp:48-70); rho beyond rhomax_fatal ends the reference run
            if (rho > T.rhomax[ti])
                status_or(A.rep + r, MDELAST_FATAL_RHO_MAX);
            double t;
            int const k = tab_locate(rho, T.inv_hf, T.nfi, t);
            double dF = 0.;
            tab_eval<IP, true, true, OBS>(T.Ft + (static_cast<size_t>(ti) * T.nfi + k) * kF, t,
                                          T.inv_hf, T.inv_hf2, F, dF, d2F);
            A.rho[i] = rho;
            A.Fe[i] = F;
            if (OBS)
                A.dF2[i] = make_double2(dF, d2F);
            else
                A.dF2[i].x = dF;
        }
        warp_accumulate(F, &sacc[warp][D_FSUM]);
        if (OBS) {
            // zero for lanes without an atom
            if (!own)
                d2F = 0.;
            int q = D_CB;
#pragma unroll
            for (int u = 0; u < 6; ++u)
#pragma unroll
                for (int v = u; v < 6; ++v)
                    warp_accumulate(d2F * g[u] * g[v], &sacc[warp][q++]);
            warp_accumulate(d2F * (hv[0] * hv[0] + hv[1] * hv[1] + hv[2] * hv[2]),
                            &sacc[warp][D_LAP]);
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

// ------------------------------------------------------------------------------------
// Force pass (md_driver.cpp:300-430) with the closing half kick of velocity Verlet fused
// in (md_driver.cpp:433-452; KICK). Per pair, with X = (phi'' - phi'/r + EAM terms)/r^2:
//   dE/dr = phi' + F'_i rho'_j + F'_j rho'_i,  F_i += -(dE/dr)/r p
// Global sums (virial, Born stress, Born tensor, pair Laplacian) take each pair once, on
// its j > i visit; the Born tensor is accumulated as the 15 distinct degree-4 monomials
// X p_a p_b p_c p_d of which its 21 upper-triangle entries are made.
//
// Each atom row is walked in two loops, partners j > i (which also feed the global sums)
// and partners j < i, so the lanes of a warp do not diverge on the global-sum work. A
// row's global sums are summed in FP64 registers along the row and added, once per atom
// and combined across its TPA lanes, into FP64 block accumulators in shared memory, one
// set per lane group: the loops then keep 23 FP64 sums live instead of all 35 of the block,
// and three 128-thread blocks of the observable-step variant fit an SM instead of two.

template <bool OBS> struct RowSums64 {
    double virial = 0.;
    double sig[6] = {0., 0., 0., 0., 0., 0.};
    double cb[OBS ? 15 : 1] = {};
    double lap = 0.;
};

struct RowIn64 {
    double4 ci;
    double dFi, d2Fi;
    int ti;
    double hx, hy, hz;
};

template <bool OBS, bool UPPER, int TPA, int IP, typename IX, bool UC>
__device__ __forceinline__ void force_row(AtomsView const &A, TablesView const &T,
                                          RowIn64 const &in, PairRow<IX> const &row, int n,
                                          int sub, double &fx, double &fy, double &fz,
                                          double &epot, RowSums64<OBS> &ps, bool &warn_rmin) {
    constexpr int kF = TabFmt<IP>::kF;
    if (sub >= n)
        return;
    auto slot = [&](int k) { return UPPER ? k : A.pmaxn - 1 - k; };
    int const ti = in.ti;
    double const dFi = in.dFi, d2Fi = in.d2Fi;
    // the next partner's record and F' are loaded one iteration ahead, its list entry two
    int jn = row.at(slot(sub));
    double4 cn = A.crd[jn];
    double2 fn = A.dF2[jn];
    jn = row.at(slot(min(sub + TPA, n - 1)));
    for (int kk = sub; kk < n; kk += TPA) {
        double4 const cj = cn;
        double2 const dFj2 = fn;
        if (kk + TPA < n) {
            cn = A.crd[jn];
            fn = A.dF2[jn];
            jn = row.at(slot(min(kk + 2 * TPA, n - 1)));
        }
        double px, py, pz;
        double const r2 = min_image_r2(in.ci, cj, in.hx, in.hy, in.hz, px, py, pz);
        if (r2 > T.r_cut_sq)
            continue;
        double const dr = sqrt(r2);
        double const idr = 1. / dr;
        int const tj = static_cast<int>(cj.w);
        int const s = pair_slot(ti, tj);
        double t;
        int const k = tab_locate(dr, T.inv_hr, T.nri, t);
        const double *bundle = T.rb + (static_cast<size_t>(s) * T.nri + k) * 3 * kF;
        // TablePotential::calculate (potential.hpp:92-104)
        double V = 0., dV = 0., d2V = 0.;
        if (dr < T.pot_rmin[s])
            warn_rmin = true;
        if (UC || !(dr > T.pot_rcut[s]))
            tab_eval<IP, true, true, OBS && UPPER>(bundle, t, T.inv_hr, T.inv_hr2, V, dV, d2V);
        double dedr = dV;
        double X = 0., lap = 0.;
        if (OBS && UPPER) {
            X = d2V - dV * idr;
            lap = 2. * (d2V + 2. * dV * idr);
        }
        if (T.has_eam) {
            // rho of the lower type at bundle offset kF, of the higher type at 2 kF
            int const oi = (ti <= tj) ? kF : 2 * kF, oj = (ti < tj) ? 2 * kF : kF;
            double drho_i = 0., drho_j = 0., d2rho_i = 0., d2rho_j = 0., unused = 0.;
            if (UC || !(dr > T.eam_rcut[ti]))
                tab_eval<IP, false, true, OBS && UPPER>(bundle + oi, t, T.inv_hr, T.inv_hr2,
                                                        unused, drho_i, d2rho_i);
            if (UC || !(dr > T.eam_rcut[tj]))
                tab_eval<IP, false, true, OBS && UPPER>(bundle + oj, t, T.inv_hr, T.inv_hr2,
                                                        unused, drho_j, d2rho_j);
            double const dFj = dFj2.x;
            // the two cross terms are rounded separately and added (commutative), so
            // the i- and j-side evaluations of dE/dr are bitwise equal
            dedr = __dadd_rn(dedr, __dadd_rn(__dmul_rn(dFi, drho_j), __dmul_rn(dFj, drho_i)));
            if (OBS && UPPER) {
                double const d2Fj = dFj2.y;
                lap += 2. * (dFj * (d2rho_i + 2. * drho_i * idr) +
                             dFi * (d2rho_j + 2. * drho_j * idr));
                lap += d2Fi * (drho_j * drho_j) + d2Fj * (drho_i * drho_i);
                X += dFi * (d2rho_j - drho_j * idr) + dFj * (d2rho_i - drho_i * idr);
            }
        }
        double const sc = __dmul_rn(-dedr, idr);
        fx += __dmul_rn(sc, px);
        fy += __dmul_rn(sc, py);
        fz += __dmul_rn(sc, pz);
        epot += 0.5 * V;
        if (UPPER) {
            ps.virial += dr * dedr;
            double const xx = px * px, yy = py * py, zz = pz * pz;
            double const yz = py * pz, xz = px * pz, xy = px * py;
            double const w = dedr * idr;
            ps.sig[0] += w * xx;
            ps.sig[1] += w * yy;
            ps.sig[2] += w * zz;
            ps.sig[3] += w * yz;
            ps.sig[4] += w * xz;
            ps.sig[5] += w * xy;
            if (OBS) {
                X *= idr * idr;
                double const Xxx = X * xx, Xyy = X * yy, Xzz = X * zz;
                ps.cb[0] += Xxx * xx;  // x4
                ps.cb[1] += Xyy * yy;  // y4
                ps.cb[2] += Xzz * zz;  // z4
                ps.cb[3] += Xxx * xy;  // x3y
                ps.cb[4] += Xxx * xz;  // x3z
                ps.cb[5] += Xyy * xy;  // xy3
                ps.cb[6] += Xyy * yz;  // y3z
                ps.cb[7] += Xzz * xz;  // xz3
                ps.cb[8] += Xzz * yz;  // yz3
                ps.cb[9] += Xxx * yy;  // x2y2
                ps.cb[10] += Xxx * zz; // x2z2
                ps.cb[11] += Xyy * zz; // y2z2
                ps.cb[12] += Xxx * yz; // x2yz
                ps.cb[13] += Xyy * xz; // xy2z
                ps.cb[14] += Xzz * xy; // xyz2
                ps.lap += lap;
            }
        }
    }
}

template <bool OBS, bool KICK, int TPA, int IP, typename IX>
__global__ void __launch_bounds__(kBlock) k_force(AtomsView A, TablesView T) {
    if (halted(A)) // a list build ran out of capacity: nothing until the host regrows
        return;
    constexpr int kG = kBlock / TPA;
    __shared__ double s_acc[F_NSUM * kG];
    int const tid = threadIdx.x, grp = tid / TPA;
    for (int k = tid; k < F_NSUM * kG; k += kBlock)
        s_acc[k] = 0.;
    __syncthreads();
    int const r = A.fblk_rep[blockIdx.x];
    Replica const *R = A.rep + r;
    int const lb = blockIdx.x - R->fblk_begin, nb = R->fblk_n;
    int const apb = kBlock / TPA, sub = tid % TPA;
    int const n_slots = R->n_blocks * kBlock;
    RowIn64 in;
    in.hx = R->h[0];
    in.hy = R->h[1];
    in.hz = R->h[2];
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
            in.ci = A.crd[i];
            in.ti = static_cast<int>(in.ci.w);
            double2 const dFi2 = T.has_eam ? A.dF2[i] : make_double2(0., 0.);
            in.dFi = dFi2.x;
            in.d2Fi = OBS ? dFi2.y : 0.;
            int const nu = A.pn_up[i], nd = A.pn_dn[i];
            PairRow<IX> const row = pair_row<IX>(A, i, R->atom_begin);
            bool warn_rmin = false;
            RowSums64<OBS> ps;
            // one cutoff for every function (every setfl potential): no per-function tests
            if (T.uc64) {
                force_row<OBS, true, TPA, IP, IX, true>(A, T, in, row, nu, sub, fx, fy, fz,
                                                        epot, ps, warn_rmin);
                force_row<OBS, false, TPA, IP, IX, true>(A, T, in, row, nd, sub, fx, fy, fz,
                                                         epot, ps, warn_rmin);
            } else {
                force_row<OBS, true, TPA, IP, IX, false>(A, T, in, row, nu, sub, fx, fy, fz,
                                                         epot, ps, warn_rmin);
                force_row<OBS, false, TPA, IP, IX, false>(A, T, in, row, nd, sub, fx, fy, fz,
                                                          epot, ps, warn_rmin);
            }
            if (warn_rmin)
                status_or(A.rep + r, MDELAST_WARN_RMIN);
            sums[F_VIRIAL] = ps.virial;
#pragma unroll
            for (int k = 0; k < 6; ++k)
                sums[F_SIGMA + k] = ps.sig[k];
            if (OBS) {
#pragma unroll
                for (int k = 0; k < 15; ++k)
                    sums[F_CB + k] = ps.cb[k];
                sums[F_LAP] = ps.lap;
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
                // U2 (md_driver.cpp:446-449): v = v e + (c dt) F / m
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
    // the groups' slots into the block sums
    __syncthreads();
    double acc[F_NSUM];
#pragma unroll
    for (int k = 0; k < F_NSUM; ++k)
        acc[k] = tid < kG ? s_acc[k * kG + tid] : 0.;
    block_sum_store<F_NSUM>(acc, A.pf + static_cast<size_t>(blockIdx.x) * F_NSUM);
}

// ------------------------------------------------------------------------------------
// Opening half kick and drift (md_driver.cpp:433-499): the velocities first take the
// thermostat factor of the preceding NHC half step (Replica::s_kick, which includes the
// factor deferred from the previous step), then v = v e + (c dt) F / m, then
// c += (cf dt) v / h with the box before this step's barostat update.

__global__ void __launch_bounds__(kBlock) k_kick_drift(AtomsView A, TablesView T) {
    if (halted(A)) // a list build ran out of capacity: nothing until the host regrows
        return;
    // the grid covers the n_pad slots exactly; a warp never spans two replicas (their
    // ranges start on multiples of kTile) and its padding slots, if any, come last
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    int const r = A.rep_of[i];
    double d2 = 0.;
    if (r >= 0) {
    Replica const *R = A.rep + r;
    size_t const np = A.n_pad;
    double4 c = A.crd[i];
    double const m = T.mass[static_cast<int>(c.w)];
    double const s = R->s_kick, e = R->e_kick, cdt = R->cdt_kick, a = R->cfdt;
    double v[3] = {A.vel[i] * s, A.vel[np + i] * s, A.vel[2 * np + i] * s};
    double const f[3] = {A.frc[i], A.frc[np + i], A.frc[2 * np + i]};
#pragma unroll
    for (int k = 0; k < 3; ++k)
        v[k] = v[k] * e + cdt * f[k] / m;
    A.vel[i] = v[0];
    A.vel[np + i] = v[1];
    A.vel[2 * np + i] = v[2];
    c.x = __dadd_rn(c.x, __ddiv_rn(__dmul_rn(a, v[0]), R->h_pos[0]));
    c.y = __dadd_rn(c.y, __ddiv_rn(__dmul_rn(a, v[1]), R->h_pos[1]));
    c.z = __dadd_rn(c.z, __ddiv_rn(__dmul_rn(a, v[2]), R->h_pos[2]));
    A.crd[i] = c;
    if (A.crd_ref) {
        // squared displacement since the pair list was refreshed (position in this step's
        // box against the position in the refresh's box)
        double4 const c0 = A.crd_ref[i];
        double const dx = c.x * R->h[0] - c0.x, dy = c.y * R->h[1] - c0.y,
                     dz = c.z * R->h[2] - c0.z;
        d2 = dx * dx + dy * dy + dz * dz;
    }
    if (A.posf) // mixed precision: wrapped FP32 positions in the box after this drift
        A.posf[i] = make_float4(static_cast<float>((c.x - nint_ref(c.x)) * R->h[0] / kAng),
                                static_cast<float>((c.y - nint_ref(c.y)) * R->h[1] / kAng),
                                static_cast<float>((c.z - nint_ref(c.z)) * R->h[2] / kAng),
                                static_cast<float>(c.w));
    }
    if (A.crd_ref) {
        // the replica's largest displacement: warp maximum, then one atomic per warp
        // (non-negative doubles order like their bit patterns)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            d2 = fmax(d2, __shfl_xor_sync(0xffffffffu, d2, o));
        int const r0 = __shfl_sync(0xffffffffu, r, 0);
        if ((threadIdx.x & 31) == 0 && r0 >= 0 && d2 > 0.)
            atomicMax(reinterpret_cast<unsigned long long *>(&A.rep[r0].sub_d2),
                      static_cast<unsigned long long>(__double_as_longlong(d2)));
    }
}

// ------------------------------------------------------------------------------------
// Pair list of the pair passes: the pairs of the neighbour list within sub_r2, the same
// FP64 min-image test on both atoms of a pair (so the list is symmetric). A replica's rows
// are rebuilt when its list was rebuilt or when some atom has moved by more than half the
// radius margin since the last refresh: then every pair now within r_cut is still in the
// list. One warp per atom slot at a time, grid-striding over the slots; the warp tests 32
// entries at a time and compacts the kept ones with a ballot. The kernel runs every step
// and most steps refresh nothing: each block first asks whether any replica is due (one
// flag per thread) and returns at once if none is, so a step without a refresh costs one
// short wave instead of a warp per atom slot.
//
// Row order (`sorted`, when the row fits the warp's shared-memory scratch): each half of a
// row (partners j > i, partners j < i) is ordered by distance shell, shells kSubShell wide
// in r/r_cut, in list order within a shell (a stable counting sort: the warp counts the
// shells with shared-memory atomics, scans the counts, and places each chunk of 32 entries
// with match_any). The lanes of a warp walk their rows in step, so at every iteration they
// look up the tables at about the same r (the same neighbour shell of the lattice) and
// read a few nearby intervals instead of scattered ones. Only the order in which an atom's
// pair terms are summed changes; which pairs are kept does not.
constexpr int kSubShells = 32;
constexpr float kSubShell = 0.035f; // shell width / r_list; 32 shells reach 1.12 r_list

// Radius and shell constants of the refresh, formed once per thread: the FP32 keep radius
// (A^2, widened by 1e-5) and the inverse shell widths for r in cm and in A.
struct SubConst {
    float r2f, inv_shell, inv_shell_a;
};

__device__ __forceinline__ SubConst sub_const(AtomsView const &A) {
    double const rs = sqrt(A.sub_r2);
    return SubConst{static_cast<float>(A.sub_r2 / (kAng * kAng) * (1. + 1e-5)),
                    static_cast<float>(1. / (kSubShell * rs)),
                    static_cast<float>(kAng / (kSubShell * rs))};
}

__device__ __forceinline__ void sublist_row(AtomsView const &A, int i, int lane, bool sorted,
                                            int *s_j, int *s_cnt, SubConst const &sc) {
    int const r = A.rep_of[i];
    if (r < 0)
        return;
    Replica const *R = A.rep + r;
    if (!(R->sub_force || R->sub_d2 > A.sub_half2))
        return;
    sorted = sorted && R->n_atoms <= (1 << 26); // the packing holds 26-bit offsets
    double4 const ci = A.crd[i];
    double const hx = R->h[0], hy = R->h[1], hz = R->h[2];
    int const nu = A.n_up[i], nd = A.n_dn[i];
    int const *row = A.nbr + static_cast<size_t>(i) * A.maxn;
    int *out = A.pnbr + static_cast<size_t>(i) * A.pmaxn;
    uint16_t *out16 = A.pnbr16 ? A.pnbr16 + static_cast<size_t>(i) * A.pmaxn : nullptr;
    int const base = R->atom_begin;
    auto put = [&](int slot, int j) {
        if (out16)
            out16[slot] = static_cast<uint16_t>(j - base);
        else
            out[slot] = j;
    };
    unsigned const lt = (1u << lane) - 1u;
    // Mixed precision: the keep test runs in FP32 on the wrapped positions the pair passes
    // read, with the minimum image they use (the same on both atoms of a pair, so the list
    // stays symmetric), against the radius widened by 1e-5: every pair within it in exact
    // arithmetic is kept, a few just beyond it too, which add zeros. FP64: the reference's
    // min image and the exact radius.
    // (the box edges in A by a product, not the pair passes' quotient: the list needs the
    // same image on both atoms of a pair, not the pair passes' last bit)
    bool const f32 = A.posf != nullptr;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    float3 L = make_float3(0.f, 0.f, 0.f), iL = L;
    if (f32) {
        pi = A.posf[i];
        L = make_float3(static_cast<float>(hx * 1e8), static_cast<float>(hy * 1e8),
                        static_cast<float>(hz * 1e8));
        iL = make_float3(__frcp_rn(L.x), __frcp_rn(L.y), __frcp_rn(L.z));
    }
    float const sub_r2f = sc.r2f, ish = f32 ? sc.inv_shell_a : sc.inv_shell;
    if (sorted) {
        s_cnt[lane] = 0;
        s_cnt[kSubShells + lane] = 0;
        __syncwarp();
    }
    int ku = 0, kd = 0;
    for (int k0 = 0; k0 < nu + nd; k0 += 32) {
        int const k = k0 + lane;
        bool keep = false, upper = k < nu;
        int j = -1;
        float r2s = 0.f; // r^2 in the units of ish (A^2 or cm^2)
        if (k < nu + nd) {
            j = row[upper ? k : A.maxn - 1 - (k - nu)];
            if (f32) {
                float dx, dy, dz;
                r2s = min_image_f(pi, A.posf[j], L, iL, dx, dy, dz);
                keep = r2s <= sub_r2f;
            } else {
                double px, py, pz;
                double const r2 = min_image_r2(ci, A.crd[j], hx, hy, hz, px, py, pz);
                keep = r2 <= A.sub_r2;
                r2s = static_cast<float>(r2);
            }
        }
        unsigned const bu = __ballot_sync(0xffffffffu, keep && upper);
        unsigned const bd = __ballot_sync(0xffffffffu, keep && !upper);
        if (sorted) {
            // kept entries to the scratch in list order (upper from the front, lower from
            // the back) with their shell in the top bits; shells counted per half
            if (keep) {
                int const q = upper ? ku + __popc(bu & lt) : A.maxn - 1 - (kd + __popc(bd & lt));
                int const sh = min(kSubShells - 1, static_cast<int>(sqrtf(r2s) * ish));
                s_j[q] = (sh << 26) | (j - base);
                atomicAdd(&s_cnt[(upper ? 0 : kSubShells) + sh], 1);
            }
        } else {
            if (keep && upper)
                put(ku + __popc(bu & lt), j);
            if (keep && !upper)
                put(A.pmaxn - 1 - (kd + __popc(bd & lt)), j);
        }
        ku += __popc(bu);
        kd += __popc(bd);
    }
    if (sorted) {
        __syncwarp();
        for (int half = 0; half < 2; ++half) {
            // exclusive scan of this half's shell counts: the shells' first output slots
            int const c = s_cnt[half * kSubShells + lane];
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int const v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o)
                    incl += v;
            }
            __syncwarp();
            s_cnt[half * kSubShells + lane] = incl - c;
            __syncwarp();
            int const n_half = half ? kd : ku;
            for (int e0 = 0; e0 < n_half; e0 += 32) {
                int const e = e0 + lane;
                bool const act = e < n_half;
                int packed = 0, sh = kSubShells; // inactive lanes: a shell no entry has
                if (act) {
                    packed = s_j[half ? A.maxn - 1 - e : e];
                    sh = packed >> 26;
                }
                unsigned const peers = __match_any_sync(0xffffffffu, sh);
                if (act) {
                    int const slot = s_cnt[half * kSubShells + sh] + __popc(peers & lt);
                    put(half ? A.pmaxn - 1 - slot : slot, base + (packed & 0x3ffffff));
                }
                __syncwarp();
                // the lowest lane of each shell's group advances that shell's next slot
                if (act && (peers & lt) == 0)
                    s_cnt[half * kSubShells + sh] += __popc(peers);
                __syncwarp();
            }
        }
    }
    if (lane == 0) {
        A.pn_up[i] = ku;
        A.pn_dn[i] = kd;
        A.crd_ref[i] = make_double4(ci.x * hx, ci.y * hy, ci.z * hz, ci.w);
    }
}

// dynamic shared memory of k_sublist: per warp of its 256-thread blocks, one row of packed
// entries (maxn) and two halves' shell counters; 0 when that exceeds kSublistSortMax or a
// replica offset does not fit the packing (the rows then keep list order)
__host__ __device__ size_t sublist_smem(int maxn) {
    size_t const b = static_cast<size_t>(256 / 32) * (maxn + 2 * kSubShells) * sizeof(int);
    return b <= kSublistSortMax ? b : 0;
}

// 5 blocks of 256 threads per SM (the launch is 5 blocks per SM): at most 48 registers
__global__ void __launch_bounds__(256, 5) k_sublist(AtomsView A) {
    if (halted(A)) // a list build ran out of capacity: nothing until the host regrows
        return;
    extern __shared__ int s_sub[];
    int due = 0;
    for (int r = threadIdx.x; r < A.n_rep; r += blockDim.x) {
        Replica const *R = A.rep + r;
        due |= R->sub_force || R->sub_d2 > A.sub_half2;
    }
    if (!__syncthreads_or(due))
        return;
    int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool const sorted = sublist_smem(A.maxn) > 0;
    int *s_j = s_sub + static_cast<size_t>(warp) * (A.maxn + 2 * kSubShells);
    int *s_cnt = s_j + A.maxn;
    int const n_warps = gridDim.x * (blockDim.x >> 5);
    SubConst const sc = sub_const(A);
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < A.n_pad; i += n_warps)
        sublist_row(A, i, lane, sorted, s_j, s_cnt, sc);
}

__global__ void k_sub_invalidate(AtomsView A) {
    for (int r = threadIdx.x; r < A.n_rep; r += blockDim.x)
        A.rep[r].sub_force = 1;
}

// ------------------------------------------------------------------------------------
// Readout of one per-atom field in the C-ABI layout (x, y, z interleaved per atom) for
// replica r, applying the deferred velocity factor.

__global__ void k_readout(AtomsView A, TablesView T, int r, int field, double *out,
                          const double *pos0, int stepped) {
    Replica const *R = A.rep + r;
    int const n = R->n_atoms;
    int const a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n)
        return;
    int const i = R->atom_begin + a;
    size_t const np = A.n_pad;
    switch (field) {
    case MDELAST_ATOM_POSITIONS: {
        if (!stepped) {
            out[3 * a] = pos0[3 * a];
            out[3 * a + 1] = pos0[3 * a + 1];
            out[3 * a + 2] = pos0[3 * a + 2];
        } else {
            double4 const c = A.crd[i];
            out[3 * a] = __dmul_rn(__dadd_rn(c.x, -nint_ref(c.x)), R->h_pos[0]);
            out[3 * a + 1] = __dmul_rn(__dadd_rn(c.y, -nint_ref(c.y)), R->h_pos[1]);
            out[3 * a + 2] = __dmul_rn(__dadd_rn(c.z, -nint_ref(c.z)), R->h_pos[2]);
        }
        break;
    }
    case MDELAST_ATOM_COORDINATES: {
        double4 const c = A.crd[i];
        out[3 * a] = c.x;
        out[3 * a + 1] = c.y;
        out[3 * a + 2] = c.z;
        break;
    }
    case MDELAST_ATOM_VELOCITIES:
        out[3 * a] = A.vel[i] * R->vscale;
        out[3 * a + 1] = A.vel[np + i] * R->vscale;
        out[3 * a + 2] = A.vel[2 * np + i] * R->vscale;
        break;
    case MDELAST_ATOM_FORCES:
        out[3 * a] = A.frc[i];
        out[3 * a + 1] = A.frc[np + i];
        out[3 * a + 2] = A.frc[2 * np + i];
        break;
    case MDELAST_ATOM_RHO:
        out[a] = A.rho[i];
        break;
    case MDELAST_ATOM_EPOT:
        out[a] = A.epot[i];
        break;
    case MDELAST_ATOM_EKIN: {
        double const m = T.mass[static_cast<int>(A.crd[i].w)];
        double const vx = A.vel[i] * R->vscale, vy = A.vel[np + i] * R->vscale,
                     vz = A.vel[2 * np + i] * R->vscale;
        out[a] = 0.5 * m * (vx * vx + vy * vy + vz * vz);
        break;
    }
    default:
        break;
    }
}

// The reference-format half list of replica r: for each atom its partners j > i, in
// ascending order (md_driver.cpp:283-294). counts[a] = n_up of atom a (pass 1) and the
// sorted entries written at point[a] (pass 2).
__global__ void k_half_list_counts(AtomsView A, int r, int *counts) {
    Replica const *R = A.rep + r;
    int const a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= R->n_atoms)
        return;
    counts[a] = A.n_up[R->atom_begin + a];
}

__global__ void k_half_list_fill(AtomsView A, int r, const int *point, int *out) {
    Replica const *R = A.rep + r;
    int const a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= R->n_atoms)
        return;
    int const i = R->atom_begin + a;
    int const n = A.n_up[i];
    int *o = out + point[a];
    for (int k = 0; k < n; ++k)
        o[k] = A.nbr[static_cast<size_t>(i) * A.maxn + k] - R->atom_begin;
    for (int k = 1; k < n; ++k) { // insertion sort of a short run
        int const v = o[k];
        int m = k - 1;
        while (m >= 0 && o[m] > v) {
            o[m + 1] = o[m];
            --m;
        }
        o[m + 1] = v;
    }
}

__global__ void k_status_and(AtomsView A, unsigned mask) {
    for (int r = threadIdx.x; r < A.n_rep; r += blockDim.x)
        atomicAnd(&A.rep[r].obs.status, mask);
}

// Table values on the device for the table checks: which 0 pair slot s, 1 rho of type s,
// 2 F of type s. Same code paths as the pair kernels.
__global__ void k_table_eval(TablesView T, int which, int s, const double *x, int n,
                             double *out) {
    int const q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n)
        return;
    double const xv = x[q];
    double t;
    double v[3] = {0., 0., 0.};
    bool const bs = T.interp == MDELAST_BSPLINE;
    int const kF = bs ? TabFmt<MDELAST_BSPLINE>::kF : TabFmt<MDELAST_QUINTIC>::kF;
    if (which == 2) {
        int const k = tab_locate(xv, T.inv_hf, T.nfi, t);
        const double *p = T.Ft + (static_cast<size_t>(s) * T.nfi + k) * kF;
        if (bs)
            tab_eval<MDELAST_BSPLINE, true, true, true>(p, t, T.inv_hf, T.inv_hf2, v[0], v[1],
                                                        v[2]);
        else
            tab_eval<MDELAST_QUINTIC, true, true, true>(p, t, T.inv_hf, T.inv_hf2, v[0], v[1],
                                                        v[2]);
    } else {
        int const k = tab_locate(xv, T.inv_hr, T.nri, t);
        int slot, off;
        double rc;
        if (which == 0) {
            slot = s;
            off = 0;
            rc = T.pot_rcut[s];
        } else {
            slot = pair_slot(s, s);
            off = kF;
            rc = T.eam_rcut[s];
        }
        if (!(xv > rc)) {
            const double *p = T.rb + (static_cast<size_t>(slot) * T.nri + k) * 3 * kF + off;
            if (bs)
                tab_eval<MDELAST_BSPLINE, true, true, true>(p, t, T.inv_hr, T.inv_hr2, v[0],
                                                            v[1], v[2]);
            else
                tab_eval<MDELAST_QUINTIC, true, true, true>(p, t, T.inv_hr, T.inv_hr2, v[0],
                                                            v[1], v[2]);
        }
    }
    out[3 * q] = v[0];
    out[3 * q + 1] = v[1];
    out[3 * q + 2] = v[2];
}

namespace {
template <bool OBS, int IP, typename IX>
void density_tpa_ix(int tpa, int grid, cudaStream_t s, AtomsView const &A, TablesView const &T) {
    switch (tpa) {
    case 1: k_density<OBS, 1, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    case 4: k_density<OBS, 4, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    case 8: k_density<OBS, 8, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    default: k_density<OBS, 16, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    }
}
template <bool OBS, int IP>
void density_tpa(int tpa, int grid, cudaStream_t s, AtomsView const &A, TablesView const &T) {
    if (A.pnbr16)
        density_tpa_ix<OBS, IP, uint16_t>(tpa, grid, s, A, T);
    else
        density_tpa_ix<OBS, IP, int>(tpa, grid, s, A, T);
}
template <bool OBS, bool KICK, int IP, typename IX>
void force_tpa_ix(int tpa, int grid, cudaStream_t s, AtomsView const &A, TablesView const &T) {
    switch (tpa) {
    case 1: k_force<OBS, KICK, 1, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    case 4: k_force<OBS, KICK, 4, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    case 8: k_force<OBS, KICK, 8, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    default: k_force<OBS, KICK, 16, IP, IX><<<grid, kBlock, 0, s>>>(A, T); break;
    }
}
template <bool OBS, bool KICK, int IP>
void force_tpa(int tpa, int grid, cudaStream_t s, AtomsView const &A, TablesView const &T) {
    if (A.pnbr16)
        force_tpa_ix<OBS, KICK, IP, uint16_t>(tpa, grid, s, A, T);
    else
        force_tpa_ix<OBS, KICK, IP, int>(tpa, grid, s, A, T);
}
template <int IP>
void density_ip(bool obs, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                TablesView const &T) {
    if (obs)
        density_tpa<true, IP>(tpa, grid, s, A, T);
    else
        density_tpa<false, IP>(tpa, grid, s, A, T);
}
template <int IP>
void force_ip(bool obs, bool kick, int tpa, int grid, cudaStream_t s, AtomsView const &A,
              TablesView const &T) {
    if (obs && kick)
        force_tpa<true, true, IP>(tpa, grid, s, A, T);
    else if (obs)
        force_tpa<true, false, IP>(tpa, grid, s, A, T);
    else if (kick)
        force_tpa<false, true, IP>(tpa, grid, s, A, T);
    else
        force_tpa<false, false, IP>(tpa, grid, s, A, T);
}
} // namespace

bool valid_tpa(int tpa) { return tpa == 1 || tpa == 4 || tpa == 8 || tpa == 16; }

void launch_density(bool obs, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                    TablesView const &T) {
    if (T.interp == MDELAST_BSPLINE)
        density_ip<MDELAST_BSPLINE>(obs, tpa, grid, s, A, T);
    else
        density_ip<MDELAST_QUINTIC>(obs, tpa, grid, s, A, T);
}

void launch_force(bool obs, bool kick, int tpa, int grid, cudaStream_t s, AtomsView const &A,
                  TablesView const &T) {
    if (T.interp == MDELAST_BSPLINE)
        force_ip<MDELAST_BSPLINE>(obs, kick, tpa, grid, s, A, T);
    else
        force_ip<MDELAST_QUINTIC>(obs, kick, tpa, grid, s, A, T);
}

} // namespace mdelast
