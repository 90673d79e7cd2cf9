// Pair correlation g(r) of one replica (md_driver.cpp:732-862): every pair i < j with
// min-image distance dr < rmaxg adds one to bin floor(dr / drg) of the total histogram
// and, by type pair, of the partial one; then the reference's normalisations.
//
// Counting is exact: dr comes from the same FP64 operations as the reference's (the
// min-image arithmetic the neighbour list uses, a correctly rounded sqrt and divide), so
// every pair lands in the reference's bin; integer counters make the sum order-free; and
// the normalisation repeats the reference's operation order without contraction, so g(r)
// equals the reference's to the last bit.
//
// Work split: one block per pair of 128-atom tiles (I <= J) of the replica; the J tile is
// staged in shared memory and each thread scans it for its own atom of tile I. Counts go to
// a per-block shared histogram when it fits (one atomic per non-zero bin flushes it), else
// straight to the global counters. O(N^2 / 2) pair tests: about 91 M for 13,500 atoms.
#include "gr_kernels.cuh"

#include "device.cuh"

namespace mdelast {

namespace {

constexpr int kGrTile = static_cast<int>(kGrTileAtoms);
constexpr size_t kGrSharedMax = 96 * 1024;

// block index q -> tile pair (I, J), I <= J, rows of the upper triangle of T x T tiles
__device__ __forceinline__ void tile_pair(long q, int T, int &I, int &J) {
    int i = 0;
    long rowlen = T;
    while (q >= rowlen) {
        q -= rowlen;
        ++i;
        --rowlen;
    }
    I = i;
    J = i + static_cast<int>(q);
}

__global__ void __launch_bounds__(kGrTile)
    k_gr_count(GrArgs g, double r2_skip, int shared_hist) {
    extern __shared__ unsigned char s_raw[];
    double4 *sj = reinterpret_cast<double4 *>(s_raw);
    unsigned *sh = reinterpret_cast<unsigned *>(s_raw + sizeof(double4) * kGrTile);
    int const nbins = static_cast<int>(gr_count_slots(g.n_rg, g.ntypes));
    int const T = (g.n + kGrTile - 1) / kGrTile;
    int I, J;
    tile_pair(blockIdx.x, T, I, J);
    if (shared_hist)
        for (int k = threadIdx.x; k < nbins; k += blockDim.x)
            sh[k] = 0u;
    int const j0 = J * kGrTile;
    int const kmax = min(kGrTile, g.n - j0);
    for (int k = threadIdx.x; k < kmax; k += blockDim.x)
        sj[k] = g.crd[j0 + k];
    __syncthreads();
    double const hx = g.rep->h[0], hy = g.rep->h[1], hz = g.rep->h[2];
    bool const total = g.mode == 0 || g.mode == 1, partial = g.mode == 1 || g.mode == 2;
    int const i = I * kGrTile + threadIdx.x;
    if (i < g.n) {
        double4 const ci = g.crd[i];
        int const ti = static_cast<int>(ci.w);
        // the diagonal tile counts only j > i
        int const k0 = I == J ? static_cast<int>(threadIdx.x) + 1 : 0;
        for (int k = k0; k < kmax; ++k) {
            double4 const cj = sj[k];
            double px, py, pz;
            double const r2 = min_image_r2(ci, cj, hx, hy, hz, px, py, pz);
            if (r2 >= r2_skip) // certainly dr >= rmaxg
                continue;
            double const dr = __dsqrt_rn(r2);
            if (!(dr < g.rmaxg))
                continue;
            int const b = static_cast<int>(floor(__ddiv_rn(dr, g.drg)));
            if (b >= g.n_rg) // unreachable for evenly spaced rg; the reference asserts it
                continue;
            if (shared_hist) {
                if (total)
                    atomicAdd(&sh[b], 1u);
                if (partial)
                    atomicAdd(&sh[(1 + pair_slot(ti, static_cast<int>(cj.w))) * g.n_rg + b],
                              1u);
            } else {
                if (total)
                    atomicAdd(&g.counts[b], 1ull);
                if (partial)
                    atomicAdd(&g.counts[(1 + pair_slot(ti, static_cast<int>(cj.w))) * g.n_rg +
                                        b],
                              1ull);
            }
        }
    }
    if (shared_hist) {
        __syncthreads();
        for (int k = threadIdx.x; k < nbins; k += blockDim.x)
            if (unsigned const c = sh[k])
                atomicAdd(&g.counts[k], static_cast<unsigned long long>(c));
    }
}

__global__ void k_count_types(GrArgs g) {
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < g.n)
        atomicAdd(&g.n_per_type[static_cast<int>(g.crd[i].w)], 1);
}

// md_driver.cpp:749-751 (total) and :786-810 (partial), in the reference's operation order
__global__ void k_gr_norm(GrArgs g) {
    int const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n_rg)
        return;
    double const pi = 3.14159265358979323846;
    // Box::volume of a diagonal box: h00 * (h11 * h22), the other cofactor terms vanish
    double const V = __dmul_rn(g.rep->h[0], __dmul_rn(g.rep->h[1], g.rep->h[2]));
    double const r = g.rg[k];
    if (g.mode == 0 || g.mode == 1) {
        double const nd = static_cast<double>(g.n);
        double const den =
            __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(2. * pi, nd), nd), r), r), g.drg);
        g.gr[k] = __dmul_rn(static_cast<double>(g.counts[k]), __ddiv_rn(V, den));
    }
    if (g.mode == 1 || g.mode == 2) {
        int s = 0;
        for (int b = 0; b < g.ntypes; ++b)
            for (int a = 0; a <= b; ++a, ++s) {
                double const Na = static_cast<double>(g.n_per_type[a]);
                double const Nb = static_cast<double>(g.n_per_type[b]);
                double pc = 0.;
                if (a == b) {
                    if (Na > 1)
                        pc = __ddiv_rn(__dmul_rn(Na, __dadd_rn(Na, -1.)), 2.);
                } else {
                    pc = __dmul_rn(Na, Nb);
                }
                double v = 0.;
                if (pc > 0.) {
                    double const pref = __ddiv_rn(V, __dmul_rn(__dmul_rn(4. * pi, pc), g.drg));
                    v = __dmul_rn(static_cast<double>(g.counts[(1 + s) * g.n_rg + k]),
                                  __ddiv_rn(pref, __dmul_rn(r, r)));
                }
                g.gr_partial[static_cast<size_t>(s) * g.n_rg + k] = v;
            }
    }
}

} // namespace

cudaError_t gr_enqueue(GrArgs const &g, cudaStream_t s) {
    size_t const nbins = gr_count_slots(g.n_rg, g.ntypes);
    cudaError_t e = cudaMemsetAsync(g.counts, 0, sizeof(unsigned long long) * nbins, s);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(g.n_per_type, 0, sizeof(int) * g.ntypes, s);
    if (e != cudaSuccess)
        return e;
    if (g.n >= 2) {
        long const blocks = gr_count_blocks(g.n);
        size_t const tile_bytes = sizeof(double4) * kGrTile;
        size_t const hist_bytes = sizeof(unsigned) * nbins;
        int const shared_hist = tile_bytes + hist_bytes <= kGrSharedMax ? 1 : 0;
        size_t const smem = tile_bytes + (shared_hist ? hist_bytes : 0);
        e = cudaFuncSetAttribute(k_gr_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kGrSharedMax));
        if (e != cudaSuccess)
            return e;
        // squared distances at or beyond this are certainly outside rmaxg after the sqrt
        double const r2_skip = g.rmaxg * g.rmaxg * (1. + 1e-12);
        k_gr_count<<<static_cast<unsigned>(blocks), kGrTile, smem, s>>>(g, r2_skip,
                                                                       shared_hist);
    }
    if (g.n > 0)
        k_count_types<<<(g.n + 255) / 256, 256, 0, s>>>(g);
    k_gr_norm<<<(g.n_rg + 255) / 256, 256, 0, s>>>(g);
    return cudaGetLastError();
}

} // namespace mdelast
