// mdelast_pair_correlation_static: g(r) of one cell whose coordinates the caller already
// holds on the device, computed without allocating any device memory.
//
// It is a variant of the driver's pair-correlation pass (gr_kernels.cu): the same tile-pair
// counting with the reference's FP64 min-image, correctly rounded sqrt and divide, integer
// counters and the reference's normalisation order (md_driver.cpp:732-862), so its results
// equal mdelast_driver_pair_correlation's bit for bit on the same coordinates. What differs
// is where the scratch lives: the bin counters and the per-type atom counts sit in one
// file-scope __device__ array of fixed size instead of buffers from cudaMalloc, and the
// inputs come as plain device arrays (scaled coordinates n x 3, types n) rather than from a
// driver.
//
// Who needs it: callers that may not allocate device memory at the point of the call, for
// example an application whose allocator owns all device memory and forbids third-party
// cudaMalloc/cudaFree, or a sampling loop that cannot afford the device-wide
// synchronisation a cudaFree performs. They call this entry point; the scratch it uses is
// part of the library's loaded image.
#include <cuda_runtime.h>

#include <mutex>

#include "device.cuh"
#include "host_tables.h"

using namespace mdelast;

// The scratch: (1 + n_types(n_types+1)/2) x n_rg bin counters (at most
// MDELAST_GR_STATIC_MAX_SLOTS) followed by kMaxTypes per-type atom counts, 64-bit each.
// Every call clears the part it uses before counting.
static __device__ __align__(256) unsigned long long
    gr_static_scratch[MDELAST_GR_STATIC_MAX_SLOTS + kMaxTypes];

namespace {

constexpr int kTileS = 128;
constexpr size_t kSharedMaxS = 96 * 1024;

constexpr size_t kStaticSlots = MDELAST_GR_STATIC_MAX_SLOTS;

struct StaticArgs {
    const double *crd;     // n x 3 scaled coordinates
    const uint32_t *types; // n
    int n, ntypes, n_rg, mode;
    double hx, hy, hz, volume;
    const double *rg;
    unsigned long long *counts; // gr_static_scratch
    unsigned long long *n_per_type;
    double *gr, *gr_partial;
};

__device__ __forceinline__ double4 load_atom(StaticArgs const &g, int i) {
    return make_double4(g.crd[3 * i], g.crd[3 * i + 1], g.crd[3 * i + 2],
                        static_cast<double>(g.types[i]));
}

__device__ __forceinline__ void tile_pair_s(long q, int T, int &I, int &J) {
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

__global__ void k_gr_static_clear(StaticArgs g, int nslots) {
    int const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nslots)
        g.counts[k] = 0ull;
    if (k < g.ntypes)
        g.n_per_type[k] = 0ull;
}

__global__ void __launch_bounds__(kTileS) k_gr_static_count(StaticArgs g, int nslots,
                                                            int shared_hist) {
    extern __shared__ unsigned char s_raw[];
    double4 *sj = reinterpret_cast<double4 *>(s_raw);
    unsigned *sh = reinterpret_cast<unsigned *>(s_raw + sizeof(double4) * kTileS);
    int const T = (g.n + kTileS - 1) / kTileS;
    int I, J;
    tile_pair_s(blockIdx.x, T, I, J);
    if (shared_hist)
        for (int k = threadIdx.x; k < nslots; k += blockDim.x)
            sh[k] = 0u;
    int const j0 = J * kTileS;
    int const kmax = min(kTileS, g.n - j0);
    for (int k = threadIdx.x; k < kmax; k += blockDim.x)
        sj[k] = load_atom(g, j0 + k);
    __syncthreads();
    bool const total = g.mode == 0 || g.mode == 1, partial = g.mode == 1 || g.mode == 2;
    // bin width and range from the bin centres (md_driver.cpp:41)
    double const drg = __dadd_rn(g.rg[1], -g.rg[0]);
    double const rmaxg = __dadd_rn(g.rg[g.n_rg - 1], __dmul_rn(0.5, drg));
    double const r2_skip = rmaxg * rmaxg * (1. + 1e-12); // certainly outside beyond this
    int const i = I * kTileS + threadIdx.x;
    if (i < g.n && g.types[i] < static_cast<uint32_t>(g.ntypes)) {
        double4 const ci = load_atom(g, i);
        int const ti = static_cast<int>(ci.w);
        int const k0 = I == J ? static_cast<int>(threadIdx.x) + 1 : 0;
        for (int k = k0; k < kmax; ++k) {
            double4 const cj = sj[k];
            if (!(cj.w < g.ntypes)) // atoms of types outside [0, n_types) are not counted
                continue;
            double px, py, pz;
            double const r2 = min_image_r2(ci, cj, g.hx, g.hy, g.hz, px, py, pz);
            if (r2 >= r2_skip)
                continue;
            double const dr = __dsqrt_rn(r2);
            if (!(dr < rmaxg))
                continue;
            int const b = static_cast<int>(floor(__ddiv_rn(dr, drg)));
            if (b >= g.n_rg)
                continue;
            int const row = (1 + pair_slot(ti, static_cast<int>(cj.w))) * g.n_rg + b;
            if (shared_hist) {
                if (total)
                    atomicAdd(&sh[b], 1u);
                if (partial)
                    atomicAdd(&sh[row], 1u);
            } else {
                if (total)
                    atomicAdd(&g.counts[b], 1ull);
                if (partial)
                    atomicAdd(&g.counts[row], 1ull);
            }
        }
    }
    if (shared_hist) {
        __syncthreads();
        for (int k = threadIdx.x; k < nslots; k += blockDim.x)
            if (unsigned const c = sh[k])
                atomicAdd(&g.counts[k], static_cast<unsigned long long>(c));
    }
}

__global__ void k_gr_static_types(StaticArgs g) {
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < g.n && g.types[i] < static_cast<uint32_t>(g.ntypes))
        atomicAdd(&g.n_per_type[g.types[i]], 1ull);
}

// md_driver.cpp:749-751 and :786-810, in the reference's operation order
__global__ void k_gr_static_norm(StaticArgs g) {
    int const k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n_rg)
        return;
    double const pi = 3.14159265358979323846;
    double const V = g.volume;
    double const drg = __dadd_rn(g.rg[1], -g.rg[0]);
    double const r = g.rg[k];
    if (g.mode == 0 || g.mode == 1) {
        // N of the total's normalisation: the atoms counted (those with a type in range),
        // which is n_atoms whenever every type is valid
        unsigned long long nv = 0;
        for (int a = 0; a < g.ntypes; ++a)
            nv += g.n_per_type[a];
        double const nd = static_cast<double>(nv);
        double const den =
            __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(2. * pi, nd), nd), r), r), drg);
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
                    double const pref = __ddiv_rn(V, __dmul_rn(__dmul_rn(4. * pi, pc), drg));
                    v = __dmul_rn(static_cast<double>(g.counts[(1 + s) * g.n_rg + k]),
                                  __ddiv_rn(pref, __dmul_rn(r, r)));
                }
                g.gr_partial[static_cast<size_t>(s) * g.n_rg + k] = v;
            }
    }
}

// Address of gr_static_scratch on each device, looked up once per device (with that
// device current) on the first call made there.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
unsigned long long *g_scratch_ptr[kMaxDevices] = {};

int scratch_for_current_device(unsigned long long **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return fail(MDELAST_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(MDELAST_ERR_UNSUPPORTED, "device %d beyond the %d devices supported", dev,
                    kMaxDevices);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, gr_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(MDELAST_ERR_CUDA, "cudaGetSymbolAddress of the g(r) scratch: %s",
                        cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<unsigned long long *>(p);
    }
    *out = g_scratch_ptr[dev];
    return MDELAST_OK;
}

} // namespace

extern "C" int mdelast_pair_correlation_static(const double *coordinates, const uint32_t *types,
                                               int32_t n_atoms, int32_t n_types,
                                               const double *box, const double *rg,
                                               int32_t n_rg, int32_t mode, double *gr,
                                               double *gr_partial, void *stream) {
    clear_error();
    if (n_atoms < 0 || n_types < 1 || n_rg < 2 || mode < 0 || mode > 2 || !box || !rg ||
        (n_atoms > 0 && (!coordinates || !types)) || ((mode == 0 || mode == 1) && !gr) ||
        ((mode == 1 || mode == 2) && !gr_partial))
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    if (!(box[0] > 0.) || !(box[1] > 0.) || !(box[2] > 0.))
        return fail(MDELAST_ERR_ARGUMENT, "box edges must be positive");
    if (n_types > kMaxTypes)
        return fail(MDELAST_ERR_CAPACITY, "%d atom types; the static g(r) scratch holds %d",
                    n_types, kMaxTypes);
    size_t const nslots = static_cast<size_t>(1 + n_types * (n_types + 1) / 2) * n_rg;
    if (nslots > kStaticSlots)
        return fail(MDELAST_ERR_CAPACITY,
                    "%d bins x %d histograms need %zu counters; the static g(r) scratch holds "
                    "%zu (MDELAST_GR_STATIC_MAX_SLOTS)",
                    n_rg, 1 + n_types * (n_types + 1) / 2, nslots, kStaticSlots);
    long const T = (static_cast<long>(n_atoms) + kTileS - 1) / kTileS;
    if (T * (T + 1) / 2 > 2147483647L)
        return fail(MDELAST_ERR_CAPACITY,
                    "g(r) of %d atoms needs more than 2^31 - 1 blocks of %d-atom tile pairs",
                    n_atoms, kTileS);
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    unsigned long long *scratch = nullptr;
    if (int rc = scratch_for_current_device(&scratch))
        return rc;
    StaticArgs g{};
    g.crd = coordinates;
    g.types = types;
    g.n = n_atoms;
    g.ntypes = n_types;
    g.n_rg = n_rg;
    g.mode = mode;
    g.hx = box[0];
    g.hy = box[1];
    g.hz = box[2];
    g.volume = box[0] * (box[1] * box[2]); // Box::volume of a diagonal box
    g.rg = rg;
    g.counts = scratch;
    g.n_per_type = scratch + kStaticSlots;
    g.gr = gr;
    g.gr_partial = gr_partial;
    int const ns = static_cast<int>(nslots);
    k_gr_static_clear<<<(ns + 255) / 256, 256, 0, s>>>(g, ns);
    if (n_atoms >= 2) {
        size_t const tile_bytes = sizeof(double4) * kTileS;
        size_t const hist_bytes = sizeof(unsigned) * nslots;
        int const shared_hist = tile_bytes + hist_bytes <= kSharedMaxS ? 1 : 0;
        size_t const smem = tile_bytes + (shared_hist ? hist_bytes : 0);
        cudaError_t const e = cudaFuncSetAttribute(
            k_gr_static_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
            static_cast<int>(kSharedMaxS));
        if (e != cudaSuccess)
            return fail(MDELAST_ERR_CUDA, "%s", cudaGetErrorString(e));
        k_gr_static_count<<<static_cast<unsigned>(T * (T + 1) / 2), kTileS, smem, s>>>(
            g, ns, shared_hist);
    }
    if (n_atoms > 0)
        k_gr_static_types<<<(n_atoms + 255) / 256, 256, 0, s>>>(g);
    k_gr_static_norm<<<(n_rg + 255) / 256, 256, 0, s>>>(g);
    cudaError_t const e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(MDELAST_ERR_CUDA, "g(r) launch: %s", cudaGetErrorString(e));
    return MDELAST_OK;
}
