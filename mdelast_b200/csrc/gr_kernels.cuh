// Pair correlation g(r) of one replica on the device (md_driver.cpp:732-862).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace mdelast {

struct Replica;

struct GrArgs {
    const double4 *crd;      // the replica's scaled coordinates, type in .w (n entries)
    const Replica *rep;      // its state on the device: the current box edges h[3]
    int n, ntypes, n_rg, mode; // mode 0 total, 1 total + partial, 2 partial only
    const double *rg;        // bin centres (device), evenly spaced, rg[0] > 0
    double drg, rmaxg;       // rg[1] - rg[0], rg[n_rg - 1] + drg / 2 (md_driver.cpp:41)
    unsigned long long *counts; // scratch: gr_count_slots(n_rg, ntypes) counters
    int *n_per_type;         // scratch: ntypes counters
    double *gr, *gr_partial; // outputs (device): n_rg, and ntypes(ntypes+1)/2 x n_rg
};

// counters of one replica's histograms: the total, then one row per type pair
__host__ __device__ inline size_t gr_count_slots(int n_rg, int ntypes) {
    return static_cast<size_t>(1 + ntypes * (ntypes + 1) / 2) * static_cast<size_t>(n_rg);
}
// Thread blocks of the pair count for n atoms: one per pair of 128-atom tiles (I <= J).
// A launch takes at most 2^31 - 1 blocks, so callers reject n beyond gr_max_atoms().
constexpr long kGrTileAtoms = 128;
__host__ inline long gr_count_blocks(long n) {
    long const T = (n + kGrTileAtoms - 1) / kGrTileAtoms;
    return T * (T + 1) / 2;
}
__host__ inline bool gr_atoms_fit(long n) { return gr_count_blocks(n) <= 2147483647L; }
// Clears the scratch, counts the pairs, normalises. Asynchronous on stream s; gr is left
// untouched for mode 2 and gr_partial for mode 0, as in the reference.
cudaError_t gr_enqueue(GrArgs const &g, cudaStream_t s);

} // namespace mdelast
