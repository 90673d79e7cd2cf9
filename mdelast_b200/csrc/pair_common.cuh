// Device helpers shared by the FP64 and the mixed-precision pair kernels.
#pragma once

#include "device.cuh"

namespace mdelast {

__device__ __forceinline__ void status_or(Replica *rep, unsigned bits) {
    atomicOr(&rep->obs.status, bits);
}

// a list build ran out of capacity: the rest of the launch's steps are skipped
__device__ __forceinline__ bool halted(AtomsView const &A) { return *A.halt != 0; }
__device__ __forceinline__ void set_halt(AtomsView const &A) { *A.halt = 1; }

// Block-wide sum of NS per-thread values into out[0..NS), warp shuffles then shared
// memory; deterministic for a fixed block size (NB threads).
template <int NS, int NB = kBlock>
__device__ __forceinline__ void block_sum_store(double (&v)[NS], double *out) {
    __shared__ double sm[NB / 32][NS];
    int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0)
            sm[warp][k] = x;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NS; k += blockDim.x) {
        double s = 0.;
#pragma unroll
        for (int w = 0; w < NB / 32; ++w)
            s += sm[w][k];
        out[k] = s;
    }
}

// TPA lanes (a power of two dividing 32) share one atom: lane `sub` takes the atom's list
// entries sub, sub + TPA, ... and the per-atom sums are combined across the lanes with
// shuffles. Every lane must reach the shuffles (padding lanes add zeros).
template <int TPA, typename V> __device__ __forceinline__ V group_sum(V x) {
#pragma unroll
    for (int o = TPA / 2; o > 0; o >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// list entry kk of an atom row: partners j > i at slots 0.., j < i at slots maxn-1 down
__device__ __forceinline__ int list_slot(int kk, int nu, int maxn) {
    return kk < nu ? kk : maxn - 1 - (kk - nu);
}

} // namespace mdelast
