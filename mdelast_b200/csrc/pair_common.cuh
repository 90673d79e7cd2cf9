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

// minimum image of pi - pj in a box of edges L (positions wrapped into [-L/2, L/2))
__device__ __forceinline__ float min_image_f(float4 pi, float4 pj, float3 L, float3 iL,
                                             float &dx, float &dy, float &dz) {
    dx = __fsub_rn(pi.x, pj.x);
    dy = __fsub_rn(pi.y, pj.y);
    dz = __fsub_rn(pi.z, pj.z);
    dx = __fmaf_rn(-L.x, rintf(__fmul_rn(dx, iL.x)), dx);
    dy = __fmaf_rn(-L.y, rintf(__fmul_rn(dy, iL.y)), dy);
    dz = __fmaf_rn(-L.z, rintf(__fmul_rn(dz, iL.z)), dz);
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

__device__ __forceinline__ void box_f(Replica const *R, float3 &L, float3 &iL) {
    L = make_float3(static_cast<float>(R->h[0] / kAng), static_cast<float>(R->h[1] / kAng),
                    static_cast<float>(R->h[2] / kAng));
    iL = make_float3(1.f / L.x, 1.f / L.y, 1.f / L.z);
}

// Sum v over the warp (fixed order) and add it to this warp's shared accumulator.
__device__ __forceinline__ void warp_accumulate(double v, double *slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0)
        *slot += v;
}

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
