// gp_scan.cuh -- carry (or borrow) propagation of multi-limb additions as a
// parallel prefix over (generate, propagate) pairs.
//
// A group of limbs generates a carry out (g) or passes a carry in through (p);
// groups compose associatively, so a carry chain of any length is a scan.
// Used by the signed add of the Chudnovsky merge and by the big-integer
// add/subtract kernels. Reference counterpart: the sequential carry loops of
// add_mag / sub_mag (src/bignum.cpp:63-104).
#pragma once
#include "gl.cuh"

namespace b2m {

struct GP {
    u32 g, p;
};
__device__ __forceinline__ GP gp_then(GP lo, GP hi) { return {hi.g | (hi.p & lo.g), hi.p & lo.p}; }

constexpr int ADD_LPT = 8;  // limbs per thread

// Exclusive block scan of GP (low threads first). blockDim multiple of 32.
__device__ __forceinline__ GP block_scan_gp(GP v, GP* ws, GP* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    GP inc = v;
    for (int off = 1; off < 32; off <<= 1) {
        GP o{__shfl_up_sync(0xFFFFFFFFu, inc.g, off), __shfl_up_sync(0xFFFFFFFFu, inc.p, off)};
        if (lane >= off) inc = gp_then(o, inc);
    }
    GP ex{__shfl_up_sync(0xFFFFFFFFu, inc.g, 1), __shfl_up_sync(0xFFFFFFFFu, inc.p, 1)};
    if (lane == 0) ex = {0, 1};
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        GP acc{0, 1};
        for (int w = 0; w < nw; ++w) {
            GP t = ws[w];
            ws[w] = acc;
            acc = gp_then(acc, t);
        }
        ws[nw] = acc;
    }
    __syncthreads();
    *total = ws[nw];
    return gp_then(ws[warp], ex);
}

}  // namespace b2m
