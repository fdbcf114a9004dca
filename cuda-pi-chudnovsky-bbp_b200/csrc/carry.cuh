// carry.cuh -- carry propagation from convolution coefficients to u32 limbs.
//
// Reference counterpart: carry_propagate (include/ntt.h:70-91), a sequential
// host loop. Here every group of G coefficients (G even) is normalised
// independently into G base-2^16 digits (G/2 limbs) plus its carry-out H,
// ignoring the carry coming in. A carry-in c (always < 2^62) then changes the
// group's carry-out by at most one, and only if c >= T = 2^(16G) - D where D
// is the group's digit value. So each group is the function
//     f(c) = H + [c >= T]     (T = "never" unless D's top bits are all ones)
// and functions of this form are closed under composition, which turns the
// whole carry into a prefix scan over groups (decoupled lookback across CTAs,
// shuffles and shared memory inside a CTA).
#pragma once
#include "gl.cuh"

namespace b2m {

constexpr u64 CS_NEVER = ~0ull;

struct CState {
    u64 h;  // carry-out when the carry-in is below t
    u64 t;  // threshold; CS_NEVER means the carry-out is h for every carry-in
};

// g after f (f applies first).
__device__ __forceinline__ CState cs_then(CState f, CState g) {
    if (f.h >= g.t) return {g.h + 1, CS_NEVER};
    if (f.h + 1 == g.t) return {g.h, f.t};
    return {g.h, CS_NEVER};
}

__device__ __forceinline__ u64 cs_eval(CState f, u64 c) { return f.h + (c >= f.t ? 1ull : 0ull); }

// Normalise G coefficients (each < 2^61) into G/2 limbs; returns the group's
// carry function. Coefficient 2i lands in the low half of limb i.
template <int G>
__device__ __forceinline__ CState group_carry(const u64* coef, u32* limb) {
    static_assert(G >= 4 && (G % 2) == 0, "group of at least two limbs");
    u64 c = 0;
#pragma unroll
    for (int i = 0; i < G; i += 2) {
        u64 x0 = coef[i] + c;
        c = x0 >> 16;
        u64 x1 = coef[i + 1] + c;
        c = x1 >> 16;
        limb[i / 2] = (u32)(x0 & 0xFFFFu) | ((u32)(x1 & 0xFFFFu) << 16);
    }
    bool upper_ones = true;
#pragma unroll
    for (int i = 2; i < G / 2; ++i) upper_ones &= (limb[i] == 0xFFFFFFFFu);
    const u64 dl = (u64)limb[0] | ((u64)limb[1] << 32);
    u64 t = CS_NEVER;
    if (upper_ones && dl != 0) {
        const u64 tt = 0ull - dl;  // 2^64 - dl
        if (tt < (1ull << 62)) t = tt;
    }
    return {c, t};
}

// Add a carry-in (< 2^62) into G/2 limbs; overflow past the group is already
// accounted for by the group's carry function and is dropped here.
template <int NL>
__device__ __forceinline__ void group_add_carry(u32* limb, u64 cin) {
    u64 s = (u64)limb[0] + (cin & 0xFFFFFFFFull);
    limb[0] = (u32)s;
    u64 k = (s >> 32) + (cin >> 32);
#pragma unroll
    for (int i = 1; i < NL; ++i) {
        s = (u64)limb[i] + k;
        limb[i] = (u32)s;
        k = s >> 32;
    }
}

__device__ __forceinline__ CState cs_shfl_up(CState s, int off) {
    CState r;
    r.h = __shfl_up_sync(0xFFFFFFFFu, s.h, off);
    r.t = __shfl_up_sync(0xFFFFFFFFu, s.t, off);
    return r;
}

// Block-wide exclusive scan of carry functions. Returns the thread's
// exclusive prefix (valid only when *has_prefix), and the block aggregate in
// *agg (all threads). `ws` needs one CState per warp. One barrier: every warp
// scans the warp aggregates itself with shuffles (no serial pass on one
// thread, no second barrier); callers synchronise before writing `ws` again.
__device__ __forceinline__ CState block_scan_carry(CState st, bool* has_prefix, CState* agg, CState* ws) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    CState inc = st;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        CState o = cs_shfl_up(inc, off);
        if (lane >= off) inc = cs_then(o, inc);
    }
    CState exw = cs_shfl_up(inc, 1);
    if (lane == 31 || (int)threadIdx.x == (int)blockDim.x - 1) ws[warp] = inc;
    __syncthreads();
    // inclusive scan of the warp aggregates, lanes [0, nwarps) meaningful
    CState wv = ws[lane < nwarps ? lane : nwarps - 1];
    for (int off = 1; off < nwarps; off <<= 1) {
        CState o = cs_shfl_up(wv, off);
        if (lane >= off) wv = cs_then(o, wv);
    }
    CState a;
    a.h = __shfl_sync(0xFFFFFFFFu, wv.h, nwarps - 1);
    a.t = __shfl_sync(0xFFFFFFFFu, wv.t, nwarps - 1);
    *agg = a;
    CState exb;  // inclusive aggregate of the warps before this one
    exb.h = __shfl_sync(0xFFFFFFFFu, wv.h, warp > 0 ? warp - 1 : 0);
    exb.t = __shfl_sync(0xFFFFFFFFu, wv.t, warp > 0 ? warp - 1 : 0);
    CState ex;
    bool has = false;
    if (warp > 0) {
        ex = exb;
        has = true;
    }
    if (lane > 0) {
        ex = has ? cs_then(ex, exw) : exw;
        has = true;
    }
    *has_prefix = has;
    return ex;
}

}  // namespace b2m
