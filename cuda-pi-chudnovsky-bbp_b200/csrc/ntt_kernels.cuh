// ntt_kernels.cu -- the sm_100a kernels of one big-integer product.
//
// Launch sequence for N = 2^L >= 2^14 (a 2- or 3-pass plan, see make_plan):
//   A: k_fwd_first (u32 limbs -> 16-bit digits -> pass 1) , k_fwd_mid ...,
//      k_fwd_last (last pass; spectrum stored register-major per CTA)
//   B: k_fwd_first, k_fwd_mid ..., k_fused_last (last forward pass, pointwise
//      product with A's spectrum and 1/N, first inverse pass, all in registers)
//   inverse: k_inv_mid for the remaining passes (pass 1 yields the
//      coefficients in natural order), k_carry (decoupled-lookback carry into
//      u32 limbs + trimmed length).
// For N <= 2^13 one CTA does the whole product (k_mul_small).
//
// Reference counterpart: mul_ntt_cuda (src/ntt_cuda.cu:179-243) whose host
// repack (include/ntt.h:56-64), 2 x (log2 N + 1) forward launches, pointwise
// (:117-121), inverse launches and host carry (include/ntt.h:70-91) these
// kernels replace.
#pragma once
#include <cuda_runtime.h>

#include "b2m_internal.h"
#include "carry.cuh"
#include "ntt_engine.cuh"

namespace b2m {

// Global index of (row, column) in pass geometry (R = 2^LOGR, S = 2^logS):
// column g = b*S + c belongs to sub-problem b, whose rows are S apart.
template <int LOGR>
__device__ __forceinline__ u64 pass_gidx(u64 g, int row, int logS) {
    return ((g >> logS) << (LOGR + logS)) + ((u64)row << logS) + (g & ((1ull << logS) - 1));
}

// Exponent of the inter-pass twiddle w_M^(bitrev(row) * c), scaled to the
// 2^32 root: x = (bitrev(row) * c) * 2^(32 - logM) mod 2^32.
template <int LOGR>
__device__ __forceinline__ u32 twiddle_exp(int row, u64 c, int logM) {
    const u64 f = __brev((u32)row) >> (32 - LOGR);
    return (u32)((f * c) << (32 - logM));
}

// ---------------------------------------------------------------------------
// Pass 1 of a forward transform: reads u32 limbs as 16-bit digits (digit n is
// half n&1 of limb n>>1; digits at or past ndig are the zero padding).
// ---------------------------------------------------------------------------
template <int LOGR>
__global__ void __launch_bounds__(256) k_fwd_first(const u32* __restrict__ limbs, u64 ndig,
                                                   u64* __restrict__ out, int logS, int logC,
                                                   int logM, RootTables tw) {
    extern __shared__ u64 sm[];
    const Tile<LOGR, MAP_COL> tl{logC};
    u64 v[Tile<LOGR, MAP_COL>::EPT];
    const u64 g0 = (u64)blockIdx.x << logC;
    const u64 smask = (1ull << logS) - 1;
    auto src = [&](int row, int col, int) -> u64 {
        const u64 n = pass_gidx<LOGR>(g0 + col, row, logS);
        if (n >= ndig) return 0;
        const u32 w = __ldg(limbs + (n >> 1));
        return (n & 1) ? (u64)(w >> 16) : (u64)(w & 0xFFFFu);
    };
    auto dst = [&](int row, int col, int, u64 x) {
        const u64 g = g0 + col;
        const u32 e = twiddle_exp<LOGR>(row, g & smask, logM);
        if (e) x = gl_mul(x, uroot(e, tw.u1, tw.u2));
        out[pass_gidx<LOGR>(g, row, logS)] = x;
    };
    fwd_columns<LOGR, MAP_COL>(v, tl, sm, tw.dtw, src, dst);
}

// A later, not-last forward pass, in place.
template <int LOGR>
__global__ void __launch_bounds__(256) k_fwd_mid(u64* __restrict__ buf, int logS, int logC, int logM,
                                                 RootTables tw) {
    extern __shared__ u64 sm[];
    const Tile<LOGR, MAP_COL> tl{logC};
    u64 v[Tile<LOGR, MAP_COL>::EPT];
    const u64 g0 = (u64)blockIdx.x << logC;
    const u64 smask = (1ull << logS) - 1;
    auto src = [&](int row, int col, int) -> u64 { return buf[pass_gidx<LOGR>(g0 + col, row, logS)]; };
    auto dst = [&](int row, int col, int, u64 x) {
        const u64 g = g0 + col;
        const u32 e = twiddle_exp<LOGR>(row, g & smask, logM);
        if (e) x = gl_mul(x, uroot(e, tw.u1, tw.u2));
        buf[pass_gidx<LOGR>(g, row, logS)] = x;
    };
    fwd_columns<LOGR, MAP_COL>(v, tl, sm, tw.dtw, src, dst);
}

// A not-last inverse pass, in place: inverse inter-pass twiddle on load, then
// the inverse column DFTs. Pass 1 of the inverse leaves the convolution
// coefficients (times N^-1 already applied) in natural order.
template <int LOGR>
__global__ void __launch_bounds__(256) k_inv_mid(u64* __restrict__ buf, int logS, int logC, int logM,
                                                 RootTables tw) {
    extern __shared__ u64 sm[];
    const Tile<LOGR, MAP_COL> tl{logC};
    u64 v[Tile<LOGR, MAP_COL>::EPT];
    const u64 g0 = (u64)blockIdx.x << logC;
    const u64 smask = (1ull << logS) - 1;
    auto src = [&](int row, int col, int) -> u64 {
        const u64 g = g0 + col;
        u64 x = buf[pass_gidx<LOGR>(g, row, logS)];
        const u32 e = twiddle_exp<LOGR>(row, g & smask, logM);
        if (e) x = gl_mul(x, uroot(0u - e, tw.u1, tw.u2));
        return x;
    };
    auto dst = [&](int row, int col, int, u64 x) { buf[pass_gidx<LOGR>(g0 + col, row, logS)] = x; };
    inv_columns<LOGR, MAP_COL>(v, tl, sm, tw.dtw, src, dst);
}

// Last forward pass of operand A (S = 1: each column is a contiguous
// sub-problem). The spectrum is written register-major inside the CTA's own
// tile (slot * T + thread), the layout in which k_fused_last reads it back.
template <int LOGR>
__global__ void __launch_bounds__(256) k_fwd_last(u64* __restrict__ buf, int logC, RootTables tw) {
    extern __shared__ u64 sm[];
    const Tile<LOGR, MAP_ROW> tl{logC};
    u64 v[Tile<LOGR, MAP_ROW>::EPT];
    u64* base = buf + ((u64)blockIdx.x << (LOGR + logC));
    const int T = tl.nthreads();
    auto src = [&](int row, int col, int) -> u64 { return base[((u64)col << LOGR) + row]; };
    auto dst = [&](int, int, int slot, u64 x) { base[(u64)slot * T + threadIdx.x] = x; };
    fwd_columns<LOGR, MAP_ROW>(v, tl, sm, tw.dtw, src, dst);
}

// Last forward pass of operand B, pointwise product with A's spectrum and
// N^-1, then the first inverse pass -- one kernel, the spectra never leave
// registers.
template <int LOGR>
__global__ void __launch_bounds__(256) k_fused_last(u64* __restrict__ bbuf, const u64* __restrict__ aspec,
                                                    int logC, u64 ninv, RootTables tw) {
    extern __shared__ u64 sm[];
    const Tile<LOGR, MAP_ROW> tl{logC};
    u64 v[Tile<LOGR, MAP_ROW>::EPT];
    const u64 off = (u64)blockIdx.x << (LOGR + logC);
    u64* base = bbuf + off;
    const u64* abase = aspec + off;
    const int T = tl.nthreads();
    auto src = [&](int row, int col, int) -> u64 { return base[((u64)col << LOGR) + row]; };
    auto mul = [&](int, int, int slot, u64 x) {
        v[slot] = gl_mul(gl_mul(x, __ldg(abase + (u64)slot * T + threadIdx.x)), ninv);
    };
    fwd_columns<LOGR, MAP_ROW>(v, tl, sm, tw.dtw, src, mul);
    auto keep = [&](int, int, int slot) -> u64 { return v[slot]; };
    auto dst = [&](int row, int col, int, u64 x) { base[((u64)col << LOGR) + row] = x; };
    inv_columns<LOGR, MAP_ROW>(v, tl, sm, tw.dtw, keep, dst);
}

// ---------------------------------------------------------------------------
// Whole product in one CTA for N = 2^LOGN <= 2^13: both transforms live in
// shared memory, the carry is a block scan. T = N/64 threads (one for N < 64).
// ---------------------------------------------------------------------------
template <int LOGN>
__global__ void __launch_bounds__(128) k_mul_small(const u32* __restrict__ a, u64 na,
                                                   const u32* __restrict__ b, u64 nb,
                                                   u32* __restrict__ out, u64 nout,
                                                   unsigned long long* out_len, u64 ninv, RootTables tw) {
    using TL = Tile<LOGN, MAP_ROW>;
    constexpr int EPT = TL::EPT, RP = TL::RP;
    extern __shared__ u64 sm[];
    u64* smA = sm;
    u64* smB = sm + RP;
    CState* s_st = reinterpret_cast<CState*>(sm + 2 * RP);
    const TL tl{0};
    u64 v[EPT];
    const u64 nda = 2 * na, ndb = 2 * nb;
    auto digit = [](const u32* p, u64 nd, u64 n) -> u64 {
        if (n >= nd) return 0;
        const u32 w = __ldg(p + (n >> 1));
        return (n & 1) ? (u64)(w >> 16) : (u64)(w & 0xFFFFu);
    };
    auto to_smA = [&](int row, int, int, u64 x) { smA[tl.saddr(row, 0)] = x; };
    fwd_columns<LOGN, MAP_ROW>(v, tl, smA, tw.dtw, [&](int row, int, int) { return digit(a, nda, row); },
                               to_smA);
    __syncthreads();
    auto mul = [&](int row, int, int slot, u64 x) { v[slot] = gl_mul(gl_mul(x, smA[tl.saddr(row, 0)]), ninv); };
    fwd_columns<LOGN, MAP_ROW>(v, tl, smB, tw.dtw, [&](int row, int, int) { return digit(b, ndb, row); },
                               mul);
    auto keep = [&](int, int, int slot) -> u64 { return v[slot]; };
    auto to_smB = [&](int row, int, int, u64 x) { smB[tl.saddr(row, 0)] = x; };
    inv_columns<LOGN, MAP_ROW>(v, tl, smB, tw.dtw, keep, to_smB);
    __syncthreads();

    // Carry: thread t owns coefficients [t*EPT, (t+1)*EPT).
    const int T = tl.nthreads();
#pragma unroll
    for (int i = 0; i < EPT; ++i) v[i] = smB[tl.saddr((int)threadIdx.x * EPT + i, 0)];
    u32 lm[EPT / 2];
    const CState st = group_carry<EPT>(v, lm);
    s_st[threadIdx.x] = st;
    __syncthreads();
    __shared__ u64 s_top;
    if (threadIdx.x == 0) {
        // Serial exclusive scan (T <= 128): s_st[t] becomes the carry into t.
        u64 c = 0;
        for (int t = 0; t < T; ++t) {
            const CState f = s_st[t];
            s_st[t].h = c;
            c = cs_eval(f, c);
        }
        s_top = 0;
    }
    __syncthreads();
    group_add_carry<EPT / 2>(lm, s_st[threadIdx.x].h);
    const u64 lbase = (u64)threadIdx.x * (EPT / 2);
    unsigned long long top = 0;
#pragma unroll
    for (int i = 0; i < EPT / 2; ++i) {
        if (lbase + i < nout) {
            out[lbase + i] = lm[i];
            if (lm[i]) top = lbase + i + 1;
        }
    }
    if (top) atomicMax((unsigned long long*)&s_top, top);
    __syncthreads();
    if (threadIdx.x == 0 && out_len) *out_len = s_top;
}

}  // namespace b2m
