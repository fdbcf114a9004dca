// ntt_kernels.cuh -- kernel bodies of one big-integer product (templates;
// instantiated per radix in ntt_fam_*.cu).
//
// Launch sequence for N = 2^L >= 2^14 (a 2- or 3-pass plan, see make_plan):
//   A: k_fwd_first (u32 limbs -> 16-bit digits -> pass 1), k_fwd_mid ...,
//      k_fwd_last (last pass)
//   B: k_fwd_first, k_fwd_mid ..., k_fused_last (last forward pass, pointwise
//      product with A's spectrum and 1/N, first inverse pass, in one tile)
//   inverse: k_inv_mid for the remaining passes (pass 1 yields the
//      coefficients in natural order), k_carry (decoupled-lookback carry into
//      u32 limbs + trimmed length).
// For N <= 2^13 one CTA does the whole product (k_mul_small).
//
// Every pass kernel: a cooperative, coalesced load of its R x C tile into
// shared memory, the column DFTs in shared memory (ntt_engine.cuh), and a
// cooperative store (with the inter-pass twiddle on the way out for forward
// passes, on the way in for inverse passes).
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

constexpr int PASS_THREADS_MAX = 1024;

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

__device__ __forceinline__ u64 digit_of(const u32* __restrict__ limbs, u64 ndig, u64 n) {
    if (n >= ndig) return 0;
    const u32 w = __ldg(limbs + (n >> 1));
    return (n & 1) ? (u64)(w >> 16) : (u64)(w & 0xFFFFu);
}

// ---------------------------------------------------------------------------
// Pass 1 of a forward transform: u32 limbs read as 16-bit digits (digit n is
// half n&1 of limb n>>1; digits at or past ndig are the zero padding).
// ---------------------------------------------------------------------------
template <int LOGR>
__global__ void __launch_bounds__(PASS_THREADS_MAX) k_fwd_first(const u32* __restrict__ limbs, u64 ndig,
                                                                u64* __restrict__ out, int logS, int logC,
                                                                int logM, RootTables tw,
                                                                const ProdJob* __restrict__ jobs, int operand) {
    extern __shared__ u64 sm[];
    if (jobs) {
        const ProdJob& J = jobs[blockIdx.y];
        limbs = operand ? J.b : J.a;
        ndig = 2 * (operand ? J.nb : J.na);
        out = operand ? J.bufB : J.bufA;
    }
    const Tile<LOGR, MAP_COL> tl{logC};
    const u64 g0 = (u64)blockIdx.x << logC;
    const int cm = (1 << logC) - 1, total = (1 << LOGR) << logC;
    const u64 smask = (1ull << logS) - 1;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int col = idx & cm, row = idx >> logC;
        sm[tl.saddr(row, col)] = digit_of(limbs, ndig, pass_gidx<LOGR>(g0 + col, row, logS));
    }
    __syncthreads();
    tile_fwd<LOGR, MAP_COL>(sm, tl, tw.dtw);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int col = idx & cm, row = idx >> logC;
        const u64 g = g0 + col;
        u64 x = sm[tl.saddr(row, col)];
        const u32 e = twiddle_exp<LOGR>(row, g & smask, logM);
        if (e) x = gl_mul(x, uroot(e, tw.u1, tw.u2));
        out[pass_gidx<LOGR>(g, row, logS)] = x;
    }
}

// A later, not-last forward pass, in place.
template <int LOGR>
__global__ void __launch_bounds__(PASS_THREADS_MAX) k_fwd_mid(u64* __restrict__ buf, int logS, int logC, int logM,
                                                              RootTables tw, const ProdJob* __restrict__ jobs,
                                                              int operand) {
    extern __shared__ u64 sm[];
    if (jobs) buf = operand ? jobs[blockIdx.y].bufB : jobs[blockIdx.y].bufA;
    const Tile<LOGR, MAP_COL> tl{logC};
    const u64 g0 = (u64)blockIdx.x << logC;
    const int cm = (1 << logC) - 1, total = (1 << LOGR) << logC;
    const u64 smask = (1ull << logS) - 1;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int col = idx & cm, row = idx >> logC;
        sm[tl.saddr(row, col)] = buf[pass_gidx<LOGR>(g0 + col, row, logS)];
    }
    __syncthreads();
    tile_fwd<LOGR, MAP_COL>(sm, tl, tw.dtw);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int col = idx & cm, row = idx >> logC;
        const u64 g = g0 + col;
        u64 x = sm[tl.saddr(row, col)];
        const u32 e = twiddle_exp<LOGR>(row, g & smask, logM);
        if (e) x = gl_mul(x, uroot(e, tw.u1, tw.u2));
        buf[pass_gidx<LOGR>(g, row, logS)] = x;
    }
}

// A not-last inverse pass, in place: inverse inter-pass twiddle on load, then
// the inverse column DFTs. Pass 1 of the inverse leaves the convolution
// coefficients (N^-1 already applied) in natural order.
template <int LOGR>
__global__ void __launch_bounds__(PASS_THREADS_MAX) k_inv_mid(u64* __restrict__ buf, int logS, int logC, int logM,
                                                              RootTables tw, const ProdJob* __restrict__ jobs) {
    extern __shared__ u64 sm[];
    if (jobs) buf = jobs[blockIdx.y].bufB;
    const Tile<LOGR, MAP_COL> tl{logC};
    const u64 g0 = (u64)blockIdx.x << logC;
    const int cm = (1 << logC) - 1, total = (1 << LOGR) << logC;
    const u64 smask = (1ull << logS) - 1;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int col = idx & cm, row = idx >> logC;
        const u64 g = g0 + col;
        u64 x = buf[pass_gidx<LOGR>(g, row, logS)];
        const u32 e = twiddle_exp<LOGR>(row, g & smask, logM);
        if (e) x = gl_mul(x, uroot(0u - e, tw.u1, tw.u2));
        sm[tl.saddr(row, col)] = x;
    }
    __syncthreads();
    tile_inv<LOGR, MAP_COL>(sm, tl, tw.dtw);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int col = idx & cm, row = idx >> logC;
        buf[pass_gidx<LOGR>(g0 + col, row, logS)] = sm[tl.saddr(row, col)];
    }
}

// Last forward pass of operand A (S = 1: each column is a contiguous
// sub-problem, so the CTA's tile is one contiguous range of R*C elements).
template <int LOGR>
__global__ void __launch_bounds__(PASS_THREADS_MAX) k_fwd_last(u64* __restrict__ buf, int logC, RootTables tw,
                                                               const ProdJob* __restrict__ jobs) {
    extern __shared__ u64 sm[];
    if (jobs) buf = jobs[blockIdx.y].bufA;
    const Tile<LOGR, MAP_ROW> tl{logC};
    u64* base = buf + ((u64)blockIdx.x << (LOGR + logC));
    const int total = (1 << LOGR) << logC;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x)
        sm[tl.saddr(idx & ((1 << LOGR) - 1), idx >> LOGR)] = base[idx];
    __syncthreads();
    tile_fwd<LOGR, MAP_ROW>(sm, tl, tw.dtw);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x)
        base[idx] = sm[tl.saddr(idx & ((1 << LOGR) - 1), idx >> LOGR)];
}

// Last forward pass of operand B, pointwise product with A's spectrum (same
// positions) and N^-1, then the first inverse pass -- one tile, one kernel.
template <int LOGR>
__global__ void __launch_bounds__(PASS_THREADS_MAX) k_fused_last(u64* __restrict__ bbuf, const u64* __restrict__ aspec,
                                                                 int logC, u64 ninv, RootTables tw,
                                                                 const ProdJob* __restrict__ jobs) {
    extern __shared__ u64 sm[];
    if (jobs) {
        bbuf = jobs[blockIdx.y].bufB;
        aspec = jobs[blockIdx.y].bufA;
    }
    const Tile<LOGR, MAP_ROW> tl{logC};
    const u64 off = (u64)blockIdx.x << (LOGR + logC);
    u64* base = bbuf + off;
    const u64* abase = aspec + off;
    const int total = (1 << LOGR) << logC;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x)
        sm[tl.saddr(idx & ((1 << LOGR) - 1), idx >> LOGR)] = base[idx];
    __syncthreads();
    tile_fwd<LOGR, MAP_ROW>(sm, tl, tw.dtw);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int a = tl.saddr(idx & ((1 << LOGR) - 1), idx >> LOGR);
        sm[a] = gl_mul(gl_mul(sm[a], __ldg(abase + idx)), ninv);
    }
    __syncthreads();
    tile_inv<LOGR, MAP_ROW>(sm, tl, tw.dtw);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x)
        base[idx] = sm[tl.saddr(idx & ((1 << LOGR) - 1), idx >> LOGR)];
}

// ---------------------------------------------------------------------------
// Whole product in one CTA for N = 2^LOGN <= 2^13: both transforms live in
// shared memory, the carry is a block scan. max(1, N/16) threads; thread t
// owns coefficients [t*G, (t+1)*G), G = min(16, N).
// ---------------------------------------------------------------------------
template <int LOGN>
__global__ void __launch_bounds__(512) k_mul_small(const u32* __restrict__ a, u64 na, const u32* __restrict__ b,
                                                   u64 nb, u32* __restrict__ out, u64 nout,
                                                   unsigned long long* out_len, u64 ninv, RootTables tw,
                                                   const ProdJob* __restrict__ jobs) {
    if (jobs) {
        const ProdJob& J = jobs[blockIdx.x];
        a = J.a;
        b = J.b;
        na = J.na;
        nb = J.nb;
        out = J.out;
        nout = J.na + J.nb;
        out_len = J.out_len;
    }
    using TL = Tile<LOGN, MAP_ROW>;
    constexpr int N = 1 << LOGN, RP = TL::RP, G = N < 16 ? N : 16;
    extern __shared__ u64 sm[];
    u64* smA = sm;
    u64* smB = sm + RP;
    CState* s_st = reinterpret_cast<CState*>(sm + 2 * RP);
    __shared__ unsigned long long s_top;
    const TL tl{0};
    const u64 nda = 2 * na, ndb = 2 * nb;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        smA[tl.saddr(i, 0)] = digit_of(a, nda, i);
        smB[tl.saddr(i, 0)] = digit_of(b, ndb, i);
    }
    if (threadIdx.x == 0) s_top = 0;
    __syncthreads();
    tile_fwd<LOGN, MAP_ROW>(smA, tl, tw.dtw);
    tile_fwd<LOGN, MAP_ROW>(smB, tl, tw.dtw);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int s = tl.saddr(i, 0);
        smB[s] = gl_mul(gl_mul(smB[s], smA[s]), ninv);
    }
    __syncthreads();
    tile_inv<LOGN, MAP_ROW>(smB, tl, tw.dtw);

    // Carry: thread t owns G consecutive coefficients.
    const int T = blockDim.x;
    u64 v[G];
#pragma unroll
    for (int i = 0; i < G; ++i) v[i] = smB[tl.saddr((int)threadIdx.x * G + i, 0)];
    u32 lm[G / 2];
    const CState st = group_carry<G>(v, lm);
    s_st[threadIdx.x] = st;
    __syncthreads();
    if (threadIdx.x == 0) {
        // Serial exclusive scan (T <= 512): s_st[t].h becomes the carry into t.
        u64 c = 0;
        for (int t = 0; t < T; ++t) {
            const CState f = s_st[t];
            s_st[t].h = c;
            c = cs_eval(f, c);
        }
    }
    __syncthreads();
    group_add_carry<G / 2>(lm, s_st[threadIdx.x].h);
    const u64 lbase = (u64)threadIdx.x * (G / 2);
    unsigned long long top = 0;
#pragma unroll
    for (int i = 0; i < G / 2; ++i) {
        if (lbase + i < nout) {
            out[lbase + i] = lm[i];
            if (lm[i]) top = lbase + i + 1;
        }
    }
    if (top) atomicMax(&s_top, top);
    __syncthreads();
    if (threadIdx.x == 0 && out_len) *out_len = s_top;
}

}  // namespace b2m
