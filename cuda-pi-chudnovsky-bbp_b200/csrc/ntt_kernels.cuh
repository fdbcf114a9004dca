// ntt_kernels.cuh -- kernel bodies of one big-integer product (templates;
// instantiated per radix in ntt_fam_*.cu).
//
// Launch sequence for N = 2^L >= 2^14 (a 2- or 3-pass plan, see make_plan):
//   A: k_fwd_first (u32 limbs -> 16-bit digits -> pass 1), k_fwd_mid ...,
//      k_fwd_last (last pass)
//   B: k_fwd_first, k_fwd_mid ..., k_fused_last (last forward pass, pointwise
//      product with A's spectrum, first inverse pass, in one tile)
//   inverse: k_inv_mid for the remaining passes (pass 1 yields N times the
//      coefficients in natural order), k_carry (scale by 1/N, then the
//      decoupled-lookback carry into u32 limbs + trimmed length).
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
#include "school.cuh"

namespace b2m {

constexpr int PASS_THREADS_MAX = 1024;

// Occupancy target of every pass kernel: 1024 resident threads per SM
// (64 registers a thread), whatever the tile's thread count.
#define B2M_PASS_BOUNDS(T) __launch_bounds__((T), (PASS_THREADS_MAX / (T)))

// Asynchronous 8-byte copy global -> shared (no register staging, so a
// thread keeps all of its tile loads in flight), and the wait for all of the
// thread's copies.
__device__ __forceinline__ void cp_async8(u64* smem_dst, const u64* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void cp_async16(u64* smem_dst, const u64* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ ulonglong2 ldg2(const u64* p) { return __ldg(reinterpret_cast<const ulonglong2*>(p)); }

__device__ __forceinline__ u64 digit_of(const u32* __restrict__ limbs, u64 ndig, u64 n) {
    if (n >= ndig) return 0;
    const u32 w = __ldg(limbs + (n >> 1));
    return (n & 1) ? (u64)(w >> 16) : (u64)(w & 0xFFFFu);
}

// Digits of K consecutive rows of a thread's column into shared memory. A
// thread's elements gi0 + k*gstep share the parity of gi0 (gstep is even), so
// each takes the same half of its limb; when the last of them is below ndig
// (every tile but the operand's last) no element needs the bounds check.
template <int K, class G>
__device__ __forceinline__ void load_digits(u64* sm, const G& gp, const u32* __restrict__ limbs, u64 ndig) {
    if (!(gp.gstep & 1) && gp.gi0 + (u64)(K - 1) * gp.gstep < ndig) {
        const u32* lp = limbs + (gp.gi0 >> 1);
        const u64 ls = gp.gstep >> 1;
        const u32 sh = (u32)(gp.gi0 & 1) << 4;
#pragma unroll
        for (int k = 0; k < K; ++k) sm[gp.sa0 + G::soff(k)] = (u64)((__ldg(lp + k * ls) >> sh) & 0xFFFFu);
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) sm[gp.sa0 + G::soff(k)] = digit_of(limbs, ndig, gp.gi0 + k * gp.gstep);
    }
}

// Digits of K chunks of column pairs (ColPair): digit pair n, n+1 (n even)
// is one u32 limb, and n < ndig (ndig even) covers both digits.
template <int K, class P>
__device__ __forceinline__ void load_digit_pairs(u64* sm, const P& pp, const u32* __restrict__ limbs, u64 ndig) {
    if (pp.gi0 + (u64)(K - 1) * pp.gstep < ndig) {
        const u32* lp = limbs + (pp.gi0 >> 1);
        const u64 ls = pp.gstep >> 1;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const u32 w = __ldg(lp + j * ls);
            st2(sm + pp.sa0 + P::soff(j), make_ulonglong2(w & 0xFFFFu, w >> 16));
        }
    } else {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const u64 n = pp.gi0 + j * pp.gstep;
            const u32 w = n < ndig ? __ldg(limbs + (n >> 1)) : 0u;
            st2(sm + pp.sa0 + P::soff(j), make_ulonglong2(w & 0xFFFFu, w >> 16));
        }
    }
}

// Column-mapped pass geometry (first, middle and non-last inverse passes).
// The tile is rows [0, R) of columns [g0, g0 + C), C <= S, so all of it lies in
// one sub-problem b = g0 >> logS. Thread t owns column col = t mod C and rows
// row0 + k*DR (row0 = t / C, DR = R/16, k < 16): its global indices step by
// DR*S, its shared addresses by a compile-time offset, and the bit-reversed
// row is brev(row0) + brev(k*DR) (disjoint bits), so the inter-pass twiddle
// exponent w_M^(brev(row) * c) is e0 + brev(k*DR) * (c << (32 - logM)).
template <class TL>
struct ColPass {
    static constexpr int DR = TL::T >> TL::LC;
    static constexpr int PER = (TL::R * TL::C) / TL::T;
    static_assert(PER == 16 && DR >= 1, "16 elements per thread");
    int col, row0, sa0;
    u64 gi0, gstep, ti0;  // ti0: index in the pass's twiddle table (row0, c)
    u32 e0, ec;
    __device__ __forceinline__ ColPass(int logS, int logM) {
        col = (int)threadIdx.x & (TL::C - 1);
        row0 = (int)threadIdx.x >> TL::LC;
        sa0 = TL::saddr(row0, col);
        const u64 g = ((u64)blockIdx.x << TL::LC) + col;
        const u64 c = g & ((1ull << logS) - 1);
        gi0 = ((g >> logS) << (TL::LR + logS)) + ((u64)row0 << logS) + c;
        ti0 = ((u64)row0 << logS) + c;
        gstep = (u64)DR << logS;
        const u32 sh = 32 - logM;
        const u32 f0 = __brev((u32)row0) >> (32 - TL::LR);
        ec = (u32)c << sh;
        e0 = f0 * ec;
    }
    // shared-address offset and bit-reversed row part of element k
    static constexpr int soff(int k) { return (k * DR + ((k * DR) >> 6)) << TL::LC; }
    static constexpr u32 fk(int k) { return (u32)brev_c(k * DR, TL::LR); }
};

// The same tile moved as 16-byte column pairs: thread t moves columns
// 2*(t mod C/2) and the next one of rows r0 + j*DR2 (r0 = t / (C/2) < DR2,
// j < 8). Pairs start at even columns of a sub-problem of stride S >= C, so
// the global, table and shared addresses are 16-byte aligned, and r0 < DR2
// with DR2 a power of two keeps the padded shared offsets linear in j.
template <class TL>
struct ColPair {
    static constexpr int CP = TL::C / 2;
    static constexpr int DR2 = TL::T / CP;
    static constexpr int PER = (TL::R * CP) / TL::T;
    static_assert(TL::LC >= 1 && PER == 8, "column pairs: eight 16-byte chunks per thread");
    int sa0;
    u64 gi0, gstep, ti0;
    __device__ __forceinline__ explicit ColPair(int logS) {
        const int cp = (int)threadIdx.x & (CP - 1);
        const int r0 = (int)threadIdx.x / CP;
        sa0 = TL::saddr(r0, 2 * cp);
        const u64 g = ((u64)blockIdx.x << TL::LC) + 2 * cp;
        const u64 c = g & ((1ull << logS) - 1);
        gi0 = ((g >> logS) << (TL::LR + logS)) + ((u64)r0 << logS) + c;
        ti0 = ((u64)r0 << logS) + c;
        gstep = (u64)DR2 << logS;
    }
    static constexpr int soff(int j) { return (j * DR2 + ((j * DR2) >> 6)) << TL::LC; }
};

// Row-mapped (contiguous) tile of the last forward / first inverse pass:
// element idx = t + k*T of the R*C block, row idx mod R, column idx / R.
template <class TL>
struct RowPass {
    static_assert(TL::T >= 64, "row-mapped tiles have at least 64 threads");
    static constexpr int PER = (TL::R * TL::C) / TL::T;
    int sa0;
    __device__ __forceinline__ RowPass() {
        const int t = (int)threadIdx.x;
        sa0 = TL::T >= TL::R ? TL::saddr(t & (TL::R - 1), t >> TL::LR) : TL::saddr(t, 0);
    }
    static constexpr int KR = TL::T >= TL::R ? 1 : TL::R / TL::T;  // loop steps per column
    static constexpr int soff(int k) {
        if (TL::T >= TL::R) return k * (TL::T >> TL::LR) * TL::RP;
        const int kr = k % KR, kc = k / KR;
        return kc * TL::RP + kr * TL::T + ((kr * TL::T) >> 6);
    }
};

// ---------------------------------------------------------------------------
// Pass 1 of a forward transform: u32 limbs read as 16-bit digits (digit n is
// half n&1 of limb n>>1; digits at or past ndig are the zero padding).
// ---------------------------------------------------------------------------
template <int LOGR, int LOGC>
__global__ void B2M_PASS_BOUNDS((Tile<LOGR, LOGC, MAP_COL>::T))
k_fwd_first(const u32* __restrict__ limbs, u64 ndig, u64* __restrict__ out, int logS, int logM, RootTables tw,
            const u64* __restrict__ ttab, const ProdJob* __restrict__ jobs, int operand) {
    using TL = Tile<LOGR, LOGC, MAP_COL>;
    using G = ColPass<TL>;
    extern __shared__ u64 sm[];
    if (jobs) {
        const ProdJob& J = jobs[blockIdx.y];
        limbs = operand ? J.b : J.a;
        ndig = 2 * (operand ? J.nb : J.na);
        out = operand ? J.bufB : J.bufA;
    }
    const G gp(logS, logM);
    // The digits fill at most half of the transform for almost every product
    // (N >= 2 (na + nb)): rows [R/2, R) of every column are then zero, and
    // the half-zero tile transform neither reads nor needs them. Tiles of
    // two or more columns move digit pairs (one limb each).
    if (2 * ndig <= (1ull << logM)) {
        if constexpr (TL::LC >= 1) load_digit_pairs<4>(sm, ColPair<TL>(logS), limbs, ndig);  // rows < R/2
        else load_digits<G::PER / 2>(sm, gp, limbs, ndig);  // rows row0 + k*DR < R/2
        __syncthreads();
        tile_fwd<TL, fwd_rt<TL>(), true>(sm, tw.dtw);
    } else {
        if constexpr (TL::LC >= 1) load_digit_pairs<8>(sm, ColPair<TL>(logS), limbs, ndig);
        else load_digits<G::PER>(sm, gp, limbs, ndig);
        __syncthreads();
        tile_fwd<TL>(sm, tw.dtw);
    }
    if constexpr (TL::LC >= 1) {
        if (ttab) {
            const ColPair<TL> pp(logS);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                ulonglong2 v = ld2(sm + pp.sa0 + ColPair<TL>::soff(j));
                const ulonglong2 t = ldg2(ttab + pp.ti0 + j * pp.gstep);
                v.x = gl_mul(v.x, t.x);
                v.y = gl_mul(v.y, t.y);
                st2(out + pp.gi0 + j * pp.gstep, v);
            }
            return;
        }
    }
    if (ttab) {
#pragma unroll
        for (int k = 0; k < G::PER; ++k)
            out[gp.gi0 + k * gp.gstep] = gl_mul(sm[gp.sa0 + G::soff(k)], __ldg(ttab + gp.ti0 + k * gp.gstep));
    } else {
#pragma unroll
        for (int k = 0; k < G::PER; ++k) {
            u64 x = sm[gp.sa0 + G::soff(k)];
            const u32 e = gp.e0 + G::fk(k) * gp.ec;
            if (e) x = gl_mul(x, uroot(e, tw.u1, tw.u2));
            out[gp.gi0 + k * gp.gstep] = x;
        }
    }
}

// A later, not-last forward pass, in place.
template <int LOGR, int LOGC>
__global__ void B2M_PASS_BOUNDS((Tile<LOGR, LOGC, MAP_COL>::T))
k_fwd_mid(u64* __restrict__ buf, int logS, int logM, RootTables tw, const u64* __restrict__ ttab,
          const ProdJob* __restrict__ jobs, int operand, u64 zstride) {
    using TL = Tile<LOGR, LOGC, MAP_COL>;
    using G = ColPass<TL>;
    extern __shared__ u64 sm[];
    if (jobs) buf = operand ? jobs[blockIdx.y].bufB : jobs[blockIdx.y].bufA;
    buf += blockIdx.z * zstride;  // sub-transform of a radix-3 plan
    const G gp(logS, logM);
    if constexpr (TL::LC >= 1) {
        const ColPair<TL> pp(logS);
#pragma unroll
        for (int j = 0; j < 8; ++j) cp_async16(sm + pp.sa0 + ColPair<TL>::soff(j), buf + pp.gi0 + j * pp.gstep);
    } else {
#pragma unroll
        for (int k = 0; k < G::PER; ++k) cp_async8(sm + gp.sa0 + G::soff(k), buf + gp.gi0 + k * gp.gstep);
    }
    cp_async_wait_all();
    __syncthreads();
    tile_fwd<TL>(sm, tw.dtw);
    if constexpr (TL::LC >= 1) {
        if (ttab) {
            const ColPair<TL> pp(logS);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                ulonglong2 v = ld2(sm + pp.sa0 + ColPair<TL>::soff(j));
                const ulonglong2 t = ldg2(ttab + pp.ti0 + j * pp.gstep);
                v.x = gl_mul(v.x, t.x);
                v.y = gl_mul(v.y, t.y);
                st2(buf + pp.gi0 + j * pp.gstep, v);
            }
            return;
        }
    }
    if (ttab) {
#pragma unroll
        for (int k = 0; k < G::PER; ++k)
            buf[gp.gi0 + k * gp.gstep] = gl_mul(sm[gp.sa0 + G::soff(k)], __ldg(ttab + gp.ti0 + k * gp.gstep));
    } else {
#pragma unroll
        for (int k = 0; k < G::PER; ++k) {
            u64 x = sm[gp.sa0 + G::soff(k)];
            const u32 e = gp.e0 + G::fk(k) * gp.ec;
            if (e) x = gl_mul(x, uroot(e, tw.u1, tw.u2));
            buf[gp.gi0 + k * gp.gstep] = x;
        }
    }
}

// A not-last inverse pass, in place: inverse inter-pass twiddle on load, then
// the inverse column DFTs. Pass 1 of the inverse leaves N times the
// convolution coefficients (mod p) in natural order; the carry kernel scales.
template <int LOGR, int LOGC>
__global__ void B2M_PASS_BOUNDS((Tile<LOGR, LOGC, MAP_COL>::T))
k_inv_mid(u64* __restrict__ buf, int logS, int logM, RootTables tw, const u64* __restrict__ ttab,
          const ProdJob* __restrict__ jobs, u64 zstride) {
    using TL = Tile<LOGR, LOGC, MAP_COL>;
    using G = ColPass<TL>;
    extern __shared__ u64 sm[];
    if (jobs) buf = jobs[blockIdx.y].bufB;
    buf += blockIdx.z * zstride;
    const G gp(logS, logM);
    // the tile arrives by asynchronous copies while the twiddles load; each
    // thread then multiplies the elements it copied
    bool paired = false;
    if constexpr (TL::LC >= 1) {
        if (ttab) {
            paired = true;
            const ColPair<TL> pp(logS);
#pragma unroll
            for (int j = 0; j < 8; ++j) cp_async16(sm + pp.sa0 + ColPair<TL>::soff(j), buf + pp.gi0 + j * pp.gstep);
            ulonglong2 t[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) t[j] = ldg2(ttab + pp.ti0 + j * pp.gstep);
            cp_async_wait_all();
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                u64* p = sm + pp.sa0 + ColPair<TL>::soff(j);
                ulonglong2 v = ld2(p);
                v.x = gl_mul(v.x, t[j].x);
                v.y = gl_mul(v.y, t[j].y);
                st2(p, v);
            }
        }
    }
    if (!paired) {
#pragma unroll
        for (int k = 0; k < G::PER; ++k) cp_async8(sm + gp.sa0 + G::soff(k), buf + gp.gi0 + k * gp.gstep);
        if (ttab) {
            u64 t[G::PER];
#pragma unroll
            for (int k = 0; k < G::PER; ++k) t[k] = __ldg(ttab + gp.ti0 + k * gp.gstep);
            cp_async_wait_all();
#pragma unroll
            for (int k = 0; k < G::PER; ++k) {
                u64& v = sm[gp.sa0 + G::soff(k)];
                v = gl_mul(v, t[k]);
            }
        } else {
            cp_async_wait_all();
#pragma unroll
            for (int k = 0; k < G::PER; ++k) {
                const u32 e = gp.e0 + G::fk(k) * gp.ec;
                u64& v = sm[gp.sa0 + G::soff(k)];
                if (e) v = gl_mul(v, uroot(0u - e, tw.u1, tw.u2));
            }
        }
    }
    __syncthreads();
    tile_inv<TL>(sm, tw.dtw);
    if constexpr (TL::LC >= 1) {
        const ColPair<TL> pp(logS);
#pragma unroll
        for (int j = 0; j < 8; ++j) st2(buf + pp.gi0 + j * pp.gstep, ld2(sm + pp.sa0 + ColPair<TL>::soff(j)));
    } else {
#pragma unroll
        for (int k = 0; k < G::PER; ++k) buf[gp.gi0 + k * gp.gstep] = sm[gp.sa0 + G::soff(k)];
    }
}

// Last forward pass of operand A (S = 1: each column is a contiguous
// sub-problem, so the CTA's tile is one contiguous range of R*C elements).
template <int LOGR, int LOGC>
__global__ void B2M_PASS_BOUNDS((Tile<LOGR, LOGC, MAP_ROW>::T))
k_fwd_last(u64* __restrict__ buf, RootTables tw, const ProdJob* __restrict__ jobs, u64 zstride) {
    using TL = Tile<LOGR, LOGC, MAP_ROW>;
    using G = RowPass<TL>;
    extern __shared__ u64 sm[];
    if (jobs) buf = jobs[blockIdx.y].bufA;
    buf += blockIdx.z * zstride;
    const G gp;
    u64* base = buf + ((u64)blockIdx.x << (LOGR + LOGC)) + threadIdx.x;
#pragma unroll
    for (int k = 0; k < G::PER; ++k) cp_async8(sm + gp.sa0 + G::soff(k), base + k * TL::T);
    cp_async_wait_all();
    __syncthreads();
    tile_fwd<TL>(sm, tw.dtw);
#pragma unroll
    for (int k = 0; k < G::PER; ++k) base[k * TL::T] = sm[gp.sa0 + G::soff(k)];
}

// Last forward pass of operand B, pointwise product with A's spectrum (same
// positions; times ninv unless ninv is 1, i.e. unless the carry kernel applies
// N^-1), then the first inverse pass -- one tile, one kernel.
// aspec null (no job table): a square, B's spectrum times itself.
template <int LOGR, int LOGC>
__global__ void B2M_PASS_BOUNDS((Tile<LOGR, LOGC, MAP_ROW>::T))
k_fused_last(u64* __restrict__ bbuf, const u64* __restrict__ aspec, u64 ninv, RootTables tw,
             const ProdJob* __restrict__ jobs, u64 zstride) {
    using TL = Tile<LOGR, LOGC, MAP_ROW>;
    using G = RowPass<TL>;
    extern __shared__ u64 sm[];
    if (jobs) {
        bbuf = jobs[blockIdx.y].bufB;
        aspec = jobs[blockIdx.y].bufA;
    }
    const bool square = aspec == nullptr;
    bbuf += blockIdx.z * zstride;
    if (!square) aspec += blockIdx.z * zstride;
    const G gp;
    const u64 off = ((u64)blockIdx.x << (LOGR + LOGC)) + threadIdx.x;
    u64* base = bbuf + off;
    const u64* abase = aspec + off;
#pragma unroll
    for (int k = 0; k < G::PER; ++k) cp_async8(sm + gp.sa0 + G::soff(k), base + k * TL::T);
    cp_async_wait_all();
    __syncthreads();
    tile_fwd<TL, true>(sm, tw.dtw);
    // ninv == 1: the carry kernel applies N^-1 (single products and batches)
    if (square) {
#pragma unroll
        for (int k = 0; k < G::PER; ++k) {
            u64& v = sm[gp.sa0 + G::soff(k)];
            v = gl_mul(v, v);
            if (ninv != 1) v = gl_mul(v, ninv);
        }
    } else {
#pragma unroll
        for (int k = 0; k < G::PER; ++k) {
            u64& v = sm[gp.sa0 + G::soff(k)];
            v = gl_mul(v, __ldg(abase + k * TL::T));
            if (ninv != 1) v = gl_mul(v, ninv);
        }
    }
    __syncthreads();
    tile_inv<TL>(sm, tw.dtw);
#pragma unroll
    for (int k = 0; k < G::PER; ++k) base[k * TL::T] = sm[gp.sa0 + G::soff(k)];
}

// ---------------------------------------------------------------------------
// Whole product in one CTA for N = 2^LOGN <= 2^13: both transforms live in
// shared memory, the carry is a block scan. max(1, N/16) threads; thread t
// owns coefficients [t*G, (t+1)*G), G = min(16, N). A product whose
// schoolbook cost is lower (school_cheaper) is computed that way instead, by
// the same threads in the same shared memory.
// ---------------------------------------------------------------------------
constexpr int small_threads(int logn) { return logn >= 4 ? 1 << (logn - 4) : 1; }
constexpr int small_min_blocks(int logn) {
    return PASS_THREADS_MAX / small_threads(logn) < 32 ? PASS_THREADS_MAX / small_threads(logn) : 32;
}

template <int LOGN>
__global__ void __launch_bounds__(small_threads(LOGN), small_min_blocks(LOGN)) k_mul_small(const u32* __restrict__ a, u64 na, const u32* __restrict__ b,
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
    using TL = Tile<LOGN, 0, MAP_ROW>;
    constexpr int N = 1 << LOGN, RP = TL::RP, G = N < 16 ? N : 16;
    extern __shared__ u64 sm[];
    u64* smA = sm;
    u64* smB = sm + RP;
    CState* s_st = reinterpret_cast<CState*>(sm + 2 * RP);
    __shared__ unsigned long long s_top;
    if (school_cheaper(na, nb, LOGN)) {
        school_cta(a, na, b, nb, out, out_len, reinterpret_cast<unsigned char*>(sm), s_st, &s_top);
        return;
    }
    const u64 nda = 2 * na, ndb = 2 * nb;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        smA[TL::saddr(i, 0)] = digit_of(a, nda, i);
        smB[TL::saddr(i, 0)] = digit_of(b, ndb, i);
    }
    if (threadIdx.x == 0) s_top = 0;
    __syncthreads();
    tile_fwd<TL, true>(smA, tw.dtw);
    tile_fwd<TL, true>(smB, tw.dtw);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int s = TL::saddr(i, 0);
        smB[s] = gl_mul(gl_mul(smB[s], smA[s]), ninv);
    }
    __syncthreads();
    tile_inv<TL>(smB, tw.dtw);

    // Carry: thread t owns G consecutive coefficients.
    const int T = blockDim.x;
    u64 v[G];
#pragma unroll
    for (int i = 0; i < G; ++i) v[i] = smB[TL::saddr((int)threadIdx.x * G + i, 0)];
    u32 lm[G / 2];
    const CState st = group_carry<G>(v, lm);
    u64 cin;
    if (T >= 32) {
        bool has;
        CState agg;
        const CState ex = block_scan_carry(st, &has, &agg, s_st);
        cin = has ? cs_eval(ex, 0) : 0;
    } else {
        s_st[threadIdx.x] = st;
        __syncthreads();
        if (threadIdx.x == 0) {
            // Serial exclusive scan: s_st[t].h becomes the carry into t.
            u64 c = 0;
            for (int t = 0; t < T; ++t) {
                const CState f = s_st[t];
                s_st[t].h = c;
                c = cs_eval(f, c);
            }
        }
        __syncthreads();
        cin = s_st[threadIdx.x].h;
    }
    group_add_carry<G / 2>(lm, cin);
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
