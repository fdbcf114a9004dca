// ntt_engine.cuh -- the shared-memory tile transform engine.
//
// A length-N transform (N = 2^L) is split into passes of radix R_k = 2^r_k.
// Pass k sees the array as B_k independent sub-problems of M_k = R_k * S_k
// contiguous elements, each an R_k x S_k row-major matrix (S_k = product of
// the later radices). Forward pass k runs, for every column, a length-R_k
// decimation-in-frequency DFT down the column, then multiplies element
// (storage row s, column c) by w_{M_k}^(bitrev(s) * c) (the "inter-pass"
// twiddle). The inverse pass undoes exactly that, in reverse pass order,
// with decimation-in-time. Forward output is in bit-reversed order overall and
// the inverse consumes it as such, so no permutation pass exists anywhere.
//
// Inside a CTA a pass holds a tile of R rows x C columns in shared memory.
// The length-R column DFT is R = 2^A * 8^q: one leading radix-2^A step, then
// radix-8 levels. Consecutive pairs of radix-8 levels form a radix-64 group
// whose inner twiddles are powers of 8 (= 2^3, the 64th root of unity in the
// chosen root chain), so they are shifts, not multiplies; one table twiddle
// per element follows each group. Every level is a rolled loop of 8-element
// register DFTs (compile-time shift roots), so the code stays small enough
// for the instruction cache and registers stay low enough for full CTAs.
//
// Reference counterpart: the per-stage radix-2 launches of src/ntt_cuda.cu
// (k_bit_reverse :75-84, k_butterfly :99-114, k_scale :124-128), which this
// replaces; the algebra is the same DFT over GF(p) (src/ntt_cpu.cpp:64-104).
#pragma once
#include "gl.cuh"

namespace b2m {

// ---------------------------------------------------------------------------
// Register DFTs on E = 2^e consecutive registers.
// dft_fwd: natural-order input, bit-reversed output (decimation in frequency).
// dft_inv: bit-reversed input, natural-order output (decimation in time),
//          inverse roots, unscaled (1/N is folded into the pointwise step).
// The root of unity of order 2h is 2^(96/h).
// ---------------------------------------------------------------------------
template <int E>
GL_FN void dft_fwd(u64* x) {
#pragma unroll
    for (int h = E / 2; h >= 1; h >>= 1) {
#pragma unroll
        for (int b = 0; b < E; b += 2 * h) {
#pragma unroll
            for (int j = 0; j < h; ++j) {
                u64 a = x[b + j], c = x[b + j + h];
                x[b + j] = gl_add(a, c);
                x[b + j + h] = gl_shl(gl_sub(a, c), (96 * j) / h);
            }
        }
    }
}

template <int E>
GL_FN void dft_inv(u64* x) {
#pragma unroll
    for (int h = 1; h < E; h <<= 1) {
#pragma unroll
        for (int b = 0; b < E; b += 2 * h) {
#pragma unroll
            for (int j = 0; j < h; ++j) {
                u64 a = x[b + j], c = x[b + j + h];
                if (j == 0) {
                    x[b + j] = gl_add(a, c);
                    x[b + j + h] = gl_sub(a, c);
                } else {
                    // c * w^-j with w^-j = 2^(192 - 96j/h) = -2^(96 - 96j/h)
                    u64 t = gl_shl(c, 96 - (96 * j) / h);
                    x[b + j] = gl_sub(a, t);
                    x[b + j + h] = gl_add(a, t);
                }
            }
        }
    }
}

constexpr int brev_c(int v, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1) << (bits - 1 - i);
    return r;
}

enum { MAP_COL = 0, MAP_ROW = 1 };

// Tile geometry. MAP_COL: columns are the fastest-varying index of task
// enumeration and of the [R][C] shared layout (used when a row segment of C
// columns is contiguous in global memory, S >= C). MAP_ROW: rows fastest and
// a [C][R] layout (S == 1: every column is a contiguous sub-problem).
// Shared memory is padded by one row every 64 rows against bank conflicts.
template <int LOGR, int MAP>
struct Tile {
    static constexpr int R = 1 << LOGR;
    static constexpr int RP = R + (R >> 6);
    int logC;

    __device__ __forceinline__ int saddr(int row, int col) const {
        const int pr = row + (row >> 6);
        return MAP == MAP_COL ? (pr << logC) + col : col * RP + pr;
    }
    // Address step between rows S apart inside one task. Every task's rows
    // are either S >= 64 apart with S a multiple of 64, or all inside one
    // 64-row block, so the padded address is linear: base + m * step.
    template <int S>
    __device__ __forceinline__ int step() const {
        constexpr int PS = S >= 64 ? S + S / 64 : S;
        return MAP == MAP_COL ? (PS << logC) : PS;
    }
    // Instance q of a step with JW positions per block -> (col, blk, j).
    __device__ __forceinline__ void decode(int q, int logjw, int& col, int& blk, int& j) const {
        if (MAP == MAP_COL) {
            col = q & ((1 << logC) - 1);
            const int r = q >> logC;
            j = r & ((1 << logjw) - 1);
            blk = r >> logjw;
        } else {
            j = q & ((1 << logjw) - 1);
            const int r = q >> logjw;
            const int lognb = LOGR - 6 - logjw;  // only used by radix-64 groups
            blk = r & ((1 << lognb) - 1);
            col = r >> lognb;
        }
    }
};

// Number of radix-8 levels and the leading radix exponent of a length-2^LOGR DFT.
template <int LOGR>
struct Steps {
    static constexpr int A = LOGR % 3;      // leading radix 2^A (0: none)
    static constexpr int Q = LOGR / 3;      // radix-8 levels
    static constexpr int G = Q / 2;         // radix-64 groups
    static constexpr bool LONE = (Q & 1);   // trailing lone radix-8 (L = 8)
};

// ---------------------------------------------------------------------------
// Leading radix-2^A step over the whole column (L = R): task (col, j),
// j in [0, R/2^A); elements at rows j + m*(R/2^A). Forward: DFT then
// w_R^(j*k); inverse: w_R^(-j*k) then inverse DFT.
// ---------------------------------------------------------------------------
template <int LOGR, int MAP, int A, bool INV>
__device__ __forceinline__ void lead_step(u64* sm, const Tile<LOGR, MAP>& tl, const u64* __restrict__ dtw) {
    constexpr int E = 1 << A, R = 1 << LOGR, LOGJ = LOGR - A, JW = R >> A;
    const int tasks = JW << tl.logC;
    for (int q = threadIdx.x; q < tasks; q += blockDim.x) {
        int col, j;
        if (MAP == MAP_COL) {
            col = q & ((1 << tl.logC) - 1);
            j = q >> tl.logC;
        } else {
            j = q & (JW - 1);
            col = q >> LOGJ;
        }
        u64 x[E];
        u64* ptr = sm + tl.saddr(j, col);
        const int st = tl.template step<JW>();
#pragma unroll
        for (int m = 0; m < E; ++m) x[m] = ptr[m * st];
        if (!INV) {
            dft_fwd<E>(x);
#pragma unroll
            for (int i = 1; i < E; ++i) x[i] = gl_mul(x[i], __ldg(dtw + R + ((j * brev_c(i, A)) & (R - 1))));
        } else {
#pragma unroll
            for (int i = 1; i < E; ++i)
                x[i] = gl_mul(x[i], __ldg(dtw + R + ((R - ((j * brev_c(i, A)) & (R - 1))) & (R - 1))));
            dft_inv<E>(x);
        }
#pragma unroll
        for (int m = 0; m < E; ++m) ptr[m * st] = x[m];
    }
}

// ---------------------------------------------------------------------------
// Radix-64 group on blocks of L = 2^LOGL rows: instance (col, blk, j) with
// j in [0, L/64) owns rows blk*L + j + u*(L/64), u in [0, 64), u = u1 + 8*u2.
//  level 1: for each u1, DFT-8 over u2; slot i1 (k1 = brev3(i1)) times
//           8^(u1*k1) = 2^(3*u1*k1) -- a shift; stored at u = u1 + 8*i1.
//  level 2: for each i1, DFT-8 over u1; slot i2 times w_L^(j*k),
//           k = k1 + 8*k2 (skipped when L == 64); stored at u = 8*i1 + i2,
//           i.e. bitrev6(k).
// Task order puts the level index (u1 or i1) outermost so it is uniform
// across a warp whenever the tile has >= 32 instances.
// ---------------------------------------------------------------------------
template <int LOGR, int MAP, int LOGL, bool INV>
__device__ __forceinline__ void group64(u64* sm, const Tile<LOGR, MAP>& tl, const u64* __restrict__ dtw) {
    constexpr int L = 1 << LOGL, LOGJ = LOGL - 6, JW = 1 << LOGJ;
    const int logni = LOGR - 6 + tl.logC;  // instances = C * R / 64
    const int ni = 1 << logni;
    const int tasks = ni << 3;
    // ---- level 1 (forward) / level 1 inverse (second, for INV) ----
    auto level1 = [&]() {
        for (int q = threadIdx.x; q < tasks; q += blockDim.x) {
            const int u1 = q >> logni;
            int col, blk, j;
            tl.decode(q & (ni - 1), LOGJ, col, blk, j);
            u64* ptr = sm + tl.saddr(blk * L + j + u1 * JW, col);
            const int st = tl.template step<8 * JW>();
            u64 x[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) x[m] = ptr[m * st];
            if (!INV) {
                dft_fwd<8>(x);
#pragma unroll
                for (int i = 1; i < 8; ++i) x[i] = gl_shl(x[i], 3 * u1 * brev_c(i, 3));
            } else {
#pragma unroll
                for (int i = 1; i < 8; ++i) {
                    const int s = 3 * u1 * brev_c(i, 3);
                    x[i] = s ? gl_shl(x[i], 192 - s) : x[i];
                }
                dft_inv<8>(x);
            }
#pragma unroll
            for (int m = 0; m < 8; ++m) ptr[m * st] = x[m];
        }
    };
    auto level2 = [&]() {
        for (int q = threadIdx.x; q < tasks; q += blockDim.x) {
            const int i1 = q >> logni;
            int col, blk, j;
            tl.decode(q & (ni - 1), LOGJ, col, blk, j);
            u64* ptr = sm + tl.saddr(blk * L + j + i1 * 8 * JW, col);
            const int st = tl.template step<JW>();
            const int k1 = brev_c(i1, 3);
            u64 x[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) x[m] = ptr[m * st];
            if (!INV) {
                dft_fwd<8>(x);
                if (L > 64) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int k = k1 + 8 * brev_c(i, 3);
                        x[i] = gl_mul(x[i], __ldg(dtw + L + ((j * k) & (L - 1))));
                    }
                }
            } else {
                if (L > 64) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int k = k1 + 8 * brev_c(i, 3);
                        x[i] = gl_mul(x[i], __ldg(dtw + L + ((L - ((j * k) & (L - 1))) & (L - 1))));
                    }
                }
                dft_inv<8>(x);
            }
#pragma unroll
            for (int m = 0; m < 8; ++m) ptr[m * st] = x[m];
        }
    };
    if (!INV) {
        level1();
        __syncthreads();
        level2();
    } else {
        level2();
        __syncthreads();
        level1();
    }
}

// Trailing lone radix-8 level (L = 8, no twiddle): task (col, blk).
template <int LOGR, int MAP, bool INV>
__device__ __forceinline__ void lone8(u64* sm, const Tile<LOGR, MAP>& tl) {
    constexpr int LOGNB = LOGR - 3;
    const int tasks = 1 << (LOGNB + tl.logC);
    for (int q = threadIdx.x; q < tasks; q += blockDim.x) {
        int col, blk;
        if (MAP == MAP_COL) {
            col = q & ((1 << tl.logC) - 1);
            blk = q >> tl.logC;
        } else {
            blk = q & ((1 << LOGNB) - 1);
            col = q >> LOGNB;
        }
        u64* ptr = sm + tl.saddr(blk * 8, col);
        const int st = tl.template step<1>();
        u64 x[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) x[m] = ptr[m * st];
        if (!INV) dft_fwd<8>(x);
        else dft_inv<8>(x);
#pragma unroll
        for (int m = 0; m < 8; ++m) ptr[m * st] = x[m];
    }
}

// Radix-64 groups from block size 2^LOGL down, G groups.
template <int LOGR, int MAP, int LOGL, int G, bool INV>
__device__ __forceinline__ void groups_fwd(u64* sm, const Tile<LOGR, MAP>& tl, const u64* dtw) {
    if constexpr (G > 0) {
        group64<LOGR, MAP, LOGL, false>(sm, tl, dtw);
        __syncthreads();
        groups_fwd<LOGR, MAP, LOGL - 6, G - 1, false>(sm, tl, dtw);
    }
}
template <int LOGR, int MAP, int LOGL, int G>
__device__ __forceinline__ void groups_inv(u64* sm, const Tile<LOGR, MAP>& tl, const u64* dtw) {
    // inverse order: smallest block first
    if constexpr (G > 0) {
        groups_inv<LOGR, MAP, LOGL - 6, G - 1>(sm, tl, dtw);
        group64<LOGR, MAP, LOGL, true>(sm, tl, dtw);
        __syncthreads();
    }
}

// Whole column DFTs of the tile held in shared memory (callers synchronise
// before; the functions end with the tile synchronised).
template <int LOGR, int MAP>
__device__ __forceinline__ void tile_fwd(u64* sm, const Tile<LOGR, MAP>& tl, const u64* dtw) {
    using S = Steps<LOGR>;
    if constexpr (S::A > 0) {
        lead_step<LOGR, MAP, S::A, false>(sm, tl, dtw);
        __syncthreads();
    }
    groups_fwd<LOGR, MAP, LOGR - S::A, S::G, false>(sm, tl, dtw);
    if constexpr (S::LONE) {
        lone8<LOGR, MAP, false>(sm, tl);
        __syncthreads();
    }
}

template <int LOGR, int MAP>
__device__ __forceinline__ void tile_inv(u64* sm, const Tile<LOGR, MAP>& tl, const u64* dtw) {
    using S = Steps<LOGR>;
    if constexpr (S::LONE) {
        lone8<LOGR, MAP, true>(sm, tl);
        __syncthreads();
    }
    groups_inv<LOGR, MAP, LOGR - S::A, S::G>(sm, tl, dtw);
    if constexpr (S::A > 0) {
        lead_step<LOGR, MAP, S::A, true>(sm, tl, dtw);
        __syncthreads();
    }
}

// w_{2^logM}^e from the two-level universal tables of RHO powers:
// u1[x & 0xFFFF] * u2[x >> 16] with x = e * 2^(32 - logM) (mod 2^32).
__device__ __forceinline__ u64 uroot(u32 x, const u64* __restrict__ u1, const u64* __restrict__ u2) {
    return gl_mul(__ldg(u1 + (x & 0xFFFFu)), __ldg(u2 + (x >> 16)));
}

}  // namespace b2m
