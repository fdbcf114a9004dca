// ntt_engine.cuh -- the register/shared-memory transform engine.
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
// Inside a CTA a pass works on a tile of R rows x C columns. The column DFT
// of length R is split into radix steps of E = 64 (and one leading step of
// 2^(r mod 6)); every thread owns 64 elements in registers for each step,
// the 64-point DFT is fully unrolled with power-of-two (shift) twiddles, and
// the twiddles between steps come from resident tables. Steps exchange data
// in place through a padded shared-memory copy of the tile; the first step
// reads and the last step writes global memory directly.
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
//          inverse roots, unscaled (the caller folds 1/N in elsewhere).
// The root of unity of order 2h is 2^(96/h); all shift amounts are
// compile-time constants once the loops are unrolled.
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

// ---------------------------------------------------------------------------
// Step structure of a length-2^LOGR column DFT.
// ---------------------------------------------------------------------------
constexpr int nsteps_of(int logr) { return logr <= 6 ? 1 : logr / 6 + ((logr % 6) ? 1 : 0); }
constexpr int step_loge(int logr, int s) {
    return logr <= 6 ? logr : (((logr % 6) != 0 && s == 0) ? (logr % 6) : 6);
}
constexpr int step_logl(int logr, int s) {
    int l = logr;
    for (int i = 0; i < s; ++i) l -= step_loge(logr, i);
    return l;
}

enum { MAP_COL = 0, MAP_ROW = 1 };

// Tile geometry. MAP_COL: consecutive instances walk columns first (used when
// a row segment of C columns is contiguous in global memory, i.e. S >= C).
// MAP_ROW: consecutive instances walk rows first (S == 1: every column is a
// contiguous sub-problem). Shared memory is padded by one row every 64 rows
// so that the 64-row blocks of the last step do not collide on banks.
template <int LOGR, int MAP>
struct Tile {
    static constexpr int R = 1 << LOGR;
    static constexpr int EPT = LOGR < 6 ? R : 64;   // elements per thread
    static constexpr int RP = R + (R >> 6);          // padded rows
    int logC;

    __device__ __forceinline__ int cols() const { return 1 << logC; }
    __device__ __forceinline__ int nthreads() const { return (R << logC) / EPT; }
    __device__ __forceinline__ int smem_elems() const { return RP << logC; }

    template <int LOGE, int LOGL>
    __device__ __forceinline__ void decode(int q, int& col, int& blk, int& j) const {
        constexpr int LOGJ = LOGL - LOGE;
        if (MAP == MAP_COL) {
            col = q & ((1 << logC) - 1);
            int r = q >> logC;
            j = r & ((1 << LOGJ) - 1);
            blk = r >> LOGJ;
        } else {
            j = q & ((1 << LOGJ) - 1);
            int r = q >> LOGJ;
            constexpr int LOGNB = LOGR - LOGL;
            blk = r & ((1 << LOGNB) - 1);
            col = r >> LOGNB;
        }
    }
    __device__ __forceinline__ int saddr(int row, int col) const {
        int pr = row + (row >> 6);
        return MAP == MAP_COL ? (pr << logC) + col : col * RP + pr;
    }
};

// Load phase of one radix step: v[u*E + t] = src(row, col, slot) for the
// thread's 64/E instances (slot = u*E + t is the register index).
template <int LOGR, int MAP, int LOGE, int LOGL, class Src>
__device__ __forceinline__ void step_load(u64* v, const Tile<LOGR, MAP>& tl, Src src) {
    constexpr int E = 1 << LOGE, EPT = Tile<LOGR, MAP>::EPT, NI = EPT / E;
    constexpr int JW = 1 << (LOGL - LOGE);
    const int T = tl.nthreads();
#pragma unroll
    for (int u = 0; u < NI; ++u) {
        int col, blk, j;
        tl.template decode<LOGE, LOGL>((int)threadIdx.x + u * T, col, blk, j);
        const int row0 = (blk << LOGL) + j;
#pragma unroll
        for (int t = 0; t < E; ++t) v[u * E + t] = src(row0 + t * JW, col, u * E + t);
    }
}

// Store phase: dst(row, col, slot, value) for register slot u*E + i, which
// holds the element belonging at row blk*L + j + i*(L/E).
template <int LOGR, int MAP, int LOGE, int LOGL, class Dst>
__device__ __forceinline__ void step_store(const u64* v, const Tile<LOGR, MAP>& tl, Dst dst) {
    constexpr int E = 1 << LOGE, EPT = Tile<LOGR, MAP>::EPT, NI = EPT / E;
    constexpr int JW = 1 << (LOGL - LOGE);
    const int T = tl.nthreads();
#pragma unroll
    for (int u = 0; u < NI; ++u) {
        int col, blk, j;
        tl.template decode<LOGE, LOGL>((int)threadIdx.x + u * T, col, blk, j);
        const int row0 = (blk << LOGL) + j;
#pragma unroll
        for (int i = 0; i < E; ++i) dst(row0 + i * JW, col, u * E + i, v[u * E + i]);
    }
}

// Compute phase, forward: E-point DFT, then register i (frequency
// k = bitrev(i)) is multiplied by w_L^(j*k) from the dense root table
// dtw[L + e] = w_L^e.
template <int LOGR, int MAP, int LOGE, int LOGL>
__device__ __forceinline__ void step_fwd(u64* v, const Tile<LOGR, MAP>& tl, const u64* __restrict__ dtw) {
    constexpr int E = 1 << LOGE, EPT = Tile<LOGR, MAP>::EPT, NI = EPT / E;
    constexpr int L = 1 << LOGL;
    const int T = tl.nthreads();
#pragma unroll
    for (int u = 0; u < NI; ++u) {
        dft_fwd<E>(v + u * E);
        if (L > E) {
            int col, blk, j;
            tl.template decode<LOGE, LOGL>((int)threadIdx.x + u * T, col, blk, j);
#pragma unroll
            for (int i = 1; i < E; ++i) {
                const int k = brev_c(i, LOGE);
                const int e = (j * k) & (L - 1);
                v[u * E + i] = gl_mul(v[u * E + i], __ldg(dtw + L + e));
            }
        }
    }
}

// Compute phase, inverse: multiply register i by w_L^(-j*k), then the
// inverse E-point DFT (bit-reversed in, natural out).
template <int LOGR, int MAP, int LOGE, int LOGL>
__device__ __forceinline__ void step_inv(u64* v, const Tile<LOGR, MAP>& tl, const u64* __restrict__ dtw) {
    constexpr int E = 1 << LOGE, EPT = Tile<LOGR, MAP>::EPT, NI = EPT / E;
    constexpr int L = 1 << LOGL;
    const int T = tl.nthreads();
#pragma unroll
    for (int u = 0; u < NI; ++u) {
        if (L > E) {
            int col, blk, j;
            tl.template decode<LOGE, LOGL>((int)threadIdx.x + u * T, col, blk, j);
#pragma unroll
            for (int i = 1; i < E; ++i) {
                const int k = brev_c(i, LOGE);
                const int e = (L - ((j * k) & (L - 1))) & (L - 1);
                v[u * E + i] = gl_mul(v[u * E + i], __ldg(dtw + L + e));
            }
        }
        dft_inv<E>(v + u * E);
    }
}

// ---------------------------------------------------------------------------
// Whole column DFTs over the tile.
//
// fwd_columns: step 0 loads through `src`, intermediate steps exchange via
// shared memory `sm` (in place), the last step stores through `dst`.
// inv_columns: the mirror (last forward step first).
// `sm` may be nullptr when the DFT has a single step.
// ---------------------------------------------------------------------------
template <int LOGR, int MAP, int S, class Src, class Dst>
__device__ __forceinline__ void fwd_from(u64* v, const Tile<LOGR, MAP>& tl, u64* sm,
                                         const u64* dtw, Src src, Dst dst) {
    constexpr int NS = nsteps_of(LOGR);
    constexpr int LOGE = step_loge(LOGR, S), LOGL = step_logl(LOGR, S);
    if constexpr (S == 0) {
        step_load<LOGR, MAP, LOGE, LOGL>(v, tl, src);
    } else {
        step_load<LOGR, MAP, LOGE, LOGL>(v, tl, [&](int row, int col, int) { return sm[tl.saddr(row, col)]; });
    }
    step_fwd<LOGR, MAP, LOGE, LOGL>(v, tl, dtw);
    if constexpr (S + 1 == NS) {
        if constexpr (NS == 1) __syncthreads();  // stores may land where others still load
        step_store<LOGR, MAP, LOGE, LOGL>(v, tl, dst);
    } else {
        step_store<LOGR, MAP, LOGE, LOGL>(v, tl, [&](int row, int col, int, u64 x) { sm[tl.saddr(row, col)] = x; });
        __syncthreads();
        fwd_from<LOGR, MAP, S + 1>(v, tl, sm, dtw, src, dst);
    }
}

template <int LOGR, int MAP, class Src, class Dst>
__device__ __forceinline__ void fwd_columns(u64* v, const Tile<LOGR, MAP>& tl, u64* sm,
                                            const u64* dtw, Src src, Dst dst) {
    fwd_from<LOGR, MAP, 0>(v, tl, sm, dtw, src, dst);
}

// Inverse steps run S = NS-1 down to 0.
template <int LOGR, int MAP, int S, class Src, class Dst>
__device__ __forceinline__ void inv_from(u64* v, const Tile<LOGR, MAP>& tl, u64* sm,
                                         const u64* dtw, Src src, Dst dst) {
    constexpr int NS = nsteps_of(LOGR);
    constexpr int LOGE = step_loge(LOGR, S), LOGL = step_logl(LOGR, S);
    if constexpr (S == NS - 1) {
        step_load<LOGR, MAP, LOGE, LOGL>(v, tl, src);
    } else {
        step_load<LOGR, MAP, LOGE, LOGL>(v, tl, [&](int row, int col, int) { return sm[tl.saddr(row, col)]; });
    }
    step_inv<LOGR, MAP, LOGE, LOGL>(v, tl, dtw);
    if constexpr (S == 0) {
        if constexpr (NS == 1) __syncthreads();
        step_store<LOGR, MAP, LOGE, LOGL>(v, tl, dst);
    } else {
        step_store<LOGR, MAP, LOGE, LOGL>(v, tl, [&](int row, int col, int, u64 x) { sm[tl.saddr(row, col)] = x; });
        __syncthreads();
        inv_from<LOGR, MAP, S - 1>(v, tl, sm, dtw, src, dst);
    }
}

template <int LOGR, int MAP, class Src, class Dst>
__device__ __forceinline__ void inv_columns(u64* v, const Tile<LOGR, MAP>& tl, u64* sm,
                                            const u64* dtw, Src src, Dst dst) {
    inv_from<LOGR, MAP, nsteps_of(LOGR) - 1>(v, tl, sm, dtw, src, dst);
}

// w_{2^logM}^e from the two-level universal tables of RHO powers:
// u1[x & 0xFFFF] * u2[x >> 16] with x = e * 2^(32 - logM) (mod 2^32).
__device__ __forceinline__ u64 uroot(u32 x, const u64* __restrict__ u1, const u64* __restrict__ u2) {
    return gl_mul(__ldg(u1 + (x & 0xFFFFu)), __ldg(u2 + (x >> 16)));
}

}  // namespace b2m
