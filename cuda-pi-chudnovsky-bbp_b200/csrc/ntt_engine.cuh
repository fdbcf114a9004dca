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
//          inverse roots, unscaled (1/N is applied by the carry kernel, or by
//          the pointwise step of the one-CTA product).
// The root of unity of order 2h is 2^(96/h).
// ---------------------------------------------------------------------------
// ZH: the upper half x[E/2 .. E) is known to be zero (the first level of the
// first forward pass, whose input holds at most N/2 digits): the first level
// is then x[j + E/2] = x[j] * w^j, no additions.
template <int E, bool ZH = false>
GL_FN void dft_fwd(u64* x) {
    if constexpr (ZH) {
#pragma unroll
        for (int j = 1; j < E / 2; ++j) x[j + E / 2] = gl_shl(x[j], (96 * j) / (E / 2));
        x[E / 2] = x[0];
    }
#pragma unroll
    for (int h = ZH ? E / 4 : E / 2; h >= 1; h >>= 1) {
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

// Two adjacent u64 (16-byte aligned) in one access.
__device__ __forceinline__ ulonglong2 ld2(const u64* p) { return *reinterpret_cast<const ulonglong2*>(p); }
__device__ __forceinline__ void st2(u64* p, ulonglong2 v) { *reinterpret_cast<ulonglong2*>(p) = v; }

// Tile geometry, all compile-time: R = 2^LOGR rows by C = 2^LOGC columns,
// T = max(1, R*C/16) threads, so every radix-8 level is two 8-point tasks per
// thread and every load or store loop is 16 elements per thread.
// MAP_COL: columns are the fastest-varying index of task enumeration and of
// the [R][C] shared layout (used when a row segment of C columns is contiguous
// in global memory, S >= C). MAP_ROW: rows fastest and a [C][R] layout (S == 1:
// every column is a contiguous sub-problem). Shared memory is padded by one row
// every 64 rows against bank conflicts.
template <int LOGR, int LOGC, int MAP>
struct Tile {
    static constexpr int LR = LOGR, LC = LOGC, MAPK = MAP;
    static constexpr int R = 1 << LOGR;
    static constexpr int C = 1 << LOGC;
    static constexpr int RP = R + (R >> 6);
    static constexpr int LOGT = LOGR + LOGC >= 4 ? LOGR + LOGC - 4 : 0;
    static constexpr int T = 1 << LOGT;
    // Column-mapped tiles of two or more columns run their inverse 8-point
    // tasks in pairs of adjacent columns: the two tasks' elements are
    // adjacent in shared memory (16-byte aligned: even column, rows of
    // C >= 2 elements), so each pair of elements is one 16-byte access, and
    // a twiddle that depends only on the row serves both columns. Forward
    // tasks stay single: with their eight specialised level-1 bodies the
    // paired form measured slower (more code, register spills).
    static constexpr bool PAIR = MAP == MAP_COL && LOGC >= 1 && LOGR + LOGC >= 5;

    static constexpr int pad(int row) { return row + (row >> 6); }
    __device__ __forceinline__ static int saddr(int row, int col) {
        return MAP == MAP_COL ? (pad(row) << LOGC) + col : col * RP + pad(row);
    }
    // Address step between rows S apart inside one task. Every task's rows
    // are either S >= 64 apart with S a multiple of 64, or all inside one
    // 64-row block, so the padded address is linear: base + m * step.
    template <int S>
    static constexpr int step() {
        return MAP == MAP_COL ? ((S >= 64 ? S + S / 64 : S) << LOGC) : (S >= 64 ? S + S / 64 : S);
    }
    // Instance q of a step with 2^LOGJW positions per block -> (col, blk, j).
    template <int LOGJW>
    __device__ __forceinline__ static void decode(int q, int& col, int& blk, int& j) {
        if (MAP == MAP_COL) {
            col = q & (C - 1);
            const int r = q >> LOGC;
            j = r & ((1 << LOGJW) - 1);
            blk = r >> LOGJW;
        } else {
            constexpr int LOGNB = LOGR - 6 - LOGJW;  // only used by radix-64 groups
            j = q & ((1 << LOGJW) - 1);
            const int r = q >> LOGJW;
            blk = r & ((1 << LOGNB) - 1);
            col = r >> LOGNB;
        }
    }
};

// Runs f(q) for the task indices q of this thread: TASKS tasks over T threads
// (both powers of two), a rolled loop with a compile-time trip count.
template <int TASKS, int T, typename F>
__device__ __forceinline__ void for_tasks(F&& f) {
    if constexpr (TASKS >= T) {
#pragma unroll
        for (int k = 0; k < TASKS / T; ++k) f((int)threadIdx.x + k * T);
    } else {
        if ((int)threadIdx.x < TASKS) f((int)threadIdx.x);
    }
}

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
template <class TL, int A, bool INV, bool ZH = false>
__device__ __forceinline__ void lead_step(u64* sm, const u64* __restrict__ dtw) {
    constexpr int E = 1 << A, R = TL::R, LOGJ = TL::LR - A, JW = R >> A;
    if constexpr (TL::PAIR && INV) {
        for_tasks<(JW << (TL::LC - 1)), TL::T>([&](int p) {
            const int col = (p << 1) & (TL::C - 1), j = (p << 1) >> TL::LC;
            u64 x[E], y[E];
            u64* ptr = sm + TL::saddr(j, col);
            constexpr int st = TL::template step<JW>();
#pragma unroll
            for (int m = 0; m < (ZH ? E / 2 : E); ++m) {
                const ulonglong2 v = ld2(ptr + m * st);
                x[m] = v.x;
                y[m] = v.y;
            }
            if (!INV) {
                dft_fwd<E, ZH>(x);
                dft_fwd<E, ZH>(y);
#pragma unroll
                for (int i = 1; i < E; ++i) {
                    const u64 w = __ldg(dtw + R + ((j * brev_c(i, A)) & (R - 1)));
                    x[i] = gl_mul(x[i], w);
                    y[i] = gl_mul(y[i], w);
                }
            } else {
#pragma unroll
                for (int i = 1; i < E; ++i) {
                    const u64 w = __ldg(dtw + R + ((R - ((j * brev_c(i, A)) & (R - 1))) & (R - 1)));
                    x[i] = gl_mul(x[i], w);
                    y[i] = gl_mul(y[i], w);
                }
                dft_inv<E>(x);
                dft_inv<E>(y);
            }
#pragma unroll
            for (int m = 0; m < E; ++m) st2(ptr + m * st, make_ulonglong2(x[m], y[m]));
        });
        return;
    }
    for_tasks<(JW << TL::LC), TL::T>([&](int q) {
        int col, j;
        if (TL::MAPK == MAP_COL) {
            col = q & (TL::C - 1);
            j = q >> TL::LC;
        } else {
            j = q & (JW - 1);
            col = q >> LOGJ;
        }
        u64 x[E];
        u64* ptr = sm + TL::saddr(j, col);
        constexpr int st = TL::template step<JW>();
#pragma unroll
        for (int m = 0; m < (ZH ? E / 2 : E); ++m) x[m] = ptr[m * st];
        if (!INV) {
            dft_fwd<E, ZH>(x);
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
    });
}

// Level-1 twiddles of a radix-64 group, slot i (k1 = brev3(i)) times
// 8^(u1 * k1) = 2^(3 u1 k1) (inverse: its inverse), with u1 a compile-time
// constant so every shift folds to its fixed word offset.
template <int U1, bool INV>
__device__ __forceinline__ void level1_twiddle(u64* x) {
#pragma unroll
    for (int i = 1; i < 8; ++i) {
        const int s = 3 * U1 * brev_c(i, 3);
        x[i] = gl_shl(x[i], INV ? (s ? 192 - s : 0) : s);
    }
}

// The same for a warp-uniform run-time u1 in [0, 8), two ways:
//  RT = false: one uniform branch to the compile-time form (eight specialised
//    bodies per direction; fastest where a kernel holds one direction);
//  RT = true: shift amounts 3 * u1 * k1 (mod 192) formed at run time and one
//    out-of-line run-time shift routine, so the kernel carries one copy of the
//    code -- the fused pass (both directions in one kernel) was bound by
//    instruction fetch with the specialised bodies, and the inverse passes
//    measured faster this way too.
template <bool INV, bool RT>
__device__ __forceinline__ void level1_twiddle(u64* x, int u1) {
    if constexpr (RT) {
        if (u1 == 0) return;
#pragma unroll
        for (int i = 1; i < 8; ++i) {
            const u32 s = (u32)(3 * brev_c(i, 3)) * (u32)u1;  // < 192
            x[i] = gl_shl_rt(x[i], INV ? 192u - s : s);
        }
    } else {
        switch (u1) {
            case 0: break;
            case 1: level1_twiddle<1, INV>(x); break;
            case 2: level1_twiddle<2, INV>(x); break;
            case 3: level1_twiddle<3, INV>(x); break;
            case 4: level1_twiddle<4, INV>(x); break;
            case 5: level1_twiddle<5, INV>(x); break;
            case 6: level1_twiddle<6, INV>(x); break;
            default: level1_twiddle<7, INV>(x); break;
        }
    }
}

// Both columns of a paired task: one run-time shift call per element pair.
template <bool INV, bool RT>
__device__ __forceinline__ void level1_twiddle2(u64* x, u64* y, int u1) {
    if constexpr (RT) {
        if (u1 == 0) return;
#pragma unroll
        for (int i = 1; i < 8; ++i) {
            const u32 s = (u32)(3 * brev_c(i, 3)) * (u32)u1;  // < 192
            const ulonglong2 r = gl_shl_rt2(x[i], y[i], INV ? 192u - s : s);
            x[i] = r.x;
            y[i] = r.y;
        }
    } else {
        level1_twiddle<INV, RT>(x, u1);
        level1_twiddle<INV, RT>(y, u1);
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
template <class TL, int LOGL, bool INV, bool RT, bool ZH = false>
__device__ __forceinline__ void group64(u64* sm, const u64* __restrict__ dtw) {
    constexpr int L = 1 << LOGL, LOGJ = LOGL - 6, JW = 1 << LOGJ;
    constexpr int LOGNI = TL::LR - 6 + TL::LC;  // instances = C * R / 64
    constexpr int NI = 1 << LOGNI;
    constexpr int TASKS = NI << 3;
    auto level1 = [&]() {
        if constexpr (TL::PAIR && INV) {
            for_tasks<TASKS / 2, TL::T>([&](int p) {
                const int u1 = p >> (LOGNI - 1);
                int col, blk, j;
                TL::template decode<LOGJ>((p & (NI / 2 - 1)) << 1, col, blk, j);
                u64* ptr = sm + TL::saddr(blk * L + j + u1 * JW, col);
                constexpr int st = TL::template step<8 * JW>();
                u64 x[8], y[8];
#pragma unroll
                for (int m = 0; m < (ZH ? 4 : 8); ++m) {
                    const ulonglong2 v = ld2(ptr + m * st);
                    x[m] = v.x;
                    y[m] = v.y;
                }
                if (!INV) {
                    dft_fwd<8, ZH>(x);
                    dft_fwd<8, ZH>(y);
                    level1_twiddle2<false, RT>(x, y, u1);
                } else {
                    level1_twiddle2<true, RT>(x, y, u1);
                    dft_inv<8>(x);
                    dft_inv<8>(y);
                }
#pragma unroll
                for (int m = 0; m < 8; ++m) st2(ptr + m * st, make_ulonglong2(x[m], y[m]));
            });
            return;
        }
        if constexpr (RT && TL::LC >= 1) {
            // run-time shifts: a thread's two tasks are instances inst and
            // inst + NI/2 of the same u1, so one call shifts both (tiles of
            // one column, the single-CTA products among them, keep single
            // tasks: two live tasks there spill)
            for_tasks<TASKS / 2, TL::T>([&](int p) {
                const int u1 = p >> (LOGNI - 1);
                const int inst = p & (NI / 2 - 1);
                int col, blk, j;
                TL::template decode<LOGJ>(inst, col, blk, j);
                u64* ptr0 = sm + TL::saddr(blk * L + j + u1 * JW, col);
                TL::template decode<LOGJ>(inst + NI / 2, col, blk, j);
                u64* ptr1 = sm + TL::saddr(blk * L + j + u1 * JW, col);
                constexpr int st = TL::template step<8 * JW>();
                u64 x[8], y[8];
#pragma unroll
                for (int m = 0; m < (ZH ? 4 : 8); ++m) {
                    x[m] = ptr0[m * st];
                    y[m] = ptr1[m * st];
                }
                if (!INV) {
                    dft_fwd<8, ZH>(x);
                    dft_fwd<8, ZH>(y);
                    level1_twiddle2<false, true>(x, y, u1);
                } else {
                    level1_twiddle2<true, true>(x, y, u1);
                    dft_inv<8>(x);
                    dft_inv<8>(y);
                }
#pragma unroll
                for (int m = 0; m < 8; ++m) {
                    ptr0[m * st] = x[m];
                    ptr1[m * st] = y[m];
                }
            });
            return;
        }
        for_tasks<TASKS, TL::T>([&](int q) {
            const int u1 = q >> LOGNI;
            int col, blk, j;
            TL::template decode<LOGJ>(q & (NI - 1), col, blk, j);
            u64* ptr = sm + TL::saddr(blk * L + j + u1 * JW, col);
            constexpr int st = TL::template step<8 * JW>();
            u64 x[8];
#pragma unroll
            for (int m = 0; m < (ZH ? 4 : 8); ++m) x[m] = ptr[m * st];
            if (!INV) {
                dft_fwd<8, ZH>(x);
                level1_twiddle<false, RT>(x, u1);
            } else {
                level1_twiddle<true, RT>(x, u1);
                dft_inv<8>(x);
            }
#pragma unroll
            for (int m = 0; m < 8; ++m) ptr[m * st] = x[m];
        });
    };
    auto level2 = [&]() {
        if constexpr (TL::PAIR && INV) {
            for_tasks<TASKS / 2, TL::T>([&](int p) {
                const int i1 = p >> (LOGNI - 1);
                int col, blk, j;
                TL::template decode<LOGJ>((p & (NI / 2 - 1)) << 1, col, blk, j);
                u64* ptr = sm + TL::saddr(blk * L + j + i1 * 8 * JW, col);
                constexpr int st = TL::template step<JW>();
                const int k1 = brev_c(i1, 3);
                u64 x[8], y[8];
#pragma unroll
                for (int m = 0; m < 8; ++m) {
                    const ulonglong2 v = ld2(ptr + m * st);
                    x[m] = v.x;
                    y[m] = v.y;
                }
                if (!INV) {
                    dft_fwd<8>(x);
                    dft_fwd<8>(y);
                    if (L > 64) {
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const int k = k1 + 8 * brev_c(i, 3);
                            const u64 w = __ldg(dtw + L + ((j * k) & (L - 1)));
                            x[i] = gl_mul(x[i], w);
                            y[i] = gl_mul(y[i], w);
                        }
                    }
                } else {
                    if (L > 64) {
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const int k = k1 + 8 * brev_c(i, 3);
                            const u64 w = __ldg(dtw + L + ((L - ((j * k) & (L - 1))) & (L - 1)));
                            x[i] = gl_mul(x[i], w);
                            y[i] = gl_mul(y[i], w);
                        }
                    }
                    dft_inv<8>(x);
                    dft_inv<8>(y);
                }
#pragma unroll
                for (int m = 0; m < 8; ++m) st2(ptr + m * st, make_ulonglong2(x[m], y[m]));
            });
            return;
        }
        for_tasks<TASKS, TL::T>([&](int q) {
            const int i1 = q >> LOGNI;
            int col, blk, j;
            TL::template decode<LOGJ>(q & (NI - 1), col, blk, j);
            u64* ptr = sm + TL::saddr(blk * L + j + i1 * 8 * JW, col);
            constexpr int st = TL::template step<JW>();
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
        });
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
template <class TL, bool INV>
__device__ __forceinline__ void lone8(u64* sm) {
    constexpr int LOGNB = TL::LR - 3;
    if constexpr (TL::PAIR && INV) {
        for_tasks<(1 << (LOGNB + TL::LC - 1)), TL::T>([&](int p) {
            const int col = (p << 1) & (TL::C - 1), blk = (p << 1) >> TL::LC;
            u64* ptr = sm + TL::saddr(blk * 8, col);
            constexpr int st = TL::template step<1>();
            u64 x[8], y[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const ulonglong2 v = ld2(ptr + m * st);
                x[m] = v.x;
                y[m] = v.y;
            }
            if (!INV) {
                dft_fwd<8>(x);
                dft_fwd<8>(y);
            } else {
                dft_inv<8>(x);
                dft_inv<8>(y);
            }
#pragma unroll
            for (int m = 0; m < 8; ++m) st2(ptr + m * st, make_ulonglong2(x[m], y[m]));
        });
        return;
    }
    for_tasks<(1 << (LOGNB + TL::LC)), TL::T>([&](int q) {
        int col, blk;
        if (TL::MAPK == MAP_COL) {
            col = q & (TL::C - 1);
            blk = q >> TL::LC;
        } else {
            blk = q & ((1 << LOGNB) - 1);
            col = q >> LOGNB;
        }
        u64* ptr = sm + TL::saddr(blk * 8, col);
        constexpr int st = TL::template step<1>();
        u64 x[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) x[m] = ptr[m * st];
        if (!INV) dft_fwd<8>(x);
        else dft_inv<8>(x);
#pragma unroll
        for (int m = 0; m < 8; ++m) ptr[m * st] = x[m];
    });
}

// Radix-64 groups from block size 2^LOGL down, G groups.
template <class TL, int LOGL, int G, bool RT, bool ZH = false>
__device__ __forceinline__ void groups_fwd(u64* sm, const u64* dtw) {
    if constexpr (G > 0) {
        group64<TL, LOGL, false, RT, ZH>(sm, dtw);
        __syncthreads();
        groups_fwd<TL, LOGL - 6, G - 1, RT>(sm, dtw);
    }
}
template <class TL, int LOGL, int G, bool RT>
__device__ __forceinline__ void groups_inv(u64* sm, const u64* dtw) {
    // inverse order: smallest block first
    if constexpr (G > 0) {
        groups_inv<TL, LOGL - 6, G - 1, RT>(sm, dtw);
        group64<TL, LOGL, true, RT>(sm, dtw);
        __syncthreads();
    }
}

// Whole column DFTs of the tile held in shared memory (callers synchronise
// before; the functions end with the tile synchronised). RT selects the form
// of the level-1 twiddles (level1_twiddle above): forward tiles with one
// radix-64 group keep the specialised bodies, tiles with two groups (whose
// specialised code stalled on instruction fetch) and all inverse tiles use
// the run-time shifts.
// ZH: rows [R/2, R) of every column are zero (first forward pass of an
// operand holding at most N/2 digits), so the first butterfly level of the
// column DFT -- in the lead step, or in the first group when there is none --
// has no additions and its zero half is not read.
// Level-1 twiddle form of a forward tile: run-time shifts where the tile has
// two radix-64 groups, or one group and a lone radix-8 level in 2^9 rows of
// two or more columns (two tasks per call: fwd_mid<9> 0.488 -> 0.469 ms at
// 2^26 points); the eight specialised bodies elsewhere (2^8-row tiles
// measured 4-6% slower with run-time shifts).
template <class TL>
constexpr bool fwd_rt() {
    return Steps<TL::LR>::G >= 2 || (TL::LR == 9 && TL::LC >= 1);
}

template <class TL, bool RT = fwd_rt<TL>(), bool ZH = false>
__device__ __forceinline__ void tile_fwd(u64* sm, const u64* dtw) {
    using S = Steps<TL::LR>;
    if constexpr (S::A > 0) {
        lead_step<TL, S::A, false, ZH>(sm, dtw);
        __syncthreads();
        groups_fwd<TL, TL::LR - S::A, S::G, RT>(sm, dtw);
    } else {
        groups_fwd<TL, TL::LR - S::A, S::G, RT, ZH>(sm, dtw);
    }
    if constexpr (S::LONE) {
        lone8<TL, false>(sm);
        __syncthreads();
    }
}

template <class TL, bool RT = true>
__device__ __forceinline__ void tile_inv(u64* sm, const u64* dtw) {
    using S = Steps<TL::LR>;
    if constexpr (S::LONE) {
        lone8<TL, true>(sm);
        __syncthreads();
    }
    groups_inv<TL, TL::LR - S::A, S::G, RT>(sm, dtw);
    if constexpr (S::A > 0) {
        lead_step<TL, S::A, true>(sm, dtw);
        __syncthreads();
    }
}

// w_{2^logM}^e from the two-level universal tables of RHO powers:
// u1[x & 0xFFFF] * u2[x >> 16] with x = e * 2^(32 - logM) (mod 2^32).
__device__ __forceinline__ u64 uroot(u32 x, const u64* __restrict__ u1, const u64* __restrict__ u2) {
    return gl_mul(__ldg(u1 + (x & 0xFFFFu)), __ldg(u2 + (x >> 16)));
}

}  // namespace b2m
