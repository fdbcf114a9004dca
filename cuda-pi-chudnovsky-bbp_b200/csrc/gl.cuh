// gl.cuh -- Goldilocks field GF(p), p = 2^64 - 2^32 + 1, for host and device.
//
// Same field as the reference's include/goldilocks.h:83-189 (constants, add,
// sub, 128-bit Solinas fold, mul, pow, inverse), written afresh for this
// backend: every function keeps values canonical in [0, p), and multiplication
// by a power of two (gl_shl) is a shift plus a fold instead of a full multiply,
// which is what makes the radix-64 register butterflies cheap:
//   2^64 == 2^32 - 1 (mod p), 2^96 == -1, 2^192 == 1,
// so 2 has order 192 and 8 = 2^3 is a primitive 64th root of unity.
//
// The transform root used throughout is RHO, a primitive 2^32-th root chosen
// so that RHO^(2^26) == 8. With it every power-of-two root in the transform is
// a power of RHO and the radix-64 roots are exactly the shift roots, so the
// register butterflies (shifts) and the table twiddles (powers of RHO) agree.
// RHO = 7^(5 (p-1) / 2^32); the reference uses 7^((p-1)/N) per size
// (goldilocks.h:187-189). Only the product integer is defined by the
// reference, not the spectrum, so the choice of root is free.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define GL_FN __host__ __device__ __forceinline__
#else
#define GL_FN inline
#endif

namespace b2m {

typedef unsigned long long u64;
typedef unsigned int u32;

constexpr u64 GL_P = 0xFFFFFFFF00000001ull;
constexpr u64 GL_EPS = 0xFFFFFFFFull;  // 2^64 mod p
constexpr u64 GL_RHO = 0xe2af70635744fd26ull;

GL_FN u64 gl_mulhi(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (u64)(((unsigned __int128)a * b) >> 64);
#endif
}

// a - b for a < 2^64, b <= p: a borrow wraps by 2^64 == EPS too many, and
// since b - a <= p the corrected value cannot borrow again. Canonical when
// a is. The device version is one 32-bit borrow chain plus the borrow bit
// beta, and the correction d - beta*EPS = d + beta - beta*2^32 is done by a
// wide multiply-add and a multiply-add on the high word: the integer ALU
// pipe (which bounds the transforms) issues three instructions, the
// otherwise idle FMA pipe the rest.
GL_FN u64 gl_sub(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
    u32 d0, d1, bt;
    asm("sub.cc.u32 %0, %3, %5;\n\t"
        "subc.cc.u32 %1, %4, %6;\n\t"
        "subc.u32 %2, 0, 0;"
        : "=r"(d0), "=r"(d1), "=r"(bt)
        : "r"((u32)a), "r"((u32)(a >> 32)), "r"((u32)b), "r"((u32)(b >> 32)));
    // bt = -beta (0 or 0xFFFFFFFF)
    u64 r;
    asm("mad.wide.u32 %0, %1, 1, %2;" : "=l"(r) : "r"(0u - bt), "l"(((u64)d1 << 32) | d0));
    return ((u64)((u32)(r >> 32) + bt) << 32) | (u32)r;
#else
    u64 d = a - b;
    return (a < b) ? d - GL_EPS : d;
#endif
}

// a + b for canonical a, b, computed as a - (p - b) (p - b <= p, so gl_sub
// applies): two instructions for p - b and gl_sub, instead of an add
// followed by two range checks.
GL_FN u64 gl_add(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
    u32 n0, n1;
    asm("sub.cc.u32 %0, 1, %2;\n\t"
        "subc.u32 %1, -1, %3;\n\t"
        : "=r"(n0), "=r"(n1)
        : "r"((u32)b), "r"((u32)(b >> 32)));
    return gl_sub(a, ((u64)n1 << 32) | n0);
#else
    u64 s = a + b;
    u64 t = s + GL_EPS;            // s - p (mod 2^64)
    bool wrap = s < a;             // a + b >= 2^64
    return (wrap || s >= GL_P) ? t : s;
#endif
}

GL_FN u64 gl_neg(u64 a) { return a ? GL_P - a : 0; }

// lo + h * 2^64 for h < 2^32:  == lo + h * EPS, with h*EPS < 2^64.
GL_FN u64 gl_fold32(u64 lo, u64 h) {
    u64 t1 = h * GL_EPS;
    u64 t2 = lo + t1;
    if (t2 < t1) t2 += GL_EPS;     // the second fold cannot carry again
    return t2 >= GL_P ? t2 - GL_P : t2;
}

// Full 128-bit value hi:lo reduced: hi = hh*2^32 + hl contributes
// hl*2^64 == hl*EPS and hh*2^96 == -hh.
GL_FN u64 gl_reduce128(u64 lo, u64 hi) {
    u64 hh = hi >> 32, hl = hi & 0xFFFFFFFFull;
    u64 t0 = lo - hh;
    if (lo < hh) t0 -= GL_EPS;
    return gl_fold32(t0, hl);
}

#if defined(__CUDA_ARCH__)
// ---------------------------------------------------------------------------
// Device folds on 32-bit words. A value V = H*2^32 + P - L with H < 2^32 and
// -p < V < 2^64 is one borrow chain: on a borrow, V + p is the wrapped
// difference minus EPS (the wrap added 2^64 = p + EPS).
// ---------------------------------------------------------------------------
__device__ __forceinline__ u64 gl_hpl(u32 H, u32 P, u32 Lc, u32 Ll) {
    u32 d0, d1;
    asm("{\n\t.reg .u32 m;\n\t"
        "sub.cc.u32 %0, %3, %5;\n\t"
        "subc.cc.u32 %1, %2, %4;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t}"
        : "=r"(d0), "=r"(d1)
        : "r"(H), "r"(P), "r"(Lc), "r"(Ll));
    return ((u64)d1 << 32) | d0;
}

// End-around sum of two words: (a + b) mod 2^32 plus the carry, and the carry.
// For a + b <= 2^33 - 2 the result fits a word, and
// (a + b) * 2^32 == result * 2^32 - carry (mod p) since 2^64 == 2^32 - 1.
__device__ __forceinline__ u32 gl_ea_add(u32 a, u32 b, u32& c) {
    u32 t;
    asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, 0, 0;" : "=r"(t), "=r"(c) : "r"(a), "r"(b));
    return t + c;
}

// a + b + c as a 33-bit value hi:lo.
__device__ __forceinline__ void gl_add3(u32 a, u32 b, u32 c, u32& hi, u32& lo) {
    asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, 0, 0;" : "=r"(lo), "=r"(hi) : "r"(a), "r"(b));
    asm("add.cc.u32 %0, %0, %2;\n\taddc.u32 %1, %1, 0;" : "+r"(lo), "+r"(hi) : "r"(c));
}

__device__ __forceinline__ u64 gl_canon(u64 r) { return r >= GL_P ? r - GL_P : r; }
#endif

// a * b. Device: the 128-bit product r3:r2:r1:r0 from 32-bit multiply-adds,
// then V == (r1 + r2)*2^32 + r0 - r2 - r3 folded with one end-around carry
// and one borrow chain (range -2^33 < V < 2^64), and one range check.
GL_FN u64 gl_mul(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
    const u32 a0 = (u32)a, a1 = (u32)(a >> 32), b0 = (u32)b, b1 = (u32)(b >> 32);
    u32 r0, r1, r2, r3;
    asm("mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "addc.u32 %3, 0, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, %3;"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
    u32 hc, lc, ll;
    const u32 h = gl_ea_add(r1, r2, hc);
    gl_add3(r2, r3, hc, lc, ll);
    return gl_canon(gl_hpl(h, r0, lc, ll));
#else
    return gl_reduce128(a * b, gl_mulhi(a, b));
#endif
}

#if defined(__CUDA_ARCH__)
// x * 2^t for x < 2^64 and 0 < t < 32, canonical: x*2^t = W2*2^64 + L
// (L = W1:W0, W2 < 2^t), and W2*2^64 == W2*EPS, so U = L + W2*EPS < 2p. One
// wide multiply-add forms U mod 2^64 = T; U overflowed 2^64 exactly when
// T < L (the added W2*EPS < 2^64). The canonical value is T + EPS (mod
// 2^64) when U overflowed (then U - p = T + EPS, no wrap since T < 2^63) or
// when T >= p (T + EPS carries), and T otherwise.
__device__ __forceinline__ u64 gl_shl_w0(u64 x, int t) {
    const u32 x0 = (u32)x, x1 = (u32)(x >> 32);
    const u64 L = ((u64)__funnelshift_l(x0, x1, t) << 32) | (x0 << t);
    const u32 W2 = x1 >> (32 - t);
    u64 T;
    asm("mad.wide.u32 %0, %1, -1, %2;" : "=l"(T) : "r"(W2), "l"(L));
    u32 e0, e1, c;
    asm("add.cc.u32 %0, %3, -1;\n\taddc.cc.u32 %1, %4, 0;\n\taddc.u32 %2, 0, 0;"
        : "=r"(e0), "=r"(e1), "=r"(c)
        : "r"((u32)T), "r"((u32)(T >> 32)));
    return ((T < L) | c) ? (((u64)e1 << 32) | e0) : T;
}

// x * 2^(32 + t) for x < 2^64 and 0 <= t < 32, canonical: with W = x*2^t =
// W2:W1:W0, x*2^(32+t) = W0*2^32 + W1*2^64 + W2*2^96 == (W0 + W1)*2^32 -
// (W1 + W2). Writing W0 + W1 = hc*2^32 + h (hc*2^64 == hc*EPS), the first
// term is A = (h + hc)*2^32 - hc, the 64-bit word pair (h, -hc) -- at most
// p - 1, since hc = 1 forces h <= 2^32 - 2 -- and the second B = W1 + W2 <
// 2^33, so the value is gl_sub(A, B), canonical.
__device__ __forceinline__ u64 gl_shl_w1(u64 x, int t) {
    const u32 x0 = (u32)x, x1 = (u32)(x >> 32);
    const u32 W0 = x0 << t, W1 = t ? __funnelshift_l(x0, x1, t) : x1, W2 = t ? x1 >> (32 - t) : 0u;
    u32 h, hc;
    asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, 0, 0;" : "=r"(h), "=r"(hc) : "r"(W0), "r"(W1));
    return gl_sub(((u64)h << 32) | (0u - hc), (u64)W1 + W2);
}

// x * 2^(64 + t) for x < 2^64 and 0 <= t < 32, canonical: W0*2^64 + W1*2^96
// + W2*2^128 == W0*EPS - W1 - W2*2^32 = W0*2^32 - ((W2 + c)*2^32 + l) where
// c:l = W0 + W1; the subtrahend is below 2^(32+t) + 2^33 <= p and the
// minuend at most p - 1, so gl_sub gives the canonical value.
__device__ __forceinline__ u64 gl_shl_w2(u64 x, int t) {
    const u32 x0 = (u32)x, x1 = (u32)(x >> 32);
    const u32 W0 = x0 << t, W1 = t ? __funnelshift_l(x0, x1, t) : x1, W2 = t ? x1 >> (32 - t) : 0u;
    u32 l, c;
    asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, 0, 0;" : "=r"(l), "=r"(c) : "r"(W0), "r"(W1));
    return gl_sub((u64)W0 << 32, ((u64)(W2 + c) << 32) | l);
}

#endif

// x * 2^s for canonical x and 0 <= s < 192. Written so that, with s known at
// compile time (the register butterflies), every branch folds away; with s
// warp-uniform at run time the branches are uniform.
//
// Device: s = 96n + 32w + t; the word offset w selects gl_shl_w0/w1/w2
// (each canonical for any 64-bit input), and 2^96 == -1 negates.
GL_FN u64 gl_shl(u64 x, int s) {
#if defined(__CUDA_ARCH__)
    if (s == 0) return x;
    const bool neg = s >= 96;
    if (neg) s -= 96;
    const int t = s & 31, w = s >> 5;
    u64 r;
    if (w == 0) r = t ? gl_shl_w0(x, t) : x;
    else if (w == 1) r = gl_shl_w1(x, t);
    else r = gl_shl_w2(x, t);
    return neg ? gl_sub(0, r) : r;
#else
    bool neg = false;
    if (s >= 96) { s -= 96; neg = true; }   // 2^96 == -1
    u64 r;
    if (s == 0) {
        r = x;
    } else if (s <= 32) {
        r = gl_fold32(x << s, x >> (64 - s));
    } else if (s < 64) {
        r = gl_reduce128(x << s, x >> (64 - s));
    } else if (s == 64) {
        r = gl_reduce128(0, x);
    } else {
        // x*2^(s-64) = zl + zh*2^64 (zh < 2^32); times 2^64:
        // zl*2^64 + zh*2^128 == zl*2^64 - zh*2^32.
        u64 zl = x << (s - 64), zh = x >> (128 - s);
        r = gl_sub(gl_reduce128(0, zl), zh << 32);
    }
    return neg ? gl_neg(r) : r;
#endif
}

// x * 2^(160 + t) for x < 2^64 and a run-time 0 <= t < 32, canonical, branch
// free: 2^(160+t) = -2^(64+t), and gl_shl_w2's value A - B negated is B - A
// (A = W0*2^32 <= p - 1 is a valid subtrahend, B < p). This is N^-1 = 2^(192-k)
// for N = 2^k.
__device__ __forceinline__ u64 gl_shl_160(u64 x, int t) {
    const u32 x0 = (u32)x, x1 = (u32)(x >> 32);
    const u32 W0 = x0 << t, W1 = __funnelshift_l(x0, x1, t), W2 = __funnelshift_l(x1, 0u, t);
    u32 l, c;
    asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, 0, 0;" : "=r"(l), "=r"(c) : "r"(W0), "r"(W1));
    return gl_sub(((u64)(W2 + c) << 32) | l, (u64)W0 << 32);
}

#if defined(__CUDA_ARCH__)
// x * 2^(32w + t) for a word offset w in {0, 1, 2} and 0 <= t < 32, the three
// folds of the run-time shift (t = 0 needs no case of its own: the funnel
// shifts give W2 = 0 and the folds stay exact).
__device__ __forceinline__ u64 gl_shl_wt(u64 x, u32 w, u32 t) {
    const u32 x0 = (u32)x, x1 = (u32)(x >> 32);
    const u32 W0 = x0 << t, W1 = __funnelshift_l(x0, x1, t), W2 = __funnelshift_l(x1, 0u, t);
    if (w == 0) {
        const u64 L = ((u64)W1 << 32) | W0;
        u64 T;
        asm("mad.wide.u32 %0, %1, -1, %2;" : "=l"(T) : "r"(W2), "l"(L));
        u32 e0, e1, c;
        asm("add.cc.u32 %0, %3, -1;\n\taddc.cc.u32 %1, %4, 0;\n\taddc.u32 %2, 0, 0;"
            : "=r"(e0), "=r"(e1), "=r"(c)
            : "r"((u32)T), "r"((u32)(T >> 32)));
        return ((T < L) | c) ? (((u64)e1 << 32) | e0) : T;
    } else if (w == 1) {
        u32 h, hc;
        asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, 0, 0;" : "=r"(h), "=r"(hc) : "r"(W0), "r"(W1));
        return gl_sub(((u64)h << 32) | (0u - hc), (u64)W1 + W2);
    } else {
        u32 l, c;
        asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, 0, 0;" : "=r"(l), "=r"(c) : "r"(W0), "r"(W1));
        return gl_sub((u64)W0 << 32, ((u64)(W2 + c) << 32) | l);
    }
}
#endif

// x * 2^s for x < 2^64 and a run-time, warp-uniform 0 <= s < 192: one copy
// of the three word-offset folds behind uniform branches, so a site costs a
// few hundred bytes of code instead of one specialised body per shift amount.
static __device__ __noinline__ u64 gl_shl_rt(u64 x, u32 s) {
#if defined(__CUDA_ARCH__)
    const bool neg = s >= 96;
    if (neg) s -= 96;
    const u64 r = gl_shl_wt(x, s >> 5, s & 31);
    return neg ? gl_sub(0, r) : r;
#else
    return gl_shl(x, (int)s);
#endif
}

// The same shift of two values (one call, one decode of s): the paired
// inverse tile tasks shift both columns' elements by the same amount.
static __device__ __noinline__ ulonglong2 gl_shl_rt2(u64 x, u64 y, u32 s) {
#if defined(__CUDA_ARCH__)
    const bool neg = s >= 96;
    if (neg) s -= 96;
    const u32 w = s >> 5, t = s & 31;
    u64 rx, ry;
    if (w == 0) {
        rx = gl_shl_wt(x, 0, t);
        ry = gl_shl_wt(y, 0, t);
    } else if (w == 1) {
        rx = gl_shl_wt(x, 1, t);
        ry = gl_shl_wt(y, 1, t);
    } else {
        rx = gl_shl_wt(x, 2, t);
        ry = gl_shl_wt(y, 2, t);
    }
    if (neg) {
        rx = gl_sub(0, rx);
        ry = gl_sub(0, ry);
    }
    return make_ulonglong2(rx, ry);
#else
    return make_ulonglong2(gl_shl(x, (int)s), gl_shl(y, (int)s));
#endif
}

GL_FN u64 gl_pow(u64 b, u64 e) {
    u64 r = 1;
    while (e) {
        if (e & 1) r = gl_mul(r, b);
        b = gl_mul(b, b);
        e >>= 1;
    }
    return r;
}

GL_FN u64 gl_inv(u64 a) { return gl_pow(a, GL_P - 2); }

// Primitive 2^l-th root of unity in the RHO chain (l <= 32).
GL_FN u64 gl_root2(int l) { return gl_pow(GL_RHO, 1ull << (32 - l)); }

}  // namespace b2m
