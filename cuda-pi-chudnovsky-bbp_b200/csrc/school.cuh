// school.cuh -- schoolbook product of two small u32-limb numbers by one CTA.
//
// The one-CTA NTT product (k_mul_small) costs about N log2 N * 75 integer
// instructions for N transform points; a schoolbook product costs about
// 4.5 instructions per limb multiply-add, so for most products of up to
// 2^13 points (na + nb <= 4096 limbs) it is the cheaper of the two. Reference
// counterpart: mul_schoolbook (src/bignum.cpp:125-143), the same column
// products, here with every column sum of a thread's four-column block
// accumulated in 96 bits by one carry chain per multiply-add, and the carries
// resolved by a block scan of carry functions (carry.cuh).
#pragma once
#include "carry.cuh"

namespace b2m {

// Products whose schoolbook cost is below this many limb multiply-adds per
// transform point and level of the NTT they would otherwise use.
#ifndef B2M_SCHOOL_MACS_PER_POINT_LEVEL
#define B2M_SCHOOL_MACS_PER_POINT_LEVEL 16
#endif
constexpr unsigned long long SCHOOL_MACS_PER_POINT_LEVEL = B2M_SCHOOL_MACS_PER_POINT_LEVEL;

__device__ __forceinline__ bool school_cheaper(u64 na, u64 nb, int logn) {
    return na * nb <= ((1ull << logn) * (unsigned long long)logn) * SCHOOL_MACS_PER_POINT_LEVEL;
}

// (lo, mid, hi) += x * y as one 96-bit carry chain.
__device__ __forceinline__ void mac96(u32& lo, u32& mid, u32& hi, u32 x, u32 y) {
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(lo), "+r"(mid), "+r"(hi)
        : "r"(x), "r"(y));
}

// Bytes of shared memory school_cta needs: both operands and three words of
// every column sum.
__host__ __device__ constexpr u64 school_smem_bytes(u64 na, u64 nb) { return 16 * (na + nb) + 16; }

// out[0, na + nb) = a * b and *out_len = its trimmed length (when out_len is
// not null), by all threads of the block. `smem`: school_smem_bytes(na, nb)
// bytes; `st`: one CState per thread. nout = na + nb.
static __device__ __noinline__ void school_cta(const u32* __restrict__ a, u64 na, const u32* __restrict__ b, u64 nb,
                                               u32* __restrict__ out, unsigned long long* out_len, unsigned char* smem,
                                               CState* st, unsigned long long* s_top) {
    const int T = blockDim.x, t = threadIdx.x;
    const int la = (int)na, lb = (int)nb, nc = la + lb;
    u32* sa = reinterpret_cast<u32*>(smem);
    u32* sb = sa + la;
    u32* c0 = sb + lb;  // column sums: c0 + c1 * 2^32 + c2 * 2^64
    u32* c1 = c0 + nc;
    u32* c2 = c1 + nc;
    for (int i = t; i < la; i += T) sa[i] = __ldg(a + i);
    for (int j = t; j < lb; j += T) sb[j] = __ldg(b + j);
    if (t == 0) *s_top = 0;
    __syncthreads();

    // Column sums, four consecutive columns a task, tasks strided over threads.
    // Window w[c] = b[k0 + c - i] slides down one limb per step of i.
    for (int k0 = 4 * t; k0 < nc; k0 += 4 * T) {
        u32 lo[4] = {0, 0, 0, 0}, mid[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
        const int i0 = k0 - lb + 1 > 0 ? k0 - lb + 1 : 0;
        const int i1 = k0 + 3 < la - 1 ? k0 + 3 : la - 1;
        u32 w[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int j = k0 + c - i0;
            w[c] = (j >= 0 && j < lb) ? sb[j] : 0u;
        }
        for (int i = i0; i <= i1; ++i) {
            const u32 x = sa[i];
#pragma unroll
            for (int c = 0; c < 4; ++c) mac96(lo[c], mid[c], hi[c], x, w[c]);
            w[3] = w[2];
            w[2] = w[1];
            w[1] = w[0];
            const int j = k0 - i - 1;  // never >= lb: i >= i0
            w[0] = j >= 0 ? sb[j] : 0u;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (k0 + c < nc) {
                c0[k0 + c] = lo[c];
                c1[k0 + c] = mid[c];
                c2[k0 + c] = hi[c];
            }
        }
    }
    __syncthreads();

    // Carries: thread t owns columns [t*G, (t+1)*G), G >= 2 so that a carry
    // in (< 2^45) changes a range's carry out by at most one. Its limbs with
    // no carry in (written back over c0) and its carry function
    // f(c) = h + [c >= th]. Only the last non-empty range can be one limb
    // long, and only empty ranges, whose functions nothing uses, follow it.
    int G = (nc + T - 1) / T;
    if (G < 2) G = 2;
    const int k_beg = t * G < nc ? t * G : nc, k_end = k_beg + G < nc ? k_beg + G : nc;
    u64 carry = 0;
    bool upper_ones = true;
    u64 dl = 0;
    for (int k = k_beg; k < k_end; ++k) {
        const u64 s0 = (u64)c0[k] + carry;  // carry < 2^45: column sums are below 2^76
        const u32 limb = (u32)s0;
        carry = (s0 >> 32) + c1[k] + ((u64)c2[k] << 32);
        c0[k] = limb;
        const int m = k - k_beg;
        if (m == 0) dl = limb;
        else if (m == 1) dl |= (u64)limb << 32;
        else upper_ones &= (limb == 0xFFFFFFFFu);
    }
    CState f{carry, CS_NEVER};
    if (k_end - k_beg >= 2 && upper_ones && dl != 0) {
        const u64 tt = 0ull - dl;  // 2^(32G) - L with L's upper limbs all ones
        if (tt < (1ull << 62)) f.t = tt;
    }
    u64 cin = 0;
    if (T >= 32) {
        bool has;
        CState agg;
        const CState ex = block_scan_carry(f, &has, &agg, st);
        cin = has ? cs_eval(ex, 0) : 0;
    } else {
        st[t] = f;
        __syncthreads();
        if (t == 0) {
            u64 c = 0;
            for (int u = 0; u < T; ++u) {
                const CState g = st[u];
                st[u].h = c;
                c = cs_eval(g, c);
            }
        }
        __syncthreads();
        cin = st[t].h;
    }
    // Add the carry in and store; the carry out of the range is f(cin).
    unsigned long long top = 0;
    for (int k = k_beg; k < k_end; ++k) {
        const u64 s0 = (u64)c0[k] + (cin & 0xFFFFFFFFull);
        const u32 limb = (u32)s0;
        cin = (cin >> 32) + (s0 >> 32);
        out[k] = limb;
        if (limb) top = (unsigned long long)k + 1;
    }
    if (top) atomicMax(s_top, top);
    __syncthreads();
    if (t == 0 && out_len) *out_len = *s_top;
}

}  // namespace b2m
