// school.cuh -- schoolbook product of two small u32-limb numbers by one CTA.
//
// The one-CTA NTT product (k_mul_small) costs about N log2 N * 75 integer
// instructions for N transform points; a schoolbook product costs about
// 4.5 instructions per limb multiply-add, so for the smaller and the
// unbalanced products of up to 2^13 points (na + nb <= 4096 limbs) it is the
// cheaper of the two. Reference
// counterpart: mul_schoolbook (src/bignum.cpp:125-143), the same column
// products, here with every column sum of a thread's four-column block
// accumulated in 96 bits by one carry chain per multiply-add, and the carries
// resolved by a block scan of carry functions (carry.cuh).
#pragma once
#include "carry.cuh"

namespace b2m {

// A product takes the schoolbook path when na * nb <= SCHOOL_MACS_PER_POINT * N
// for the N-point one-CTA NTT it would otherwise use. Measured on a B200 in
// batches of 4096 products: schoolbook ~0.28 us per 10^6 limb multiply-adds,
// one-CTA NTT ~4e-5 us per transform point (2^11..2^13 points), so the two
// cost the same near na * nb = 140 N; below ~256 limbs the schoolbook is 2-4x
// faster, at 2048 x 2048 limbs 3x slower.
#ifndef B2M_SCHOOL_MACS_PER_POINT
#define B2M_SCHOOL_MACS_PER_POINT 128
#endif
constexpr unsigned long long SCHOOL_MACS_PER_POINT = B2M_SCHOOL_MACS_PER_POINT;

__device__ __forceinline__ bool school_cheaper(u64 na, u64 nb, int logn) {
    return na * nb <= (1ull << logn) * SCHOOL_MACS_PER_POINT;
}

// (lo, mid, hi) += x * y as one 96-bit carry chain.
__device__ __forceinline__ void mac96(u32& lo, u32& mid, u32& hi, u32 x, u32 y) {
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(lo), "+r"(mid), "+r"(hi)
        : "r"(x), "r"(y));
}

// Bytes of shared memory school_cta needs: both operands (b padded by up to
// seven words) and three words of every column sum.
__host__ __device__ constexpr u64 school_smem_bytes(u64 na, u64 nb) { return 16 * (na + nb) + 48; }

// out[0, na + nb) = a * b and *out_len = its trimmed length (when out_len is
// not null), by all threads of the block. `smem`: school_smem_bytes(na, nb)
// bytes; `st`: one CState per thread. nout = na + nb.
static __device__ __noinline__ void school_cta(const u32* __restrict__ a, u64 na, const u32* __restrict__ b, u64 nb,
                                               u32* __restrict__ out, unsigned long long* out_len, unsigned char* smem,
                                               CState* st, unsigned long long* s_top) {
    const int T = blockDim.x, t = threadIdx.x;
    const int la = (int)na, lb = (int)nb, nc = la + lb;
    // b is stored as four interleaved quarter arrays, b[j] at (j & 3) * qb +
    // (j >> 2), so that lanes reading b[k0 + c - i] with k0 = 4 * lane read
    // consecutive words.
    const int qb = (lb + 3) / 4 + 1;
    u32* sa = reinterpret_cast<u32*>(smem);
    u32* sb = sa + la;
    u32* c0 = sb + 4 * qb;  // column sums: c0 + c1 * 2^32 + c2 * 2^64
    u32* c1 = c0 + nc;
    u32* c2 = c1 + nc;
    for (int i = t; i < la; i += T) sa[i] = __ldg(a + i);
    for (int j = t; j < lb; j += T) sb[(j & 3) * qb + (j >> 2)] = __ldg(b + j);
    if (t == 0) *s_top = 0;
    __syncthreads();

    // Column sums. A group of L = min(32, T) lanes (one warp or less) takes a
    // block of 4L consecutive columns, lane l the four at k0 = K0 + 4l, and
    // all lanes of the group step through the block's whole range of i
    // together (terms outside a lane's own range read b as zero), so the loop
    // is warp-uniform. Window w[c] = b[k0 + c - i] slides down a limb a step.
    const int L = T < 32 ? T : 32, lane = t % L, group = t / L, ngroups = T / L;
    for (int K0 = 4 * L * group; K0 < nc; K0 += 4 * L * ngroups) {
        const int k0 = K0 + 4 * lane;
        const int i0 = K0 - lb + 1 > 0 ? K0 - lb + 1 : 0;
        const int i1 = K0 + 4 * L - 1 < la - 1 ? K0 + 4 * L - 1 : la - 1;
        u32 lo[4] = {0, 0, 0, 0}, mid[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
        u32 w[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int j = k0 + c - i0;
            w[c] = (j >= 0 && j < lb) ? sb[(j & 3) * qb + (j >> 2)] : 0u;
        }
        for (int i = i0; i <= i1; ++i) {
            const u32 x = sa[i];
#pragma unroll
            for (int c = 0; c < 4; ++c) mac96(lo[c], mid[c], hi[c], x, w[c]);
            w[3] = w[2];
            w[2] = w[1];
            w[1] = w[0];
            const int j = k0 - i - 1;
            w[0] = (j >= 0 && j < lb) ? sb[(j & 3) * qb + (j >> 2)] : 0u;
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
