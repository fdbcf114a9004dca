// b2m_chudnovsky.cu -- Chudnovsky binary splitting, level by level, on the device.
//
// Reference counterpart: chudnovsky_bs (src/chudnovsky.cpp:64-102), a
// depth-first recursion that splits [a, b) at the midpoint and merges
//     P = PL*PR,  Q = QL*QR,  T = TL*QR + PL*TR      (:98-100)
// over leaves p(k) = (6k-5)(2k-1)(6k-1), q(k) = k^3 * 640320^3/24,
// t(k) = (-1)^k p(k) (13591409 + 545140134 k), and p(0) = q(0) = 1,
// t(0) = 13591409 (:68-90). Every product goes through mul_dispatch one at a
// time (src/bignum.cpp:204-232) and every value lives in host std::vectors.
//
// Here the tree is built bottom-up, a level at a time, with every value
// resident in HBM: level 0 holds the b - a leaves, and level l+1 merges
// nodes (2i, 2i+1) of level l (an odd last node is carried up unchanged).
// P and Q are products and T/Q is the exact partial sum of the series, so the
// root (P, Q, T) does not depend on the shape of the tree and equals the
// reference's. Per level all 4 * m/2 products run together: a warp per
// product (schoolbook) while operands are at most 64 limbs, otherwise the
// batched NTT buckets (b2m_batch's launch_bucket). T is then formed by a
// sign-magnitude add/subtract kernel (the reference's BigInt operator+,
// src/bignum.cpp:310-325). Values of a level sit at a fixed stride (the
// level's length bound); only three maximum lengths per level come back to
// the host, to plan the next level.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "b2m.h"
#include "b2m_context.h"
#include "b2m_internal.h"
#include "gp_scan.cuh"

namespace b2m {

typedef unsigned __int128 u128;

constexpr uint64_t BS_MAX_TERMS = 2000000;  // leaves fit 4 limbs (k^3 < 2^63)
constexpr uint64_t SCHOOL_MAX = 64;         // warp-per-product schoolbook up to this many limbs
constexpr int SCHOOL_WARPS = 8;

// One level: m nodes; family f in {P=0, Q=1, T=2} at limbs[f] + i*stride[f];
// trimmed lengths len[f*m + i]; sign[i] of T (P and Q are positive).
struct LevelView {
    uint64_t m;
    uint64_t stride[3];
    u32* limbs[3];
    u64* len;
    int* sign;
};

// ---------------------------------------------------------------------------- leaves
__device__ __forceinline__ void put128(u32* dst, u64* len, u128 v) {
    int n = 0;
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        const u32 x = (u32)(v >> (32 * w));
        dst[w] = x;
        if (x) n = w + 1;
    }
    *len = (u64)n;
}

__global__ void k_bs_leaves(u64 a, LevelView L) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.m) return;
    const u64 k = a + i;
    u128 p, q, t;
    int s = 1;
    if (k == 0) {
        p = 1;
        q = 1;
        t = 13591409u;
    } else {
        p = (u128)((6 * k - 5) * (2 * k - 1)) * (6 * k - 1);
        q = (u128)(k * k * k) * 10939058860032000ull;
        t = p * (u128)(13591409ull + 545140134ull * k);
        if (k & 1) s = -1;
    }
    put128(L.limbs[0] + i * L.stride[0], L.len + i, p);
    put128(L.limbs[1] + i * L.stride[1], L.len + L.m + i, q);
    put128(L.limbs[2] + i * L.stride[2], L.len + 2 * L.m + i, t);
    L.sign[i] = s;
}

__global__ void k_bs_maxlen(const u64* __restrict__ len, u64 m, unsigned long long* out) {
    unsigned long long mx[3] = {0, 0, 0};
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x)
        for (int f = 0; f < 3; ++f) mx[f] = max(mx[f], (unsigned long long)len[f * m + i]);
    for (int f = 0; f < 3; ++f) {
        for (int off = 16; off > 0; off >>= 1) mx[f] = max(mx[f], __shfl_xor_sync(0xFFFFFFFFu, mx[f], off));
        if ((threadIdx.x & 31) == 0 && mx[f]) atomicMax(out + f, mx[f]);
    }
}

// ---------------------------------------------------------------------------- products
// Operands and destination of product `kind` of merge i (see the file comment).
struct MergeProd {
    const u32* a;
    u64 na;
    const u32* b;
    u64 nb;
    u32* out;
    u64* out_len;
};
struct ScratchXY {
    u32* x;
    u32* y;
    u64 sx, sy;  // strides
    u64* lx;
    u64* ly;
};

__device__ __forceinline__ MergeProd merge_prod(const LevelView& L, const LevelView& Ln, const ScratchXY& S,
                                                u64 i, int kind) {
    const u64 l = 2 * i, r = 2 * i + 1;
    auto val = [&](int f, u64 n) { return (const u32*)(L.limbs[f] + n * L.stride[f]); };
    auto ln = [&](int f, u64 n) { return L.len[f * L.m + n]; };
    MergeProd p;
    switch (kind) {
        case 0:  // P' = PL * PR
            p = {val(0, l), ln(0, l), val(0, r), ln(0, r), Ln.limbs[0] + i * Ln.stride[0], Ln.len + i};
            break;
        case 1:  // Q' = QR * QL (QR first: X shares its spectrum)
            p = {val(1, r), ln(1, r), val(1, l), ln(1, l), Ln.limbs[1] + i * Ln.stride[1], Ln.len + Ln.m + i};
            break;
        case 2:  // X = QR * TL
            p = {val(1, r), ln(1, r), val(2, l), ln(2, l), S.x + i * S.sx, S.lx + i};
            break;
        default:  // Y = PL * TR
            p = {val(0, l), ln(0, l), val(2, r), ln(2, r), S.y + i * S.sy, S.ly + i};
    }
    return p;
}

// Warp per product: column sums (u64 + overflow count) by the lanes, then one
// lane resolves the carries. For operands of at most SCHOOL_MAX limbs.
__global__ void __launch_bounds__(SCHOOL_WARPS * 32) k_bs_school(LevelView L, LevelView Ln, ScratchXY S,
                                                                 u64 m2, u32 kinds_mask) {
    __shared__ u64 s_lo[SCHOOL_WARPS][2 * SCHOOL_MAX];
    __shared__ u32 s_hi[SCHOOL_WARPS][2 * SCHOOL_MAX];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 j = (u64)blockIdx.x * SCHOOL_WARPS + warp;
    if (j >= 4 * m2) return;
    const int kind = (int)(j & 3);
    if (!((kinds_mask >> kind) & 1)) return;
    const MergeProd p = merge_prod(L, Ln, S, j >> 2, kind);
    if (p.na == 0 || p.nb == 0) {
        if (lane == 0) *p.out_len = 0;
        return;
    }
    const int nc = (int)(p.na + p.nb - 1);
    for (int k = lane; k < nc; k += 32) {
        u64 lo = 0;
        u32 hi = 0;
        const int i0 = k - (int)p.nb + 1 > 0 ? k - (int)p.nb + 1 : 0;
        const int i1 = k < (int)p.na - 1 ? k : (int)p.na - 1;
        for (int i = i0; i <= i1; ++i) {
            const u64 prod = (u64)__ldg(p.a + i) * __ldg(p.b + k - i);
            lo += prod;
            hi += (lo < prod);
        }
        s_lo[warp][k] = lo;
        s_hi[warp][k] = hi;
    }
    __syncwarp();
    if (lane == 0) {
        u64 c = 0;
        int top = 0;
        for (int k = 0; k < nc; ++k) {
            const u128 t = ((u128)s_hi[warp][k] << 64) + s_lo[warp][k] + c;
            const u32 w = (u32)t;
            p.out[k] = w;
            if (w) top = k + 1;
            c = (u64)(t >> 32);
        }
        p.out[nc] = (u32)c;
        if ((u32)c) top = nc + 1;
        *p.out_len = (u64)top;
    }
}

// Job tables of one product kind for the NTT buckets. With spec_ws, job i's
// first operand is already transformed in the bufA of the partner product's
// job i (its workspace at spec_ws + i * spec_stride), and this job's
// workspace holds only bufB and the carry scratch.
__global__ void k_bs_build_jobs(LevelView L, LevelView Ln, ScratchXY S, u64 m2, int kind, ProdJob* jobs,
                                unsigned char* ntt_ws, u64 ws_stride, u64 npts, unsigned char* spec_ws,
                                u64 spec_stride) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m2) return;
    const MergeProd p = merge_prod(L, Ln, S, i, kind);
    ProdJob J{};
    J.a = p.a;
    J.b = p.b;
    J.na = p.na;
    J.nb = p.nb;
    J.out = p.out;
    J.out_len = reinterpret_cast<unsigned long long*>(p.out_len);
    if (ntt_ws) {
        const u64 n = npts;
        unsigned char* w = ntt_ws + i * ws_stride;
        unsigned char* scratch;
        if (spec_ws) {
            J.bufA = reinterpret_cast<u64*>(spec_ws + i * spec_stride);
            J.bufB = reinterpret_cast<u64*>(w);
            scratch = w + 8 * n;
        } else {
            J.bufA = reinterpret_cast<u64*>(w);
            J.bufB = J.bufA + n;
            scratch = w + 16 * n;
        }
        J.slots = reinterpret_cast<LookbackSlot*>(scratch);
        J.ticket = reinterpret_cast<u32*>(scratch + (n / CARRY_CHUNK) * sizeof(LookbackSlot));
    }
    jobs[i] = J;
}

// Zero the lengths the products accumulate with atomicMax and the carry scratch.
__global__ void k_bs_zero(unsigned long long* p, u64 n) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = 0;
}
__global__ void k_bs_zero_ws(const ProdJob* __restrict__ jobs, u64 njobs, u64 scratch_words) {
    // one block per job: its lookback slots + ticket, and its length
    const u64 j = blockIdx.x;
    if (j >= njobs) return;
    unsigned long long* s = reinterpret_cast<unsigned long long*>(jobs[j].slots);
    for (u64 i = threadIdx.x; i < scratch_words; i += blockDim.x) s[i] = 0;
    if (threadIdx.x == 0) *jobs[j].out_len = 0;
}

// ---------------------------------------------------------------------------- T = sx*X + sy*Y
// One CTA per merge: T' = sign(TL)*X + sign(TR)*Y (X = TL*QR, Y = PL*TR).
__global__ void k_bs_signed_add(const ScratchXY S, const int* __restrict__ sign_l, LevelView Ln, u64 m2) {
    __shared__ GP s_ws[33];
    __shared__ u32 s_carry;
    __shared__ unsigned long long s_top;
    __shared__ long long s_diff;
    const u64 i = blockIdx.x;
    if (i >= m2) return;
    const u32* X = S.x + i * S.sx;
    const u32* Y = S.y + i * S.sy;
    u64 lx = S.lx[i], ly = S.ly[i];
    int sx = sign_l[2 * i], sy = sign_l[2 * i + 1];
    if (lx == 0) sx = 0;
    if (ly == 0) sy = 0;
    u32* out = Ln.limbs[2] + i * Ln.stride[2];
    // Choose the operation: add (same signs), or big - small with big's sign.
    bool sub = false, swap = false;
    int sres;
    if (sx == 0) {
        sres = sy;
        swap = true;
        lx = 0;
    } else if (sy == 0) {
        sres = sx;
        ly = 0;
    } else if (sx == sy) {
        sres = sx;
    } else {
        sub = true;
        int c = 0;
        if (lx != ly) {
            c = lx > ly ? 1 : -1;
        } else {
            // top-down search for the highest differing limb
            if (threadIdx.x == 0) s_diff = -1;
            __syncthreads();
            const long long chunk = (long long)blockDim.x * ADD_LPT;
            for (long long hi = (long long)lx; hi > 0; hi -= chunk) {
                const long long lo = hi - chunk > 0 ? hi - chunk : 0;
                for (long long k = lo + threadIdx.x; k < hi; k += blockDim.x)
                    if (X[k] != Y[k]) atomicMax(&s_diff, k);
                __syncthreads();
                if (s_diff >= 0) break;
                __syncthreads();
            }
            const long long d = s_diff;
            if (d >= 0) c = X[d] > Y[d] ? 1 : -1;
        }
        if (c == 0) {  // exact cancellation
            if (threadIdx.x == 0) {
                Ln.len[2 * Ln.m + i] = 0;
                Ln.sign[i] = 0;
            }
            return;
        }
        swap = c < 0;
        sres = swap ? sy : sx;
    }
    const u32* A = swap ? Y : X;  // the larger magnitude when subtracting
    const u32* B = swap ? X : Y;
    const u64 la = swap ? ly : lx, lb = swap ? lx : ly;
    const u64 n = (la > lb ? la : lb) + (sub ? 0 : 1);
    if (threadIdx.x == 0) {
        s_carry = 0;
        s_top = 0;
    }
    __syncthreads();
    const u64 chunk = (u64)blockDim.x * ADD_LPT;
    for (u64 c0 = 0; c0 < n; c0 += chunk) {
        const u64 base = c0 + (u64)threadIdx.x * ADD_LPT;
        u32 av[ADD_LPT], bv[ADD_LPT];
        GP g{0, 1};
#pragma unroll
        for (int w = 0; w < ADD_LPT; ++w) {
            const u64 k = base + w;
            av[w] = k < la ? A[k] : 0;
            bv[w] = k < lb ? B[k] : 0;
            GP e;
            if (!sub) {
                const u64 s = (u64)av[w] + bv[w];
                e = {(u32)(s >> 32), (u32)((u32)s == 0xFFFFFFFFu)};
            } else {
                e = {(u32)(av[w] < bv[w]), (u32)(av[w] == bv[w])};
            }
            g = gp_then(g, e);
        }
        GP tot;
        const GP ex = block_scan_gp(g, s_ws, &tot);
        const u32 cin_chunk = s_carry;
        u32 c = ex.g | (ex.p & cin_chunk);
        unsigned long long top = 0;
#pragma unroll
        for (int w = 0; w < ADD_LPT; ++w) {
            const u64 k = base + w;
            u32 r;
            if (!sub) {
                const u64 s = (u64)av[w] + bv[w] + c;
                r = (u32)s;
                c = (u32)(s >> 32);
            } else {
                const u64 d = (u64)av[w] - bv[w] - c;
                r = (u32)d;
                c = (u32)((d >> 63) & 1);
            }
            if (k < n) {
                out[k] = r;
                if (r) top = k + 1;
            }
        }
        if (top) atomicMax(&s_top, top);
        __syncthreads();
        if (threadIdx.x == 0) s_carry = tot.g | (tot.p & cin_chunk);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        Ln.len[2 * Ln.m + i] = s_top;
        Ln.sign[i] = s_top ? sres : 0;
    }
}

// Carry the odd last node of L up to the last node of Ln.
__global__ void k_bs_copy_node(LevelView L, u64 src, LevelView Ln, u64 dst) {
    for (int f = 0; f < 3; ++f) {
        const u64 n = L.len[f * L.m + src];
        const u32* s = L.limbs[f] + src * L.stride[f];
        u32* d = Ln.limbs[f] + dst * Ln.stride[f];
        for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (u64)gridDim.x * blockDim.x) d[k] = s[k];
        if (blockIdx.x == 0 && threadIdx.x == 0) Ln.len[f * Ln.m + dst] = n;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) Ln.sign[dst] = L.sign[src];
}

// ---------------------------------------------------------------------------- host driver
struct DevAlloc {
    std::vector<void*> ptrs;
    std::vector<uint64_t> sizes;
};

}  // namespace b2m

using namespace b2m;

struct b2m_pqt {
    Context* ctx = nullptr;
    void* mem = nullptr;  // the root level's allocation
    uint64_t bytes = 0;
    LevelView root{};
    uint64_t host_len[3] = {0, 0, 0};
    int host_sign = 0;
    uint32_t levels = 0;
    uint64_t products = 0;
};

namespace b2m {

static cudaError_t alloc_level(Context* c, uint64_t m, const uint64_t stride[3], LevelView* L, void** mem,
                               uint64_t* bytes, cudaStream_t s) {
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    uint64_t off[3], tot = 0;
    for (int f = 0; f < 3; ++f) {
        off[f] = tot;
        tot += al(m * stride[f] * 4);
    }
    const uint64_t off_len = tot;
    tot += al(3 * m * 8);
    const uint64_t off_sign = tot;
    tot += al(m * 4);
    if (!budget_reserve(c, tot)) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMallocAsync(mem, tot, s);
    if (e != cudaSuccess) {
        budget_release(c, tot);
        return e;
    }
    *bytes = tot;
    unsigned char* b = static_cast<unsigned char*>(*mem);
    L->m = m;
    for (int f = 0; f < 3; ++f) {
        L->stride[f] = stride[f];
        L->limbs[f] = reinterpret_cast<u32*>(b + off[f]);
    }
    L->len = reinterpret_cast<u64*>(b + off_len);
    L->sign = reinterpret_cast<int*>(b + off_sign);
    return cudaSuccess;
}

static cudaError_t level_maxlen(const LevelView& L, unsigned long long* d_tmp, uint64_t out[3], cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(d_tmp, 0, 3 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)std::min<uint64_t>(1024, (L.m + 255) / 256);
    k_bs_maxlen<<<blocks, 256, 0, s>>>(L.len, L.m, d_tmp);
    unsigned long long h[3];
    if ((e = cudaMemcpyAsync(h, d_tmp, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    for (int f = 0; f < 3; ++f) out[f] = h[f];
    return cudaSuccess;
}

static int ceil_log2(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) ++l;
    return l;
}

// One level: L (m nodes, max lengths mx) -> Ln.
// k_bs_signed_add's operation as grid-wide passes driven from the host, for
// levels of a few merges with up to millions of limbs (the top of the tree),
// where one CTA a merge would leave the GPU idle. Reads each merge's lengths
// and signs back, compares |X| and |Y| when it subtracts, and writes T's
// magnitude, length and sign.
constexpr uint64_t BS_GRID_MAX_MERGES = 8;
constexpr uint64_t BS_GRID_MIN_LIMBS = 1 << 15;

static cudaError_t signed_add_grid(Context* c, const ScratchXY& S, const int* sign_l, const LevelView& Ln,
                                   uint64_t m2, uint64_t capT, cudaStream_t s) {
    std::vector<u64> lx(m2), ly(m2);
    std::vector<int> sg(2 * m2);
    cudaError_t e = cudaMemcpyAsync(lx.data(), S.lx, 8 * m2, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ly.data(), S.ly, 8 * m2, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sg.data(), sign_l, sizeof(int) * 2 * m2, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    const uint64_t sb = addsub_scratch_bytes(capT) + 256;
    if (!budget_reserve(c, sb)) return cudaErrorMemoryAllocation;
    void* scratch = nullptr;
    if ((e = cudaMallocAsync(&scratch, sb, s)) != cudaSuccess) {
        budget_release(c, sb);
        return e;
    }
    unsigned long long* word = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(scratch) + sb - 256);
    u32* flag = reinterpret_cast<u32*>(word + 1);
    auto read_word = [&](unsigned long long* h) {
        cudaError_t r = cudaMemcpyAsync(h, word, 8, cudaMemcpyDeviceToHost, s);
        return r == cudaSuccess ? cudaStreamSynchronize(s) : r;
    };
    for (uint64_t i = 0; i < m2 && e == cudaSuccess; ++i) {
        const u32* X = S.x + i * S.sx;
        const u32* Y = S.y + i * S.sy;
        uint64_t la = lx[i], lb = ly[i];
        int sx = la ? sg[2 * i] : 0, sy = lb ? sg[2 * i + 1] : 0;
        u32* out = Ln.limbs[2] + i * Ln.stride[2];
        bool sub = false, swap = false, cancel = false;
        int sres = 0;
        if (sx == 0) {
            sres = sy;
            swap = true;
            la = 0;
        } else if (sy == 0) {
            sres = sx;
            lb = 0;
        } else if (sx == sy) {
            sres = sx;
        } else {
            sub = true;
            int cmpv = 0;
            if (la != lb) {
                cmpv = la > lb ? 1 : -1;
            } else {
                unsigned long long d = 0;
                if ((e = cudaMemsetAsync(word, 0, 8, s)) == cudaSuccess && (e = launch_top_diff(X, Y, la, word, s)) ==
                    cudaSuccess)
                    e = read_word(&d);
                if (e == cudaSuccess && d) {
                    u32 xv = 0, yv = 0;
                    e = cudaMemcpyAsync(&xv, X + d - 1, 4, cudaMemcpyDeviceToHost, s);
                    if (e == cudaSuccess) e = cudaMemcpyAsync(&yv, Y + d - 1, 4, cudaMemcpyDeviceToHost, s);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                    cmpv = xv > yv ? 1 : -1;
                }
            }
            if (cmpv == 0) cancel = true;  // exact cancellation (or an error, reported below)
            swap = cmpv < 0;
            sres = swap ? sy : sx;
        }
        if (e != cudaSuccess) break;
        unsigned long long top = 0;
        if (!cancel) {
            const u32* A = swap ? Y : X;  // the larger magnitude when subtracting
            const u32* B = swap ? X : Y;
            const uint64_t na = swap ? lb : la, nb = swap ? la : lb;
            const uint64_t n = std::max(na, nb) + (sub ? 0 : 1);
            e = launch_addsub(A, na, B, nb, n, sub ? 1 : 0, out, scratch, flag, s);
            if (e == cudaSuccess) e = cudaMemsetAsync(word, 0, 8, s);
            if (e == cudaSuccess) e = launch_top(out, n, word, s);
            if (e == cudaSuccess) e = read_word(&top);
        }
        const u64 len = top;
        const int sign = top ? sres : 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(Ln.len + 2 * Ln.m + i, &len, 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(Ln.sign + i, &sign, sizeof(int), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // len and sign are stack values
    }
    cudaFreeAsync(scratch, s);
    budget_release(c, sb);
    return e;
}

static cudaError_t merge_level(Context* c, const LevelView& L, const uint64_t mx[3], LevelView* Ln, void** mem_n,
                               uint64_t* bytes_n, uint64_t* products, cudaStream_t s) {
    const uint64_t m = L.m, m2 = m / 2, mn = m2 + (m & 1);
    // Length bounds of the products and of T = X +- Y.
    const uint64_t capP = 2 * mx[0], capQ = 2 * mx[1], capX = mx[2] + mx[1], capY = mx[0] + mx[2];
    const uint64_t capT = std::max(capX, capY) + 1;
    const uint64_t stride[3] = {std::max<uint64_t>(capP, mx[0]), std::max<uint64_t>(capQ, mx[1]),
                                std::max<uint64_t>(capT, mx[2])};
    cudaError_t e = alloc_level(c, mn, stride, Ln, mem_n, bytes_n, s);
    if (e != cudaSuccess) return e;
    // Scratch: X, Y and their lengths.
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    const uint64_t xb = al(m2 * capX * 4), yb = al(m2 * capY * 4), lb = al(2 * m2 * 8);
    const uint64_t sbytes = xb + yb + lb;
    void* smem = nullptr;
    if (m2) {
        if (!budget_reserve(c, sbytes)) return cudaErrorMemoryAllocation;
        if ((e = cudaMallocAsync(&smem, sbytes, s)) != cudaSuccess) {
            budget_release(c, sbytes);
            return e;
        }
    }
    ScratchXY S{};
    if (m2) {
        unsigned char* sb = static_cast<unsigned char*>(smem);
        S.x = reinterpret_cast<u32*>(sb);
        S.y = reinterpret_cast<u32*>(sb + xb);
        S.sx = capX;
        S.sy = capY;
        S.lx = reinterpret_cast<u64*>(sb + xb + yb);
        S.ly = S.lx + m2;
    }
    // Operand length bounds per product kind.
    const uint64_t ka[4] = {mx[0], mx[1], mx[2], mx[0]}, kb[4] = {mx[0], mx[1], mx[1], mx[2]};
    const uint64_t cap[4] = {capP, capQ, capX, capY};
    u32 school_mask = 0;
    for (int k = 0; k < 4; ++k)
        if (std::max(ka[k], kb[k]) <= SCHOOL_MAX) school_mask |= 1u << k;
    if (m2 && school_mask) {
        const uint64_t blocks = (4 * m2 + SCHOOL_WARPS - 1) / SCHOOL_WARPS;
        k_bs_school<<<(unsigned)blocks, SCHOOL_WARPS * 32, 0, s>>>(L, *Ln, S, m2, school_mask);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    std::vector<void*> tmp;
    std::vector<uint64_t> tmpb;
    for (int k = 0; k < 4; ++k)
        if (!((school_mask >> k) & 1) && ceil_log2(2 * cap[k]) > MAX_LOGN) return cudaErrorInvalidValue;
    auto kind_plan = [&](int k) {
        int logn = 0, three = 0;
        choose_length(2 * cap[k], &logn, &three);
        return plan_for(c, logn, three);
    };
    // Pairs that share a forward spectrum: Q = QR*QL then X = QR*TL (QR), and
    // P = PL*PR then Y = PL*TR (PL). A shared pair runs both products under
    // the longer of their plans, when its five transforms cost fewer points
    // than the six of two separate products.
    const int order[4] = {1, 2, 0, 3};
    bool pair_share = false;
    Plan pair_plan;
    unsigned char* pair_ws = nullptr;
    uint64_t pair_wss = 0;
    for (int oi = 0; oi < 4 && m2 && e == cudaSuccess; ++oi) {
        const int k = order[oi];
        const bool second = (oi & 1) != 0;
        if (!second) pair_share = false;
        if ((school_mask >> k) & 1) continue;
        Plan p = kind_plan(k);
        bool use_spec = false;
        if (!second) {
            const int partner = order[oi + 1];
            if (!((school_mask >> partner) & 1)) {
                const Plan q = kind_plan(partner);
                const uint64_t n1 = plan_points(p), n2 = plan_points(q), nmax = std::max(n1, n2);
                if (5 * nmax < 3 * (n1 + n2)) {
                    if (n2 > n1) p = q;
                    pair_share = p.npass > 0;
                }
            }
            pair_plan = p;
        } else if (pair_share) {
            p = pair_plan;
            use_spec = true;
        }
        const uint64_t npts = plan_points(p);
        if ((e = twtable_ensure(c, p, s)) != cudaSuccess) break;
        const uint64_t wss = !p.npass ? 0
                             : use_spec ? al(8 * npts + carry_scratch_bytes_n(npts))
                                        : al(workspace_bytes_plan(p));
        const uint64_t tb = al(m2 * sizeof(ProdJob)) + m2 * wss;
        void* t = nullptr;
        if (!budget_reserve(c, tb)) {
            e = cudaErrorMemoryAllocation;
            break;
        }
        if ((e = cudaMallocAsync(&t, tb, s)) != cudaSuccess) {
            budget_release(c, tb);
            break;
        }
        tmp.push_back(t);
        tmpb.push_back(tb);
        ProdJob* jobs = static_cast<ProdJob*>(t);
        unsigned char* ws = wss ? static_cast<unsigned char*>(t) + al(m2 * sizeof(ProdJob)) : nullptr;
        k_bs_build_jobs<<<(unsigned)((m2 + 255) / 256), 256, 0, s>>>(L, *Ln, S, m2, k, jobs, ws, wss, npts,
                                                                    use_spec ? pair_ws : nullptr, pair_wss);
        if (wss) {
            const uint64_t scratch_words = carry_scratch_bytes_n(npts) / 8;
            k_bs_zero_ws<<<(unsigned)m2, 256, 0, s>>>(jobs, m2, scratch_words);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        for (uint64_t off = 0; off < m2 && e == cudaSuccess; off += 65535) {
            const unsigned nj = (unsigned)std::min<uint64_t>(65535, m2 - off);
            e = launch_bucket(p, jobs + off, nj, c->tw, c->d_err, s, use_spec);
        }
        if (!second) {
            pair_ws = ws;  // job i's bufA starts its workspace slot
            pair_wss = wss;
        }
    }
    *products += 4 * m2;
    if (e == cudaSuccess && m2 && m2 <= BS_GRID_MAX_MERGES && capT >= BS_GRID_MIN_LIMBS) {
        e = signed_add_grid(c, S, L.sign, *Ln, m2, capT, s);
    } else if (e == cudaSuccess && m2) {
        const uint64_t maxn = capT;
        unsigned threads = 32;
        while (threads < 1024 && (uint64_t)threads * ADD_LPT < maxn) threads <<= 1;
        k_bs_signed_add<<<(unsigned)m2, threads, 0, s>>>(S, L.sign, *Ln, m2);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && (m & 1)) {
        k_bs_copy_node<<<64, 256, 0, s>>>(L, m - 1, *Ln, mn - 1);
        e = cudaGetLastError();
    }
    for (size_t i = 0; i < tmp.size(); ++i) {
        cudaFreeAsync(tmp[i], s);
        budget_release(c, tmpb[i]);
    }
    if (smem) {
        cudaFreeAsync(smem, s);
        budget_release(c, sbytes);
    }
    return e;
}

// Wraps a finished one-node level into a b2m_pqt (takes ownership of mem).
static b2m_status finish_pqt(Context* c, const LevelView& L, void* mem, uint64_t bytes, uint32_t levels,
                             uint64_t products, cudaStream_t s, b2m_pqt** out) {
    cudaError_t e = cudaStreamSynchronize(s);
    b2m_status st = e == cudaSuccess ? take_device_error(c) : cuda_status(e, "binary splitting");
    u64 hl[3] = {0, 0, 0};
    int hs = 0;
    if (st == B2M_OK) {
        e = cudaMemcpy(hl, L.len, sizeof(hl), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(&hs, L.sign, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_status(e, "cudaMemcpy(pqt lengths)");
    }
    if (st != B2M_OK) {
        cudaFreeAsync(mem, s);
        cudaStreamSynchronize(s);
        budget_release(c, bytes);
        return st;
    }
    b2m_pqt* r = new b2m_pqt();
    r->ctx = c;
    r->mem = mem;
    r->bytes = bytes;
    r->root = L;
    r->levels = levels;
    r->products = products;
    for (int f = 0; f < 3; ++f) r->host_len[f] = hl[f];
    r->host_sign = hs;
    *out = r;
    return B2M_OK;
}

// A level of m nodes filled from device limbs: node i of family f is
// src[i][f] (len[i][f] limbs), signs sg[i]; the rest of each slot is zero.
static cudaError_t level_from(Context* c, int m, const uint32_t* const src[][3], const uint64_t len[][3],
                              const int sg[], LevelView* L, void** mem, uint64_t* bytes, cudaStream_t s) {
    uint64_t stride[3] = {1, 1, 1};
    for (int i = 0; i < m; ++i)
        for (int f = 0; f < 3; ++f) stride[f] = std::max(stride[f], len[i][f]);
    cudaError_t e = alloc_level(c, (uint64_t)m, stride, L, mem, bytes, s);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(*mem, 0, *bytes, s)) != cudaSuccess) return e;
    u64 hl[6];
    for (int i = 0; i < m; ++i)
        for (int f = 0; f < 3; ++f) {
            hl[f * m + i] = len[i][f];
            if (len[i][f] && (e = cudaMemcpyAsync(L->limbs[f] + i * stride[f], src[i][f], len[i][f] * 4,
                                                  cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
                return e;
        }
    if ((e = cudaMemcpyAsync(L->len, hl, 3 * m * sizeof(u64), cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(L->sign, sg, m * sizeof(int), cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
    return cudaStreamSynchronize(s);  // the host arrays above are on this frame
}

}  // namespace b2m

extern "C" {

b2m_status b2m_pqt_import(const uint32_t* const d_limbs[3], const uint64_t len[3], int32_t t_sign,
                          b2m_stream stream, b2m_pqt** result) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (!result || !d_limbs || !len) return B2M_ERR_INVALID_ARGUMENT;
    for (int f = 0; f < 3; ++f)
        if (len[f] && !d_limbs[f]) return B2M_ERR_INVALID_ARGUMENT;
    if (t_sign < -1 || t_sign > 1) return B2M_ERR_INVALID_ARGUMENT;
    *result = nullptr;
    cudaSetDevice(c->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t* src[1][3] = {{d_limbs[0], d_limbs[1], d_limbs[2]}};
    const uint64_t ln[1][3] = {{len[0], len[1], len[2]}};
    const int sg[1] = {t_sign};
    LevelView L{};
    void* mem = nullptr;
    uint64_t bytes = 0;
    cudaError_t e = level_from(c, 1, src, ln, sg, &L, &mem, &bytes, s);
    if (e != cudaSuccess) {
        if (mem) {
            cudaFreeAsync(mem, s);
            cudaStreamSynchronize(s);
            budget_release(c, bytes);
        }
        return cuda_status(e, "b2m_pqt_import");
    }
    return finish_pqt(c, L, mem, bytes, 0, 0, s, result);
}

b2m_status b2m_pqt_merge(const b2m_pqt* left, const b2m_pqt* right, b2m_stream stream, b2m_pqt** result) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (!left || !right || !result) return B2M_ERR_INVALID_ARGUMENT;
    *result = nullptr;
    cudaSetDevice(c->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t* src[2][3];
    uint64_t ln[2][3];
    int sg[2] = {left->host_sign, right->host_sign};
    for (int f = 0; f < 3; ++f) {
        src[0][f] = left->root.limbs[f];
        src[1][f] = right->root.limbs[f];
        ln[0][f] = left->host_len[f];
        ln[1][f] = right->host_len[f];
    }
    LevelView L{};
    void* mem = nullptr;
    uint64_t bytes = 0;
    cudaError_t e = level_from(c, 2, src, ln, sg, &L, &mem, &bytes, s);
    LevelView Ln{};
    void* mem_n = nullptr;
    uint64_t bytes_n = 0, products = left->products + right->products;
    if (e == cudaSuccess) {
        const uint64_t mx[3] = {std::max(ln[0][0], ln[1][0]), std::max(ln[0][1], ln[1][1]),
                                std::max(ln[0][2], ln[1][2])};
        e = merge_level(c, L, mx, &Ln, &mem_n, &bytes_n, &products, s);
    }
    if (mem) {
        cudaFreeAsync(mem, s);
        budget_release(c, bytes);
    }
    if (e != cudaSuccess) {
        if (mem_n) {
            cudaFreeAsync(mem_n, s);
            budget_release(c, bytes_n);
        }
        cudaStreamSynchronize(s);
        return cuda_status(e, "b2m_pqt_merge");
    }
    return finish_pqt(c, Ln, mem_n, bytes_n, std::max(left->levels, right->levels) + 1, products, s, result);
}

b2m_status b2m_chudnovsky_bs(uint64_t a, uint64_t b, b2m_stream stream, b2m_pqt** out) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (!out || b <= a) return B2M_ERR_INVALID_ARGUMENT;
    if (b > BS_MAX_TERMS) {
        set_error("b2m_chudnovsky_bs supports term indices below 2,000,000 (about 28 million digits)");
        return B2M_ERR_TOO_LARGE;
    }
    *out = nullptr;
    cudaSetDevice(c->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned long long* d_tmp = nullptr;
    cudaError_t e = cudaMallocAsync(&d_tmp, 64, s);
    if (e != cudaSuccess) return cuda_status(e, "cudaMallocAsync");
    uint64_t products = 0;
    const uint64_t stride0[3] = {4, 4, 4};
    LevelView L{};
    void* mem = nullptr;
    uint64_t bytes = 0;
    e = alloc_level(c, b - a, stride0, &L, &mem, &bytes, s);
    uint64_t mx[3] = {0, 0, 0};
    if (e == cudaSuccess) {
        k_bs_leaves<<<(unsigned)((L.m + 255) / 256), 256, 0, s>>>(a, L);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = level_maxlen(L, d_tmp, mx, s);
    uint32_t levels = 0;
    while (e == cudaSuccess && L.m > 1) {
        LevelView Ln{};
        void* mem_n = nullptr;
        uint64_t bytes_n = 0;
        e = merge_level(c, L, mx, &Ln, &mem_n, &bytes_n, &products, s);
        if (e == cudaSuccess) e = level_maxlen(Ln, d_tmp, mx, s);
        if (mem) {
            cudaFreeAsync(mem, s);
            budget_release(c, bytes);
        }
        L = Ln;
        mem = mem_n;
        bytes = bytes_n;
        ++levels;
    }
    cudaFreeAsync(d_tmp, s);
    if (e != cudaSuccess) {
        if (mem) {
            cudaFreeAsync(mem, s);
            cudaStreamSynchronize(s);
            budget_release(c, bytes);
        }
        return cuda_status(e, "binary splitting");
    }
    return finish_pqt(c, L, mem, bytes, levels, products, s, out);
}

b2m_status b2m_pqt_info(const b2m_pqt* r, uint64_t len[3], int32_t* t_sign, uint32_t* levels, uint64_t* products) {
    if (!r) return B2M_ERR_INVALID_ARGUMENT;
    if (len)
        for (int f = 0; f < 3; ++f) len[f] = r->host_len[f];
    if (t_sign) *t_sign = r->host_sign;
    if (levels) *levels = r->levels;
    if (products) *products = r->products;
    return B2M_OK;
}

const uint32_t* b2m_pqt_device(const b2m_pqt* r, int which) {
    if (!r || which < 0 || which > 2) return nullptr;
    return r->root.limbs[which];
}

b2m_status b2m_pqt_copy(const b2m_pqt* r, int which, uint32_t* host, uint64_t cap) {
    if (!r || which < 0 || which > 2 || (!host && r->host_len[which])) return B2M_ERR_INVALID_ARGUMENT;
    if (cap < r->host_len[which]) return B2M_ERR_OUTPUT_TOO_SMALL;
    cudaSetDevice(r->ctx->device);
    return cuda_status(cudaMemcpy(host, r->root.limbs[which], r->host_len[which] * 4, cudaMemcpyDeviceToHost),
                       "cudaMemcpy(pqt)");
}

b2m_status b2m_pqt_free(b2m_pqt* r) {
    if (!r) return B2M_OK;
    cudaSetDevice(r->ctx->device);
    cudaDeviceSynchronize();
    if (r->mem) {
        cudaFreeAsync(r->mem, 0);  // pool allocation: free in stream order, then wait
        cudaStreamSynchronize(0);
        budget_release(r->ctx, r->bytes);
    }
    delete r;
    return B2M_OK;
}

}  // extern "C"
