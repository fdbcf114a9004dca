// b2m_bigops.cu -- big-integer arithmetic on device-resident magnitudes, built
// on the NTT product: add / subtract with parallel carries, shifts, a Newton
// reciprocal, exact floor division, integer square root, and decimal
// conversion by divide and conquer with each level's divisions batched.
//
// Reference counterparts: divmod_knuth / div_fast (src/bignum_div.cpp:162-178),
// isqrt (src/bignum_div.cpp:189-204) and BigInt::to_decimal
// (src/bignum_div.cpp:239-267). Those are quadratic (schoolbook division, a
// Newton square root whose every step is a schoolbook division, repeated
// division by 10^9); these cost a few NTT products of the operand size each
// (O(M(n)) division and square root, O(M(n) log n) decimal conversion), and
// return the same integers: every result is exact, not approximate -- the
// Newton iterates only seed a quotient or root that a bounded correction loop
// then makes exact against the definition (remainder in [0, b), root with
// s^2 <= a < (s+1)^2).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "b2m.h"
#include "b2m_context.h"
#include "b2m_internal.h"
#include "gp_scan.cuh"

namespace b2m {
namespace big {

struct Err {
    b2m_status st;
};

// A device magnitude: n little-endian u32 limbs at p (n == 0 is zero).
struct DV {
    u32* p = nullptr;
    uint64_t n = 0;
};

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Err{cuda_status(e, what)};
}

// Stream-ordered allocations of one API call, released when it returns.
class Scope {
public:
    Scope(Context* c, cudaStream_t s) : c_(c), s_(s) { w_ = static_cast<unsigned long long*>(raw(64)); }
    ~Scope() {
        for (auto& a : v_) {
            cudaFreeAsync(a.first, s_);
            budget_release(c_, a.second);
        }
    }
    Scope(const Scope&) = delete;
    Scope& operator=(const Scope&) = delete;
    void* raw(uint64_t bytes) {
        bytes = (std::max<uint64_t>(bytes, 16) + 255) & ~255ull;
        if (!budget_reserve(c_, bytes)) {
            set_error("HBM budget exhausted");
            throw Err{B2M_ERR_OUT_OF_MEMORY};
        }
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, bytes, s_);
        if (e != cudaSuccess) {
            budget_release(c_, bytes);
            throw Err{cuda_status(e, "cudaMallocAsync")};
        }
        v_.push_back({p, bytes});
        return p;
    }
    DV vec(uint64_t n) { return {static_cast<u32*>(raw(4 * std::max<uint64_t>(n, 1))), n}; }
    DV zeros(uint64_t n) {
        DV d = vec(n);
        ck(cudaMemsetAsync(d.p, 0, 4 * std::max<uint64_t>(n, 1), s_), "cudaMemsetAsync");
        return d;
    }
    cudaStream_t s() const { return s_; }
    Context* c() const { return c_; }
    unsigned long long* word() const { return w_; }  // 64 bytes of device scratch

private:
    Context* c_;
    cudaStream_t s_;
    unsigned long long* w_ = nullptr;
    std::vector<std::pair<void*, uint64_t>> v_;
};

// ---------------------------------------------------------------------------- kernels
__global__ void k_top(const u32* __restrict__ a, u64 n, unsigned long long* out) {
    unsigned long long t = 0;
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (u64)gridDim.x * blockDim.x)
        if (a[k]) t = k + 1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, t, off);
        t = o > t ? o : t;
    }
    if ((threadIdx.x & 31) == 0 && t) atomicMax(out, t);
}

constexpr int AS_T = 256, AS_L = ADD_LPT, AS_CH = AS_T * AS_L;  // limbs per block

__device__ __forceinline__ GP limb_gp(u32 a, u32 b, int sub) {
    if (!sub) {
        const u64 s = (u64)a + b;
        return {(u32)(s >> 32), (u32)((u32)s == 0xFFFFFFFFu)};
    }
    return {(u32)(a < b), (u32)(a == b)};
}

// Carry / borrow (generate, propagate) of each block's limbs.
__global__ void __launch_bounds__(AS_T) k_as_reduce(const u32* __restrict__ A, u64 la, const u32* __restrict__ B,
                                                    u64 lb, u64 n, int sub, GP* __restrict__ agg) {
    __shared__ GP ws[AS_T / 32 + 1];
    const u64 base = (u64)blockIdx.x * AS_CH + (u64)threadIdx.x * AS_L;
    GP g{0, 1};
#pragma unroll
    for (int w = 0; w < AS_L; ++w) {
        const u64 k = base + w;
        if (k < n) g = gp_then(g, limb_gp(k < la ? A[k] : 0u, k < lb ? B[k] : 0u, sub));
    }
    GP tot;
    block_scan_gp(g, ws, &tot);
    if (threadIdx.x == 0) agg[blockIdx.x] = tot;
}

// Carry into each block (all blocks' aggregates scanned in one CTA), and the
// carry out of the top limb.
__global__ void __launch_bounds__(1024) k_as_scan(const GP* __restrict__ agg, u64 nb, u32* __restrict__ cin,
                                                  u32* __restrict__ cout) {
    __shared__ GP ws[33];
    GP acc{0, 1};
    for (u64 c0 = 0; c0 < nb; c0 += blockDim.x) {
        const u64 i = c0 + threadIdx.x;
        GP tot;
        const GP ex = block_scan_gp(i < nb ? agg[i] : GP{0, 1}, ws, &tot);
        if (i < nb) cin[i] = gp_then(acc, ex).g;
        acc = gp_then(acc, tot);
        __syncthreads();
    }
    if (threadIdx.x == 0) *cout = acc.g;
}

// out = A +- B (mod 2^(32n)); out may be A or B (each limb is read before it
// is written, by the same thread).
__global__ void __launch_bounds__(AS_T) k_as_apply(const u32* A, u64 la, const u32* B, u64 lb, u64 n, int sub,
                                                   const u32* __restrict__ cin, u32* out) {
    __shared__ GP ws[AS_T / 32 + 1];
    const u64 base = (u64)blockIdx.x * AS_CH + (u64)threadIdx.x * AS_L;
    u32 av[AS_L], bv[AS_L];
    GP g{0, 1};
#pragma unroll
    for (int w = 0; w < AS_L; ++w) {
        const u64 k = base + w;
        av[w] = k < la && k < n ? A[k] : 0u;
        bv[w] = k < lb && k < n ? B[k] : 0u;
        if (k < n) g = gp_then(g, limb_gp(av[w], bv[w], sub));
    }
    GP tot;
    const GP ex = block_scan_gp(g, ws, &tot);
    u32 c = ex.g | (ex.p & cin[blockIdx.x]);
#pragma unroll
    for (int w = 0; w < AS_L; ++w) {
        const u64 k = base + w;
        if (k >= n) break;
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
        out[k] = r;
    }
}

// out[k] = (a * 2^(32*wl + bits))[k], k < nout (bits in [0, 32)).
__global__ void k_shl(const u32* __restrict__ a, u64 na, int bits, u64 wl, u32* __restrict__ out, u64 nout) {
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < nout; k += (u64)gridDim.x * blockDim.x) {
        u32 v = 0;
        if (k >= wl && k - wl < na) v = a[k - wl] << bits;
        if (bits && k >= wl + 1 && k - wl - 1 < na) v |= a[k - wl - 1] >> (32 - bits);
        out[k] = v;
    }
}

// out[k] = floor(a / 2^(32*wl + bits))[k], k < nout (bits in [0, 32)).
__global__ void k_shr(const u32* __restrict__ a, u64 na, int bits, u64 wl, u32* __restrict__ out, u64 nout) {
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < nout; k += (u64)gridDim.x * blockDim.x) {
        u32 v = 0;
        if (k + wl < na) v = a[k + wl] >> bits;
        if (bits && k + wl + 1 < na) v |= a[k + wl + 1] << (32 - bits);
        out[k] = v;
    }
}

inline unsigned grid_for(uint64_t n, unsigned threads = 256) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + threads - 1) / threads, 65535));
}

// ---------------------------------------------------------------------------- host ops
uint64_t top_len(Scope& S, DV a) {
    if (a.n == 0) return 0;
    ck(cudaMemsetAsync(S.word(), 0, 8, S.s()), "cudaMemsetAsync");
    k_top<<<grid_for(a.n), 256, 0, S.s()>>>(a.p, a.n, S.word());
    ck(cudaGetLastError(), "k_top");
    unsigned long long h = 0;
    ck(cudaMemcpyAsync(&h, S.word(), 8, cudaMemcpyDeviceToHost, S.s()), "cudaMemcpyAsync");
    ck(cudaStreamSynchronize(S.s()), "cudaStreamSynchronize");
    return h;
}

DV trim(Scope& S, DV a) { return {a.p, top_len(S, a)}; }

// out = a +- b mod 2^(32 out.n); returns the carry (add) or borrow (sub) out.
u32 addsub(Scope& S, DV a, DV b, DV out, bool sub) {
    const uint64_t n = out.n;
    if (n == 0) return 0;
    const uint64_t nb = (n + AS_CH - 1) / AS_CH;
    GP* agg = static_cast<GP*>(S.raw(nb * sizeof(GP)));
    u32* cin = static_cast<u32*>(S.raw(nb * 4));
    u32* cout = reinterpret_cast<u32*>(S.word() + 1);
    k_as_reduce<<<(unsigned)nb, AS_T, 0, S.s()>>>(a.p, a.n, b.p, b.n, n, sub, agg);
    k_as_scan<<<1, 1024, 0, S.s()>>>(agg, nb, cin, cout);
    k_as_apply<<<(unsigned)nb, AS_T, 0, S.s()>>>(a.p, a.n, b.p, b.n, n, sub, cin, out.p);
    ck(cudaGetLastError(), "add/subtract kernels");
    u32 h = 0;
    ck(cudaMemcpyAsync(&h, cout, 4, cudaMemcpyDeviceToHost, S.s()), "cudaMemcpyAsync");
    ck(cudaStreamSynchronize(S.s()), "cudaStreamSynchronize");
    return h;
}

DV upload(Scope& S, const std::vector<u32>& h) {
    DV d = S.vec(h.size());
    if (!h.empty()) ck(cudaMemcpyAsync(d.p, h.data(), 4 * h.size(), cudaMemcpyHostToDevice, S.s()), "H2D");
    ck(cudaStreamSynchronize(S.s()), "cudaStreamSynchronize");  // h may be a temporary
    return d;
}

std::vector<u32> download(Scope& S, DV d) {
    std::vector<u32> h(d.n);
    if (d.n) ck(cudaMemcpyAsync(h.data(), d.p, 4 * d.n, cudaMemcpyDeviceToHost, S.s()), "D2H");
    ck(cudaStreamSynchronize(S.s()), "cudaStreamSynchronize");
    return h;
}

u32 limb_at(Scope& S, DV d, uint64_t k) {
    u32 h = 0;
    ck(cudaMemcpyAsync(&h, d.p + k, 4, cudaMemcpyDeviceToHost, S.s()), "D2H");
    ck(cudaStreamSynchronize(S.s()), "cudaStreamSynchronize");
    return h;
}

DV copy(Scope& S, DV a, uint64_t cap) {
    DV d = S.zeros(std::max(cap, a.n));
    if (a.n) ck(cudaMemcpyAsync(d.p, a.p, 4 * a.n, cudaMemcpyDeviceToDevice, S.s()), "D2D");
    d.n = a.n;
    return d;
}

// a * 2^(32 wl + bits), trimmed.
DV shl(Scope& S, DV a, uint64_t wl, int bits) {
    if (a.n == 0) return a;
    const uint64_t n = a.n + wl + 1;
    DV d = S.vec(n);
    k_shl<<<grid_for(n), 256, 0, S.s()>>>(a.p, a.n, bits, wl, d.p, n);
    ck(cudaGetLastError(), "k_shl");
    return trim(S, d);
}

// floor(a / 2^(32 wl + bits)), trimmed.
DV shr(Scope& S, DV a, uint64_t wl, int bits) {
    if (a.n <= wl) return {a.p, 0};
    const uint64_t n = a.n - wl;
    DV d = S.vec(n);
    k_shr<<<grid_for(n), 256, 0, S.s()>>>(a.p, a.n, bits, wl, d.p, n);
    ck(cudaGetLastError(), "k_shr");
    return trim(S, d);
}

// a + delta for delta in {-1, +1} (a + 1 may grow by one limb; a - 1 needs a > 0).
DV add_one(Scope& S, DV a, bool minus) {
    static const u32 one_h = 1;
    DV one = S.vec(1);
    ck(cudaMemcpyAsync(one.p, &one_h, 4, cudaMemcpyHostToDevice, S.s()), "H2D");
    DV d = S.vec(a.n + 1);
    addsub(S, a, one, d, minus);
    return trim(S, d);
}

// The NTT product, trimmed.
DV mul(Scope& S, DV a, DV b) {
    if (a.n == 0 || b.n == 0) return {a.p ? a.p : b.p, 0};
    int logn = 0;
    const b2m_status st = check_sizes(a.n, b.n, &logn);
    if (st != B2M_OK) throw Err{st};
    Context* c = S.c();
    const Plan p = product_plan(c, a.n, b.n);
    ck(twtable_ensure(c, p, S.s()), "twiddle table");
    DV out = S.vec(a.n + b.n);
    void* ws = p.npass ? S.raw(workspace_bytes_plan(p)) : nullptr;
    uint64_t* d_len = reinterpret_cast<uint64_t*>(S.word() + 2);
    ck(launch_product(a.p, a.n, b.p, b.n, out.p, d_len, ws, p, c->tw, c->d_err, S.s()), "product");
    unsigned long long h = 0;
    ck(cudaMemcpyAsync(&h, d_len, 8, cudaMemcpyDeviceToHost, S.s()), "D2H");
    ck(cudaStreamSynchronize(S.s()), "cudaStreamSynchronize");
    out.n = h;  // the sticky device error word is checked once, when the call ends
    return out;
}

// ---------------------------------------------------------------------------- small host arithmetic
// floor((2^(64h) - 1) / Y) for an h-limb Y whose top bit is set: schoolbook
// long division on 32-bit digits (Knuth, TAOCP vol. 2, 4.3.1, algorithm D),
// the numerator being 2h all-ones limbs. Seeds the Newton reciprocal.
std::vector<u32> recip_small(const std::vector<u32>& Y) {
    const size_t n = Y.size();
    std::vector<u32> q(n + 1, 0);
    if (n == 1) {
        const u64 v = ~0ull / Y[0];
        q[0] = (u32)v;
        q[1] = (u32)(v >> 32);
    } else {
        std::vector<u32> un(2 * n + 1, 0xFFFFFFFFu);
        un[2 * n] = 0;
        const u64 b = 1ull << 32;
        for (long j = (long)n; j >= 0; --j) {
            const u64 num = ((u64)un[j + n] << 32) | un[j + n - 1];
            u64 qhat = num / Y[n - 1], rhat = num % Y[n - 1];
            while (qhat >= b || qhat * Y[n - 2] > ((rhat << 32) | un[j + n - 2])) {
                --qhat;
                rhat += Y[n - 1];
                if (rhat >= b) break;
            }
            int64_t k = 0, t;
            for (size_t i = 0; i < n; ++i) {
                const u64 p = qhat * Y[i];
                t = (int64_t)un[i + j] - k - (int64_t)(p & 0xFFFFFFFFull);
                un[i + j] = (u32)t;
                k = (int64_t)(p >> 32) - (t >> 32);
            }
            t = (int64_t)un[j + n] - k;
            un[j + n] = (u32)t;
            if (t < 0) {
                --qhat;
                u64 c = 0;
                for (size_t i = 0; i < n; ++i) {
                    const u64 s = (u64)un[i + j] + Y[i] + c;
                    un[i + j] = (u32)s;
                    c = s >> 32;
                }
                un[j + n] += (u32)c;
            }
            q[j] = (u32)qhat;
        }
    }
    while (!q.empty() && q.back() == 0) q.pop_back();
    return q;
}
// floor(sqrt(v)) for v < 2^128 (bit by bit).
unsigned __int128 isqrt128(unsigned __int128 v) {
    unsigned __int128 res = 0, bit = (unsigned __int128)1 << 126;
    while (bit > v) bit >>= 2;
    while (bit) {
        if (v >= res + bit) {
            v -= res + bit;
            res = (res >> 1) + bit;
        } else {
            res >>= 1;
        }
        bit >>= 2;
    }
    return res;
}

std::vector<u32> from128(unsigned __int128 v) {
    std::vector<u32> h;
    while (v) {
        h.push_back((u32)v);
        v >>= 32;
    }
    return h;
}

unsigned __int128 to128(const std::vector<u32>& h) {
    unsigned __int128 v = 0;
    for (size_t i = h.size(); i-- > 0;) v = (v << 32) | h[i];
    return v;
}

// ---------------------------------------------------------------------------- Newton reciprocal
// Top h limbs of the normalized Bn (n limbs), or Bn * 2^(32(h - n)) if h > n.
DV top_limbs(Scope& S, DV Bn, uint64_t h) {
    if (h <= Bn.n) return {Bn.p + (Bn.n - h), h};
    DV d = S.zeros(h);
    ck(cudaMemcpyAsync(d.p + (h - Bn.n), Bn.p, 4 * Bn.n, cudaMemcpyDeviceToDevice, S.s()), "D2D");
    return d;
}

// X ~ 2^(64h) / Y_h, Y_h = top_limbs(Bn, h) (top bit set), within a few units:
// X_h = X_l 2^(32(h-l)) + X_l (2^(32(h+l)) - Y_h X_l) / 2^(64 l), with the
// lower precision l = floor((h + 3) / 2) seeding each step (Newton doubles
// the correct limbs; the +3 keeps a guard limb).
DV recip(Scope& S, DV Bn, uint64_t h) {
    DV Y = top_limbs(S, Bn, h);
    if (h <= 32) return trim(S, upload(S, recip_small(download(S, Y))));
    const uint64_t l = (h + 3) / 2;
    DV Xl = recip(S, Bn, l);
    DV T = mul(S, Y, Xl);
    const uint64_t e = h + l;
    DV E;
    bool neg = false;
    if (T.n <= e) {  // E = 2^(32e) - T >= 0
        E = S.vec(e);
        addsub(S, DV{T.p, 0}, T, E, true);
    } else {  // T = 2^(32e) + E', 0 <= E' < 2^(32e)
        if (T.n != e + 1 || limb_at(S, T, e) != 1) {
            set_error("Newton reciprocal diverged");
            throw Err{B2M_ERR_INTERNAL};
        }
        E = {T.p, e};
        neg = true;
    }
    E = trim(S, E);
    DV D = mul(S, Xl, E);
    DV corr = D.n > 2 * l ? DV{D.p + 2 * l, D.n - 2 * l} : DV{D.p, 0};
    DV Xs = S.zeros(h + 2);
    ck(cudaMemcpyAsync(Xs.p + (h - l), Xl.p, 4 * Xl.n, cudaMemcpyDeviceToDevice, S.s()), "D2D");
    DV X = S.vec(h + 2);
    addsub(S, Xs, corr, X, neg);
    return trim(S, X);
}

// ---------------------------------------------------------------------------- division
constexpr int MAX_FIX = 16;  // correction steps allowed after a Newton estimate

// q = floor(a / b), r = a mod b for trimmed a, b (b > 0). The estimate
// q~ = floor(top(a') X / 2^(32 s)) from the reciprocal of the normalized
// divisor is within a few units; r = a - q~ b then moves q~ to the exact
// quotient one unit at a time.
void divmod(Scope& S, DV a, DV b, DV* q, DV* r) {
    if (b.n == 0) {
        set_error("division by zero");
        throw Err{B2M_ERR_INVALID_ARGUMENT};
    }
    if (a.n < b.n) {
        *q = {a.p, 0};
        *r = a;
        return;
    }
    const int sh = __builtin_clz(limb_at(S, b, b.n - 1));
    DV Bn = sh ? shl(S, b, 0, sh) : b;
    DV An = sh ? shl(S, a, 0, sh) : a;
    const uint64_t n = b.n;
    const uint64_t m = An.n - n + 1;  // quotient limbs, at most
    const uint64_t L = m + 2;
    DV X = recip(S, Bn, L);          // ~ 2^(32(L + n)) / Bn
    const uint64_t k = An.n > L + 1 ? An.n - (L + 1) : 0;
    DV P = mul(S, DV{An.p + k, An.n - k}, X);
    const uint64_t s = L + n - k;
    DV Q = copy(S, P.n > s ? DV{P.p + s, P.n - s} : DV{P.p, 0}, m + 2);
    Q = trim(S, Q);
    DV QB = mul(S, Q, b);
    const uint64_t w = std::max(a.n, QB.n) + 1;
    DV R = S.vec(w);
    bool negative = addsub(S, a, QB, R, true) != 0;
    int it = 0;
    while (negative) {  // two's complement R < 0: add b back
        if (addsub(S, R, b, R, false)) negative = false;
        Q = add_one(S, Q, true);
        if (++it > MAX_FIX) break;
    }
    while (it <= MAX_FIX) {  // R >= b: subtract it
        DV T = S.vec(w);
        if (addsub(S, R, b, T, true)) break;
        R = T;
        Q = add_one(S, Q, false);
        ++it;
    }
    if (it > MAX_FIX) {
        set_error("division correction did not converge");
        throw Err{B2M_ERR_INTERNAL};
    }
    *q = Q;
    *r = trim(S, R);
}

// ---------------------------------------------------------------------------- square root
// ~ sqrt(floor(N / 2^(32(2k - 2h)))) to h limbs (N has at most 2k limbs):
// one Newton step x = (x0 + floor(N_h / x0)) / 2 from the root of the top
// 2l limbs, l = floor((h + 2) / 2).
DV sqrt_approx(Scope& S, DV N, uint64_t k, uint64_t h) {
    const uint64_t drop = 2 * k - 2 * h;
    DV Nh = N.n > drop ? DV{N.p + drop, N.n - drop} : DV{N.p, 0};
    if (h <= 2) {
        std::vector<u32> v = download(S, Nh);
        return trim(S, upload(S, from128(isqrt128(to128(v)))));
    }
    const uint64_t l = (h + 2) / 2;
    DV xl = sqrt_approx(S, N, k, l);
    DV x0 = shl(S, xl, h - l, 0);
    if (x0.n == 0) return x0;
    DV qv, rv;
    divmod(S, Nh, x0, &qv, &rv);
    DV s = S.vec(std::max(x0.n, qv.n) + 1);
    addsub(S, x0, qv, s, false);
    return shr(S, trim(S, s), 0, 1);
}

DV isqrt(Scope& S, DV N);

// Y ~ 2^(64h) / sqrt(N_h), N_h = floor(N / 2^(32(2k - 2h))), by Newton on the
// reciprocal square root, y <- y + y (1 - N y^2) / 2: three products a step
// and no division. The seed (h <= 8) is floor((2^(64h) - 1) / isqrt(N_h))
// from the exact root; each step starts from l = floor((h + 3) / 2) limbs.
DV rsqrt_approx(Scope& S, DV N, uint64_t k, uint64_t h) {
    const uint64_t drop = 2 * k - 2 * h;
    DV Nh = N.n > drop ? DV{N.p + drop, N.n - drop} : DV{N.p, 0};
    if (h <= 8) {
        DV root = isqrt(S, Nh);
        DV num = S.vec(2 * h);
        ck(cudaMemsetAsync(num.p, 0xFF, 8 * h, S.s()), "cudaMemsetAsync");  // 2^(64h) - 1
        DV q, r;
        divmod(S, num, root, &q, &r);
        return q;
    }
    const uint64_t l = (h + 3) / 2;
    DV Y0 = shl(S, rsqrt_approx(S, N, k, l), h - l, 0);
    DV U = mul(S, Nh, mul(S, Y0, Y0));  // ~ 2^(128h)
    const uint64_t e = 4 * h;
    DV E;
    bool neg = false;
    if (U.n <= e) {  // E = 2^(32e) - U >= 0
        E = S.vec(e);
        addsub(S, DV{U.p, 0}, U, E, true);
    } else {  // U = 2^(32e) + E'
        if (U.n != e + 1 || limb_at(S, U, e) != 1) {
            set_error("Newton reciprocal square root diverged");
            throw Err{B2M_ERR_INTERNAL};
        }
        E = {U.p, e};
        neg = true;
    }
    DV corr = shr(S, mul(S, Y0, trim(S, E)), e, 1);  // Y0 |E| / 2^(32e + 1)
    DV Y = S.vec(std::max(Y0.n, corr.n) + 1);
    addsub(S, Y0, corr, Y, neg);
    return trim(S, Y);
}

// floor(sqrt(N)) for trimmed N: an estimate -- N * Y / 2^(64k) from the
// reciprocal square root above, or for small N the division-based Newton
// root -- then the remainder R = N - s^2 moves s until 0 <= R <= 2s.
DV isqrt(Scope& S, DV N) {
    if (N.n == 0) return N;
    if (N.n <= 4) return trim(S, upload(S, from128(isqrt128(to128(download(S, N))))));
    const uint64_t k = (N.n + 1) / 2;
    DV s;
    if (N.n <= 16) {
        s = sqrt_approx(S, N, k, k);
    } else {
        DV Y = rsqrt_approx(S, N, k, k);
        s = shr(S, mul(S, N, Y), 2 * k, 0);
    }
    DV SQ = mul(S, s, s);
    const uint64_t w = std::max(N.n, SQ.n) + 2;
    DV R = S.vec(w);
    bool negative = addsub(S, N, SQ, R, true) != 0;
    int it = 0;
    while (negative && it <= MAX_FIX) {  // N - (s-1)^2 = R + 2s - 1
        DV twice = shl(S, s, 0, 1);
        DV d = add_one(S, twice, true);
        if (addsub(S, R, d, R, false)) negative = false;
        s = add_one(S, s, true);
        ++it;
    }
    while (it <= MAX_FIX) {  // N - (s+1)^2 = R - (2s + 1)
        DV d = add_one(S, shl(S, s, 0, 1), false);
        DV T = S.vec(w);
        if (addsub(S, R, d, T, true)) break;
        R = T;
        s = add_one(S, s, false);
        ++it;
    }
    if (it > MAX_FIX) {
        set_error("square-root correction did not converge");
        throw Err{B2M_ERR_INTERNAL};
    }
    return s;
}

// ---------------------------------------------------------------------------- decimal conversion
// Divide and conquer with powers P_j = 10^(9 * 2^j): a node of level j holds
// a value below P_j^2; dividing it by P_j gives two nodes below P_j (quotient
// first: the more significant digits). All nodes of a level have the same
// size and divisor, so each level is two batched products (the quotient
// estimate from P_j's reciprocal, then estimate * P_j) and one kernel that
// makes every quotient and remainder exact. Nodes below 10^72 are printed by
// one thread each.

constexpr int DC_LEAF_J = 2;     // leaves: values below P_2^2 = 10^72
constexpr int DC_LEAF_LIMBS = 8;  // 10^72 < 2^240
constexpr int DC_LEAF_GROUPS = 8;

// Job i multiplies a + i*sa by b + i*sb. With `spec` (b shared, sb = 0, its
// spectrum already in spec), b becomes every job's first operand with bufA =
// spec, and the workspace holds only bufB and the carry scratch.
__global__ void k_dc_jobs(const u32* a, u64 sa, u64 na, const u32* b, u64 sb, u64 nb, u32* out, u64 so,
                          unsigned long long* lens, ProdJob* jobs, u64 njobs, unsigned char* ws, u64 wss, u64 npts,
                          u64* spec) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= njobs) return;
    ProdJob J{};
    J.a = a + i * sa;
    J.na = na;
    J.b = b + i * sb;
    J.nb = nb;
    if (spec) {
        J.a = b;
        J.na = nb;
        J.b = a + i * sa;
        J.nb = na;
    }
    J.out = out + i * so;
    J.out_len = lens + i;
    if (wss) {
        const u64 n = npts;
        unsigned char* w = ws + i * wss;
        unsigned char* scratch;
        if (spec) {
            J.bufA = spec;
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

// The one-job table that transforms b into spec.
__global__ void k_dc_spec_job(const u32* b, u64 nb, u64* spec, ProdJob* job) {
    ProdJob J{};
    J.a = b;
    J.na = nb;
    J.bufA = spec;
    *job = J;
}

__global__ void k_dc_zero_ws(const ProdJob* __restrict__ jobs, u64 njobs, u64 scratch_words) {
    const u64 j = blockIdx.x;
    if (j >= njobs) return;
    unsigned long long* s = reinterpret_cast<unsigned long long*>(jobs[j].slots);
    for (u64 i = threadIdx.x; i < scratch_words; i += blockDim.x) s[i] = 0;
    if (threadIdx.x == 0) *jobs[j].out_len = 0;
}

// out_i = a_i * b_i for m products of na x nb limbs (strides sa, sb, so; sb = 0
// shares one b), as size-bucketed launches of the batch path. A shared b is
// transformed once and its spectrum read by every product (two transforms a
// product instead of three).
void batched_mul(Scope& S, const u32* a, uint64_t sa, uint64_t na, const u32* b, uint64_t sb, uint64_t nb, u32* out,
                 uint64_t so, uint64_t m) {
    if (m == 0) return;
    int logn = 0;
    const b2m_status st = check_sizes(na, nb, &logn);
    if (st != B2M_OK) throw Err{st};
    Context* c = S.c();
    const Plan p = product_plan(c, na, nb);
    ck(twtable_ensure(c, p, S.s()), "twiddle table");
    const uint64_t npts = plan_points(p);
    u64* spec = nullptr;
    if (sb == 0 && m > 1 && p.npass > 0) {
        spec = static_cast<u64*>(S.raw(8 * npts));
        ProdJob* sj = static_cast<ProdJob*>(S.raw(sizeof(ProdJob)));
        k_dc_spec_job<<<1, 1, 0, S.s()>>>(b, nb, spec, sj);
        ck(cudaGetLastError(), "spectrum job");
        ck(launch_bucket_spectrum(p, sj, 1, c->tw, S.s()), "shared spectrum");
    }
    const uint64_t wss = !p.npass ? 0
                         : spec   ? ((8 * npts + carry_scratch_bytes_n(npts) + 255) & ~255ull)
                                  : ((workspace_bytes_plan(p) + 255) & ~255ull);
    // at most 65535 jobs a launch, and at most ~1 GiB of transform workspace
    uint64_t chunk = 65535;
    if (wss) chunk = std::max<uint64_t>(1, std::min<uint64_t>(chunk, (1ull << 30) / wss));
    for (uint64_t off = 0; off < m; off += chunk) {
        const uint64_t nj = std::min(chunk, m - off);
        ProdJob* jobs = static_cast<ProdJob*>(S.raw(nj * sizeof(ProdJob)));
        unsigned long long* lens = static_cast<unsigned long long*>(S.raw(nj * 8));
        unsigned char* ws = wss ? static_cast<unsigned char*>(S.raw(nj * wss)) : nullptr;
        k_dc_jobs<<<(unsigned)((nj + 255) / 256), 256, 0, S.s()>>>(a + off * sa, sa, na, b + off * sb, sb, nb,
                                                                  out + off * so, so, lens, jobs, nj, ws, wss, npts,
                                                                  spec);
        if (wss) k_dc_zero_ws<<<(unsigned)nj, 256, 0, S.s()>>>(jobs, nj, carry_scratch_bytes_n(npts) / 8);
        ck(cudaGetLastError(), "job tables");
        ck(launch_bucket(p, jobs, (unsigned)nj, c->tw, c->d_err, S.s(), spec != nullptr), "batched product");
    }
}

// q~_i = limbs [s, s + nq) of product i (stride sp, pl limbs written), into
// a compact array of stride nq.
__global__ void k_dc_extract(const u32* __restrict__ prod, u64 sp, u64 pl, u64 s, u64 nq, u32* __restrict__ q,
                             u64 m) {
    const u64 total = m * nq;
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const u64 i = t / nq, k = t % nq;
        q[t] = s + k < pl ? prod[i * sp + s + k] : 0u;
    }
}

// CTA-wide out = A +- B over n limbs (A: la limbs, B: lb limbs, or B null and
// the one-limb value bsmall), carry / borrow out returned to every thread.
// out may be A. blockDim a multiple of 32.
__device__ u32 cta_addsub(const u32* A, u64 la, const u32* B, u64 lb, u32 bsmall, u32* out, u64 n, int sub,
                          GP* ws, u32* s_carry) {
    if (threadIdx.x == 0) *s_carry = 0;
    __syncthreads();
    for (u64 c0 = 0; c0 < n; c0 += (u64)blockDim.x * ADD_LPT) {
        const u64 base = c0 + (u64)threadIdx.x * ADD_LPT;
        u32 av[ADD_LPT], bv[ADD_LPT];
        GP g{0, 1};
#pragma unroll
        for (int w = 0; w < ADD_LPT; ++w) {
            const u64 k = base + w;
            av[w] = k < n && k < la ? A[k] : 0u;
            bv[w] = k < n ? (B ? (k < lb ? B[k] : 0u) : (k == 0 ? bsmall : 0u)) : 0u;
            if (k < n) g = gp_then(g, limb_gp(av[w], bv[w], sub));
        }
        GP tot;
        const GP ex = block_scan_gp(g, ws, &tot);
        const u32 cin_chunk = *s_carry;
        u32 c = ex.g | (ex.p & cin_chunk);
#pragma unroll
        for (int w = 0; w < ADD_LPT; ++w) {
            const u64 k = base + w;
            if (k >= n) break;
            u32 r;
            if (!sub) {
                const u64 x = (u64)av[w] + bv[w] + c;
                r = (u32)x;
                c = (u32)(x >> 32);
            } else {
                const u64 x = (u64)av[w] - bv[w] - c;
                r = (u32)x;
                c = (u32)((x >> 63) & 1);
            }
            out[k] = r;
        }
        __syncthreads();
        if (threadIdx.x == 0) *s_carry = tot.g | (tot.p & cin_chunk);
        __syncthreads();
    }
    return *s_carry;
}

// One CTA per node i: R = V_i - U_i (U_i = q~_i P), then q~ and R move one
// unit at a time until 0 <= R < P; writes q (node 2i) and R (node 2i + 1) of
// the next level, zero-padded to its stride. A correction count above the
// bound sets bit 2 of *err (reported as an internal error).
__global__ void k_dc_fix(const u32* __restrict__ V, u64 sin, const u32* __restrict__ U, u64 su,
                         const u32* __restrict__ QE, u64 nq, const u32* __restrict__ P, u64 n, u32* scr, u64 w,
                         u32* __restrict__ out, u64 sout, u32* err) {
    __shared__ GP ws[33];
    __shared__ u32 s_carry;
    const u64 i = blockIdx.x;
    V += i * sin;
    U += i * su;
    u32* R = scr + i * (2 * w + nq + 1);
    u32* T = R + w;
    u32* Q = T + w;  // nq + 1 limbs
    for (u64 k = threadIdx.x; k <= nq; k += blockDim.x) Q[k] = k < nq ? QE[i * nq + k] : 0u;
    __syncthreads();
    u32 neg = cta_addsub(V, sin, U, su, 0, R, w, 1, ws, &s_carry);
    int it = 0;
    while (neg && it < 64) {
        if (cta_addsub(R, w, P, n, 0, R, w, 0, ws, &s_carry)) neg = 0;
        cta_addsub(Q, nq + 1, nullptr, 0, 1, Q, nq + 1, 1, ws, &s_carry);
        ++it;
    }
    while (it < 64) {
        if (cta_addsub(R, w, P, n, 0, T, w, 1, ws, &s_carry)) break;
        u32* t = R;
        R = T;
        T = t;
        cta_addsub(Q, nq + 1, nullptr, 0, 1, Q, nq + 1, 0, ws, &s_carry);
        ++it;
    }
    if (it >= 64 && threadIdx.x == 0) atomicOr(err, 2u);
    u32* oq = out + (2 * i) * sout;
    u32* orr = out + (2 * i + 1) * sout;
    for (u64 k = threadIdx.x; k < sout; k += blockDim.x) {
        oq[k] = k < n ? Q[k] : 0u;
        orr[k] = k < n ? R[k] : 0u;
    }
}

// One thread per leaf (a value below 10^72 in 8 limbs): 72 decimal digits.
__global__ void k_dc_leaf(const u32* __restrict__ nodes, u64 stride, u64 m, char* __restrict__ out) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    u32 x[DC_LEAF_LIMBS];
#pragma unroll
    for (int k = 0; k < DC_LEAF_LIMBS; ++k) x[k] = (u64)k < stride ? nodes[i * stride + k] : 0u;
    char* o = out + i * (9 * DC_LEAF_GROUPS);
#pragma unroll 1
    for (int g = DC_LEAF_GROUPS - 1; g >= 0; --g) {
        u64 rem = 0;
#pragma unroll
        for (int k = DC_LEAF_LIMBS - 1; k >= 0; --k) {
            const u64 cur = (rem << 32) | x[k];
            x[k] = (u32)(cur / 1000000000u);
            rem = cur % 1000000000u;
        }
        u32 r = (u32)rem;
#pragma unroll
        for (int d = 8; d >= 0; --d) {
            o[9 * g + d] = (char)('0' + r % 10);
            r /= 10;
        }
    }
}

// k_dc_fix's steps for one node as grid-wide passes driven from the host:
// for the top levels, whose few nodes have up to millions of limbs, one CTA
// a node would leave the GPU idle. R = V - U over w limbs, then R += P with
// q -= 1 while R is negative, then R -= P with q += 1 while R >= P; q and R
// go to oq / orr (n limbs, zero-padded to sout). R, T: w limbs; Q: nq + 1.
void fix_node_grid(Scope& S, const u32* V, uint64_t sin, const u32* U, uint64_t su, const u32* QE, uint64_t nq,
                   DV Pj, DV R, DV T, DV Q, DV one, u32* oq, u32* orr, uint64_t sout) {
    const uint64_t n = Pj.n;
    ck(cudaMemsetAsync(Q.p, 0, 4 * (nq + 1), S.s()), "cudaMemsetAsync");
    ck(cudaMemcpyAsync(Q.p, QE, 4 * nq, cudaMemcpyDeviceToDevice, S.s()), "D2D");
    u32 neg = addsub(S, {const_cast<u32*>(V), sin}, {const_cast<u32*>(U), su}, R, true);
    int it = 0;
    while (neg && it < 64) {
        if (addsub(S, R, Pj, R, false)) neg = 0;
        addsub(S, Q, one, Q, true);
        ++it;
    }
    while (it < 64) {
        if (addsub(S, R, Pj, T, true)) break;
        std::swap(R, T);
        addsub(S, Q, one, Q, false);
        ++it;
    }
    if (it >= 64) {
        set_error("decimal conversion: a quotient correction did not converge");
        throw Err{B2M_ERR_INTERNAL};
    }
    ck(cudaMemsetAsync(oq, 0, 4 * sout, S.s()), "cudaMemsetAsync");
    ck(cudaMemsetAsync(orr, 0, 4 * sout, S.s()), "cudaMemsetAsync");
    const uint64_t k = std::min(n, sout);
    ck(cudaMemcpyAsync(oq, Q.p, 4 * std::min(k, nq + 1), cudaMemcpyDeviceToDevice, S.s()), "D2D");
    ck(cudaMemcpyAsync(orr, R.p, 4 * std::min(k, R.n), cudaMemcpyDeviceToDevice, S.s()), "D2D");
}

// Levels with at most this many nodes, of at least DC_GRID_MIN_LIMBS limbs,
// fix their nodes with grid-wide passes (fix_node_grid).
constexpr uint64_t DC_GRID_MAX_NODES = 16;
constexpr uint64_t DC_GRID_MIN_LIMBS = 1 << 15;

// -1, 0, 1 as a <, ==, > b (trimmed).
int cmp(Scope& S, DV a, DV b) {
    if (a.n != b.n) return a.n < b.n ? -1 : 1;
    DV t = S.vec(a.n);
    if (addsub(S, a, b, t, true)) return -1;
    return top_len(S, t) ? 1 : 0;
}

// Decimal digits of trimmed X, no leading zeros ("0" for zero).
std::string to_decimal(Scope& S, DV X) {
    if (X.n == 0) return "0";
    std::vector<DV> P;  // P[j] = 10^(9 2^j)
    P.push_back(upload(S, {1000000000u}));
    P[0] = trim(S, P[0]);
    while (true) {
        DV sq = mul(S, P.back(), P.back());
        if ((int)P.size() - 1 >= DC_LEAF_J && cmp(S, X, sq) < 0) {
            P.push_back(sq);
            break;
        }
        P.push_back(sq);
    }
    const int J = (int)P.size() - 2;  // X < P[J]^2 = P[J+1], J >= DC_LEAF_J
    u32* err = reinterpret_cast<u32*>(S.word() + 4);
    ck(cudaMemsetAsync(err, 0, 4, S.s()), "cudaMemsetAsync");
    // level J input: one node, X zero-padded to 2 len(P_J) limbs
    uint64_t sin = std::max<uint64_t>(2 * P[J].n, X.n);
    DV in = copy(S, X, sin);
    uint64_t m = 1;
    // Reciprocals R ~ 2^(32 E) / P_j: Newton for the top level only; below,
    // 1/P_j = P_j / P_{j+1}, so R_j = P_j * R_{j+1} (more precise than level j
    // needs), truncated to its top n + 4 limbs.
    DV R;
    uint64_t E = 0;
    for (int j = J; j > DC_LEAF_J; --j) {
        const DV Pj = P[j];
        const uint64_t n = Pj.n;
        const uint64_t L = n + 3;
        if (j == J) {
            const int sh = __builtin_clz(limb_at(S, Pj, n - 1));
            DV Pn = sh ? shl(S, Pj, 0, sh) : Pj;
            R = recip(S, Pn, L);  // ~ 2^(32 (L + n)) / Pn, Pn = P_j 2^sh
            if (sh) R = shl(S, R, 0, sh);
            E = L + n;
        } else {
            R = mul(S, Pj, R);
        }
        if (R.n > L + 1) {  // keep the top L + 1 limbs
            const uint64_t t = R.n - (L + 1);
            R = {R.p + t, R.n - t};
            E -= t;
        }
        // q~ = floor(V * R / 2^(32 E)) ~ floor(V / P_j), from V's top L + 1 limbs
        const uint64_t k = sin > L + 1 ? sin - (L + 1) : 0;
        if (E < k) {
            set_error("decimal conversion: reciprocal scale below the operand cut");
            throw Err{B2M_ERR_INTERNAL};
        }
        const uint64_t na = sin - k, sp = na + R.n;
        DV prod = S.vec(m * sp);
        batched_mul(S, in.p + k, sin, na, R.p, 0, R.n, prod.p, sp, m);
        const uint64_t s = E - k, nq = n + 1;
        DV qe = S.vec(m * nq);
        k_dc_extract<<<grid_for(m * nq), 256, 0, S.s()>>>(prod.p, sp, sp, s, nq, qe.p, m);
        ck(cudaGetLastError(), "k_dc_extract");
        const uint64_t su = nq + n;
        DV U = S.vec(m * su);
        batched_mul(S, qe.p, nq, nq, Pj.p, 0, n, U.p, su, m);
        // next level: 2m nodes below P_j = P_{j-1}^2, stride 2 len(P_{j-1})
        const uint64_t sout = j - 1 > DC_LEAF_J ? 2 * P[j - 1].n : DC_LEAF_LIMBS;
        DV out = S.vec(2 * m * sout);
        const uint64_t w = std::max(sin, su) + 1;
        if (m <= DC_GRID_MAX_NODES && w >= DC_GRID_MIN_LIMBS) {
            DV R = S.vec(w), T = S.vec(w), Q = S.vec(nq + 1);
            DV one = S.vec(1);
            static const u32 one_h = 1;
            ck(cudaMemcpyAsync(one.p, &one_h, 4, cudaMemcpyHostToDevice, S.s()), "H2D");
            for (uint64_t i = 0; i < m; ++i)
                fix_node_grid(S, in.p + i * sin, sin, U.p + i * su, su, qe.p + i * nq, nq, Pj, R, T, Q, one,
                              out.p + (2 * i) * sout, out.p + (2 * i + 1) * sout, sout);
        } else {
            DV scr = S.vec(m * (2 * w + nq + 1));
            unsigned threads = 32;
            while (threads < 1024 && (uint64_t)threads * ADD_LPT < w) threads <<= 1;
            k_dc_fix<<<(unsigned)m, threads, 0, S.s()>>>(in.p, sin, U.p, su, qe.p, nq, Pj.p, n, scr.p, w, out.p,
                                                         sout, err);
            ck(cudaGetLastError(), "k_dc_fix");
        }
        in = out;
        sin = sout;
        m *= 2;
    }
    // leaves: m nodes below 10^72 in 8-limb slots
    const uint64_t digits = m * 9 * DC_LEAF_GROUPS;
    char* d_str = static_cast<char*>(S.raw(digits));
    k_dc_leaf<<<(unsigned)((m + 127) / 128), 128, 0, S.s()>>>(in.p, sin, m, d_str);
    ck(cudaGetLastError(), "k_dc_leaf");
    std::string str(digits, '0');
    ck(cudaMemcpyAsync(&str[0], d_str, digits, cudaMemcpyDeviceToHost, S.s()), "D2H");
    u32 h_err = 0;
    ck(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, S.s()), "D2H");
    ck(cudaStreamSynchronize(S.s()), "cudaStreamSynchronize");
    if (h_err) {
        set_error("decimal conversion: a quotient correction did not converge");
        throw Err{B2M_ERR_INTERNAL};
    }
    const b2m_status e = take_device_error(S.c());
    if (e != B2M_OK) throw Err{e};
    const size_t first = str.find_first_not_of('0');
    return first == std::string::npos ? std::string("0") : str.substr(first);
}

// Wraps an API body: context, device, error translation.
template <class F>
b2m_status run_op(b2m_stream stream, F&& f) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    cudaSetDevice(c->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    try {
        Scope S(c, s);
        f(S);
    } catch (const Err& e) {
        cudaStreamSynchronize(s);
        return e.st;
    } catch (const std::exception& e) {
        cudaStreamSynchronize(s);
        set_error(e.what());
        return B2M_ERR_INTERNAL;
    }
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamSynchronize");
    return take_device_error(c);
}

void put(Scope& S, DV v, uint32_t* dst, uint64_t cap, uint64_t* len) {
    if (v.n > cap) {
        set_error("output buffer too small");
        throw Err{B2M_ERR_OUTPUT_TOO_SMALL};
    }
    if (v.n) ck(cudaMemcpyAsync(dst, v.p, 4 * v.n, cudaMemcpyDeviceToDevice, S.s()), "D2D");
    *len = v.n;
}

}  // namespace big

// ---------------------------------------------------------------------------- launchers for other files
namespace {
__global__ void k_top_diff(const u32* __restrict__ a, const u32* __restrict__ b, u64 n, unsigned long long* out) {
    unsigned long long t = 0;
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (u64)gridDim.x * blockDim.x)
        if (a[k] != b[k]) t = k + 1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, t, off);
        t = o > t ? o : t;
    }
    if ((threadIdx.x & 31) == 0 && t) atomicMax(out, t);
}
}  // namespace

uint64_t addsub_scratch_bytes(uint64_t n) {
    const uint64_t nb = (n + big::AS_CH - 1) / big::AS_CH;
    return ((nb * sizeof(GP) + 255) & ~255ull) + ((nb * 4 + 255) & ~255ull);
}

cudaError_t launch_addsub(const u32* a, uint64_t la, const u32* b, uint64_t lb, uint64_t n, int sub, u32* out,
                          void* scratch, u32* flag, cudaStream_t s) {
    if (n == 0) return cudaMemsetAsync(flag, 0, 4, s);
    const uint64_t nb = (n + big::AS_CH - 1) / big::AS_CH;
    GP* agg = static_cast<GP*>(scratch);
    u32* cin = reinterpret_cast<u32*>(static_cast<unsigned char*>(scratch) + ((nb * sizeof(GP) + 255) & ~255ull));
    big::k_as_reduce<<<(unsigned)nb, big::AS_T, 0, s>>>(a, la, b, lb, n, sub, agg);
    big::k_as_scan<<<1, 1024, 0, s>>>(agg, nb, cin, flag);
    big::k_as_apply<<<(unsigned)nb, big::AS_T, 0, s>>>(a, la, b, lb, n, sub, cin, out);
    return cudaGetLastError();
}

cudaError_t launch_top(const u32* a, uint64_t n, unsigned long long* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    big::k_top<<<big::grid_for(n), 256, 0, s>>>(a, n, out);
    return cudaGetLastError();
}

cudaError_t launch_top_diff(const u32* a, const u32* b, uint64_t n, unsigned long long* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_top_diff<<<big::grid_for(n), 256, 0, s>>>(a, b, n, out);
    return cudaGetLastError();
}

}  // namespace b2m

using namespace b2m;

extern "C" {

b2m_status b2m_divmod_device(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb, uint32_t* d_q,
                             uint64_t q_cap, uint64_t* q_len, uint32_t* d_r, uint64_t r_cap, uint64_t* r_len,
                             b2m_stream stream) {
    if ((na && !d_a) || !d_b || !nb || (d_q && !q_len) || (d_r && !r_len)) return B2M_ERR_INVALID_ARGUMENT;
    return big::run_op(stream, [&](big::Scope& S) {
        big::DV a = big::trim(S, {const_cast<u32*>(d_a), na});
        big::DV b = big::trim(S, {const_cast<u32*>(d_b), nb});
        big::DV q, r;
        big::divmod(S, a, b, &q, &r);
        if (d_q) big::put(S, q, d_q, q_cap, q_len);
        if (d_r) big::put(S, r, d_r, r_cap, r_len);
    });
}

b2m_status b2m_isqrt_device(const uint32_t* d_a, uint64_t na, uint32_t* d_out, uint64_t cap, uint64_t* out_len,
                            b2m_stream stream) {
    if ((na && !d_a) || !d_out || !out_len) return B2M_ERR_INVALID_ARGUMENT;
    return big::run_op(stream, [&](big::Scope& S) {
        big::DV a = big::trim(S, {const_cast<u32*>(d_a), na});
        big::put(S, big::isqrt(S, a), d_out, cap, out_len);
    });
}

/* compute_pi_chudnovsky (src/chudnovsky.cpp:107-164) with every step on the
 * device: the same guard digits (16), term count, tree, floor square root of
 * 10005 * 10^(2 prec), numerator 426880 * Q * sqrtC, floor division by T and
 * decimal formatting. */
b2m_status b2m_compute_pi(uint64_t digits, char* out, uint64_t cap, uint64_t* len, b2m_pi_timings* times) {
    if (!out || !len) return B2M_ERR_INVALID_ARGUMENT;
    if (cap < digits + 3) return B2M_ERR_OUTPUT_TOO_SMALL;  // "3." + digits + NUL
    const uint64_t prec = digits + 16;
    uint64_t terms = (uint64_t)((double)prec / 14.181647462725477) + 2;  // src/chudnovsky.cpp:37,54-59
    if (terms < 2) terms = 2;
    using clk = std::chrono::steady_clock;
    auto ms = [](clk::time_point a, clk::time_point b) {
        return std::chrono::duration<double, std::milli>(b - a).count();
    };
    b2m_pi_timings tm{};
    tm.terms = terms;
    const auto t0 = clk::now();
    b2m_pqt* tree = nullptr;
    b2m_status st = b2m_chudnovsky_bs(0, terms, nullptr, &tree);
    if (st != B2M_OK) return st;
    uint64_t tl[3];
    int32_t tsign = 0;
    b2m_pqt_info(tree, tl, &tsign, nullptr, nullptr);
    const auto t1 = clk::now();
    clk::time_point t2, t3, t4;
    st = big::run_op(nullptr, [&](big::Scope& S) {
        if (tsign <= 0) {
            set_error("compute_pi: T of the tree is not positive");
            throw big::Err{B2M_ERR_INTERNAL};
        }
        big::DV Q{const_cast<u32*>(b2m_pqt_device(tree, 1)), tl[1]};
        big::DV T{const_cast<u32*>(b2m_pqt_device(tree, 2)), tl[2]};
        // one = 10^prec by square-and-multiply, as pow10_big (src/chudnovsky.cpp:42-51)
        big::DV one = big::trim(S, big::upload(S, {1u})), base = big::trim(S, big::upload(S, {10u}));
        for (uint64_t e = prec; e; e >>= 1) {
            if (e & 1) one = big::mul(S, one, base);
            if (e > 1) base = big::mul(S, base, base);
        }
        big::DV rad = big::mul(S, big::mul(S, one, one), big::trim(S, big::upload(S, {10005u})));
        big::DV sqrt_c = big::isqrt(S, rad);
        t2 = clk::now();
        big::DV num = big::mul(S, big::mul(S, Q, big::trim(S, big::upload(S, {426880u}))), sqrt_c);
        big::DV q, r;
        big::divmod(S, num, T, &q, &r);
        t3 = clk::now();
        const std::string str = big::to_decimal(S, q);
        t4 = clk::now();
        std::string res;
        if (digits == 0) {
            res = "3";
        } else {
            res.reserve(digits + 2);
            res.push_back(str[0]);
            res.push_back('.');
            res.append(str, 1, (size_t)digits);
        }
        std::memcpy(out, res.c_str(), res.size() + 1);
        *len = res.size();
    });
    b2m_pqt_free(tree);
    if (st != B2M_OK) return st;
    if (times) {
        tm.tree_ms = ms(t0, t1);
        tm.sqrt_ms = ms(t1, t2);
        tm.div_ms = ms(t2, t3);
        tm.decimal_ms = ms(t3, t4);
        tm.total_ms = ms(t0, clk::now());
        *times = tm;
    }
    return B2M_OK;
}

b2m_status b2m_to_decimal_device(const uint32_t* d_a, uint64_t na, char* out, uint64_t cap, uint64_t* len,
                                 b2m_stream stream) {
    if ((na && !d_a) || !out || !len) return B2M_ERR_INVALID_ARGUMENT;
    return big::run_op(stream, [&](big::Scope& S) {
        const std::string str = big::to_decimal(S, big::trim(S, {const_cast<u32*>(d_a), na}));
        if (str.size() + 1 > cap) {
            set_error("decimal output buffer too small");
            throw big::Err{B2M_ERR_OUTPUT_TOO_SMALL};
        }
        std::memcpy(out, str.c_str(), str.size() + 1);
        *len = str.size();
    });
}

// ---- host-buffer forms (the reference's BigInt magnitudes live on the host)
static big::DV host_in(big::Scope& S, const uint32_t* h, uint64_t n) {
    big::DV d = S.vec(n);
    if (n) big::ck(cudaMemcpyAsync(d.p, h, 4 * n, cudaMemcpyHostToDevice, S.s()), "H2D");
    return big::trim(S, d);  // synchronises: h may be pageable
}
static void host_out(big::Scope& S, big::DV v, uint32_t* h, uint64_t cap, uint64_t* len) {
    if (v.n > cap) {
        set_error("output buffer too small");
        throw big::Err{B2M_ERR_OUTPUT_TOO_SMALL};
    }
    if (v.n) big::ck(cudaMemcpyAsync(h, v.p, 4 * v.n, cudaMemcpyDeviceToHost, S.s()), "D2H");
    big::ck(cudaStreamSynchronize(S.s()), "cudaStreamSynchronize");
    *len = v.n;
}

b2m_status b2m_divmod_host(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb, uint32_t* q,
                           uint64_t q_cap, uint64_t* q_len, uint32_t* r, uint64_t r_cap, uint64_t* r_len) {
    if ((na && !a) || !b || !nb || (q && !q_len) || (r && !r_len)) return B2M_ERR_INVALID_ARGUMENT;
    return big::run_op(nullptr, [&](big::Scope& S) {
        big::DV dq, dr;
        big::divmod(S, host_in(S, a, na), host_in(S, b, nb), &dq, &dr);
        if (q) host_out(S, dq, q, q_cap, q_len);
        if (r) host_out(S, dr, r, r_cap, r_len);
    });
}

b2m_status b2m_isqrt_host(const uint32_t* a, uint64_t na, uint32_t* out, uint64_t cap, uint64_t* out_len) {
    if ((na && !a) || !out || !out_len) return B2M_ERR_INVALID_ARGUMENT;
    return big::run_op(nullptr, [&](big::Scope& S) { host_out(S, big::isqrt(S, host_in(S, a, na)), out, cap, out_len); });
}

b2m_status b2m_to_decimal_host(const uint32_t* a, uint64_t na, char* out, uint64_t cap, uint64_t* len) {
    if ((na && !a) || !out || !len) return B2M_ERR_INVALID_ARGUMENT;
    return big::run_op(nullptr, [&](big::Scope& S) {
        const std::string str = big::to_decimal(S, host_in(S, a, na));
        if (str.size() + 1 > cap) {
            set_error("decimal output buffer too small");
            throw big::Err{B2M_ERR_OUTPUT_TOO_SMALL};
        }
        std::memcpy(out, str.c_str(), str.size() + 1);
        *len = str.size();
    });
}

}  // extern "C"
