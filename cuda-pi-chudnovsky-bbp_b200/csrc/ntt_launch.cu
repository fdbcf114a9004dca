// ntt_launch.cu -- pass plans and the launch sequence of one product.
//
// For N = 2^L >= 2^14 (a 2- or 3-pass plan):
//   A: first pass (u32 limbs -> 16-bit digits), middle passes, last pass
//      (spectrum register-major per CTA);
//   B: first pass, middle passes, fused last pass (B's last forward pass,
//      pointwise product with A's spectrum and N^-1, first inverse pass);
//   inverse middle/first passes (pass 1 yields the coefficients), then the
//   decoupled-lookback carry into u32 limbs and the trimmed length.
// For N <= 2^13 a single CTA does everything.
//
// Reference counterpart: mul_ntt_cuda (src/ntt_cuda.cu:179-243) -- host
// repack (include/ntt.h:56-64), bit reversal + log2 N radix-2 launches per
// transform, pointwise (:117-121), scale (:124-128), host carry
// (include/ntt.h:70-91) -- all replaced by the sequence below.
#include <cuda_runtime.h>

#include <vector>

#include <algorithm>

#include "b2m.h"
#include "b2m_context.h"
#include "b2m_internal.h"
#include "carry.cuh"
#include "ntt_engine.cuh"

namespace b2m {

// Default plans for 2^14..2^27 points: the autotuner's fastest candidate on
// a B200 for a square product of each length (uniform random limbs, median
// of three). Small lengths favour 2^12-element tiles (more CTAs for little
// work); 2^19..2^21 two passes with a 2^11..2^12 contiguous last pass; 2^22
// and up (and 2^23 within 0.4%) three passes of 2^12-element tiles, whose
// extra HBM sweep costs less than the latency that one 2^14-element CTA per
// SM leaves exposed.
namespace {
struct DefaultPlan {
    int npass, r0, r1, r2, tile;
};
constexpr int DEFAULT_MIN_LOGN = 14, DEFAULT_MAX_LOGN = 27;
constexpr DefaultPlan kDefaultPlans[DEFAULT_MAX_LOGN - DEFAULT_MIN_LOGN + 1] = {
    {2, 8, 6, 0, 12},    // 2^14
    {2, 7, 8, 0, 12},    // 2^15
    {2, 8, 8, 0, 12},    // 2^16
    {2, 8, 9, 0, 12},    // 2^17
    {2, 7, 11, 0, 12},   // 2^18
    {2, 7, 12, 0, 12},   // 2^19
    {2, 8, 12, 0, 13},   // 2^20
    {2, 9, 12, 0, 13},   // 2^21
    {3, 6, 8, 8, 12},    // 2^22
    {2, 10, 13, 0, 13},  // 2^23
    {3, 9, 9, 6, 12},    // 2^24
    {3, 9, 8, 8, 12},    // 2^25
    {3, 9, 9, 8, 12},    // 2^26
    {3, 6, 9, 12, 12},   // 2^27
};
}  // namespace

// Sub-transform plans of 3 * 2^logn-point products where the autotuner's
// fastest differs from the power-of-two default (measured on a B200 with
// na = nb = 3 * 2^(logn-2) limbs): the radix-3 step already adds a pass, and
// three shorter passes beat two long ones (2^23: [10, 13] 1.887 ms ->
// [9, 6, 8] 1.770 ms; 2^21: [9, 12] 0.502 -> [9, 6, 6] 0.471 ms).
struct Radix3Plan {
    int logn, npass, r0, r1, r2;
};
constexpr Radix3Plan kRadix3Plans[] = {
    {15, 2, 8, 7, 0}, {19, 2, 8, 11, 0}, {21, 3, 9, 6, 6}, {23, 3, 9, 6, 8},
};

Plan make_plan(int logn, int three) {
    if (three) {
        for (const Radix3Plan& d : kRadix3Plans)
            if (d.logn == logn) {
                const int r[3] = {d.r0, d.r1, d.r2};
                Plan p = make_plan_split(logn, r, d.npass, 12);
                p.three = 1;
                return p;
            }
        Plan p = make_plan(logn, 0);
        p.three = 1;
        return p;
    }
    if (logn <= SMALL_MAX_LOGN) return make_plan_split(logn, nullptr, 0, -1);
    if (logn >= DEFAULT_MIN_LOGN && logn <= DEFAULT_MAX_LOGN) {
        const DefaultPlan& d = kDefaultPlans[logn - DEFAULT_MIN_LOGN];
        const int r[3] = {d.r0, d.r1, d.r2};
        return make_plan_split(logn, r, d.npass, d.tile);
    }
    return make_plan_custom(logn, -1, 12);
}

// r0 < 0 picks a default split: two passes up to 2^26, the first radix at
// most 2^12 (a first pass keeps >= 4 columns, 32-byte rows, in its tile) and
// the last (contiguous) pass up to 2^14; three near-equal passes above.
Plan make_plan_custom(int logn, int r0, int tile) {
    if (logn <= SMALL_MAX_LOGN) return make_plan_split(logn, nullptr, 0, tile);
    int r[3];
    if (logn <= 26) {
        r[0] = r0 > 0 ? r0 : (logn / 2 < 12 ? logn / 2 : 12);
        r[1] = logn - r[0];
        return make_plan_split(logn, r, 2, tile);
    }
    r[0] = logn / 3;
    r[1] = logn / 3;
    r[2] = logn - 2 * (logn / 3);
    return make_plan_split(logn, r, 3, tile);
}

// Explicit pass radices r[0..npass) (sum logn) with one tile size (log2
// elements, <= 0 for the default); npass = 0 is the single-CTA product.
Plan make_plan_split(int logn, const int* r, int npass, int tile) {
    Plan p;
    p.logn = logn;
    p.npass = npass;
    if (npass == 0) return p;
    for (int k = 0; k < npass; ++k) p.logr[k] = r[k];
    if (tile <= 0) tile = logn >= 20 ? 14 : (logn >= 17 ? 13 : 12);
    int before = 0;
    for (int k = 0; k < p.npass; ++k) {
        const int rk = p.logr[k];
        const int after = logn - before - rk;  // log2 S
        int c = tile - rk;
        if (c < 0) c = 0;
        const int cap = (k + 1 < p.npass) ? after : (logn - rk);
        if (c > cap) c = cap;
        p.logc[k] = c;
        before += rk;
    }
    return p;
}

// Plans the autotuners time: every two-pass split with a first radix of
// 2^6..2^12 and a last of 2^6..2^14, and from 2^21 points every three-pass
// split with radices 2^6..2^12 (the last up to 2^14), each at tiles of 2^12,
// 2^13 and 2^14 elements where the radices fit.
std::vector<Plan> plan_candidates(int logn) {
    std::vector<Plan> v;
    if (logn <= SMALL_MAX_LOGN) {
        v.push_back(make_plan(logn));
        return v;
    }
    for (int r0 = 6; r0 <= 12; ++r0) {
        const int r1 = logn - r0;
        if (r1 < 6 || r1 > 14) continue;
        for (int tile = 12; tile <= 14; ++tile) {
            if (r0 > tile || r1 > tile) continue;
            const int r[2] = {r0, r1};
            v.push_back(make_plan_split(logn, r, 2, tile));
        }
    }
    if (logn >= 21) {
        for (int r0 = 6; r0 <= 12; ++r0)
            for (int r1 = 6; r1 <= 12; ++r1) {
                const int r2 = logn - r0 - r1;
                if (r2 < 6 || r2 > 14) continue;
                for (int tile = 12; tile <= 14; ++tile) {
                    if (r0 > tile || r1 > tile || r2 > tile) continue;
                    const int r[3] = {r0, r1, r2};
                    v.push_back(make_plan_split(logn, r, 3, tile));
                }
            }
    }
    if (v.empty()) v.push_back(make_plan(logn));
    return v;
}

PassGeo pass_geo(const Plan& p, int k) {
    int before = 0;
    for (int i = 0; i < k; ++i) before += p.logr[i];
    PassGeo g;
    g.logr = p.logr[k];
    g.logc = p.logc[k];
    g.logs = p.logn - before - g.logr;
    g.logm = g.logr + g.logs;
    g.grid = (unsigned)(1ull << (p.logn - g.logr - g.logc));
    // 16 elements per thread (two 8-point tasks per radix-8 level), <= 1024.
    const int logt = g.logr + g.logc - 4;
    g.block = (unsigned)(1u << (logt < 10 ? logt : 10));
    const size_t rp = (size_t)(1 << g.logr) + (size_t)((1 << g.logr) >> 6);
    g.smem = rp * ((size_t)1 << g.logc) * sizeof(u64);
    Context* c = ctx();
    if (c && k + 1 < p.npass && g.logm >= TWT_MIN_LOGM) {
        std::lock_guard<std::mutex> lk(c->twt_mu);
        for (const Context::TwTable& t : c->twt)
            if (t.logm == g.logm && t.logr == g.logr) {
                g.tfwd = t.fwd;
                g.tinv = t.inv;
                if (k == 0) g.tinv0 = t.inv0;
                break;
            }
    }
    return g;
}

// fwd[i] = w_M^(brev(row) * col), inv[i] = its inverse, i = (row << logs) + col:
// the same exponent the pass kernels form (bitrev(row) * col * 2^(32 - logM)).
__global__ void k_build_twtable(u64* __restrict__ fwd, u64* __restrict__ inv, int logm, int logr, RootTables tw) {
    const int logs = logm - logr;
    const u64 m = 1ull << logm;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x) {
        const u32 row = (u32)(i >> logs), col = (u32)(i & ((1ull << logs) - 1));
        const u64 f = __brev(row) >> (32 - logr);
        const u32 e = (u32)((f * col) << (32 - logm));
        fwd[i] = e ? uroot(e, tw.u1, tw.u2) : 1ull;
        inv[i] = e ? uroot(0u - e, tw.u1, tw.u2) : 1ull;
    }
}

__global__ void k_scale_table(u64* __restrict__ dst, const u64* __restrict__ src, u64 m, int shift) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x)
        dst[i] = gl_shl(src[i], shift);
}

// The pass-0 copy of an existing inverse table, scaled by 2^-logm (= 2^(192 -
// logm), a shift); skipped when the budget is short.
static cudaError_t twtable_ensure_inv0(Context* c, Context::TwTable& t, cudaStream_t s) {
    if (t.inv0) return cudaSuccess;
    const uint64_t bytes = 8ull << t.logm;
    if (!budget_reserve(c, bytes)) return cudaSuccess;
    u64* mem = nullptr;
    cudaError_t e = cudaMalloc(&mem, bytes);
    if (e != cudaSuccess) {
        budget_release(c, bytes);
        cudaGetLastError();
        return cudaSuccess;
    }
    const u64 m = 1ull << t.logm;
    k_scale_table<<<(unsigned)std::min<u64>(65535, (m + 255) / 256), 256, 0, s>>>(mem, t.inv, m, 192 - t.logm);
    if ((e = cudaGetLastError()) == cudaSuccess) e = cudaStreamSynchronize(s);  // built before anyone sees it
    if (e != cudaSuccess) {
        cudaFree(mem);
        budget_release(c, bytes);
        return e;
    }
    t.inv0 = mem;
    t.inv0_bytes = bytes;
    return cudaSuccess;
}

cudaError_t twtable_ensure(Context* c, const Plan& p, cudaStream_t s) {
    if (!c || p.npass < 2) return cudaSuccess;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return cudaSuccess;
    for (int k = 0; k + 1 < p.npass; ++k) {
        const PassGeo g = pass_geo(p, k);
        if (g.logm < TWT_MIN_LOGM || g.tfwd) continue;
        std::lock_guard<std::mutex> lk(c->twt_mu);
        bool have = false;
        for (const Context::TwTable& t : c->twt) have |= (t.logm == g.logm && t.logr == g.logr);
        if (have) continue;
        const uint64_t bytes = 2 * (8ull << g.logm);
        if (!budget_reserve(c, bytes)) continue;  // no room: the kernels build twiddles instead
        u64* mem = nullptr;
        cudaError_t e = cudaMalloc(&mem, bytes);
        if (e != cudaSuccess) {
            budget_release(c, bytes);
            cudaGetLastError();
            continue;
        }
        const u64 m = 1ull << g.logm;
        k_build_twtable<<<(unsigned)std::min<u64>(65535, (m + 255) / 256), 256, 0, s>>>(mem, mem + m, g.logm, g.logr,
                                                                                      c->tw);
        if ((e = cudaGetLastError()) == cudaSuccess) e = cudaStreamSynchronize(s);  // built before anyone sees it
        if (e != cudaSuccess) {
            cudaFree(mem);
            budget_release(c, bytes);
            return e;
        }
        c->twt.push_back({g.logm, g.logr, mem, mem + m, bytes});
    }
    // the scaled inverse copy for pass 0
    if (p.npass >= 2) {
        const PassGeo g = pass_geo(p, 0);
        if (g.tinv && !g.tinv0) {
            std::lock_guard<std::mutex> lk(c->twt_mu);
            for (Context::TwTable& t : c->twt)
                if (t.logm == g.logm && t.logr == g.logr) {
                    cudaError_t e = twtable_ensure_inv0(c, t, s);
                    if (e != cudaSuccess) return e;
                    break;
                }
        }
    }
    return cudaSuccess;
}

void twtable_free_all(Context* c) {
    std::lock_guard<std::mutex> lk(c->twt_mu);
    for (const Context::TwTable& t : c->twt) {
        cudaFree(t.fwd);
        budget_release(c, t.bytes);
        if (t.inv0) {
            cudaFree(t.inv0);
            budget_release(c, t.inv0_bytes);
        }
    }
    c->twt.clear();
}

uint64_t carry_scratch_bytes(int logn) { return carry_scratch_bytes_n(1ull << logn); }

uint64_t carry_scratch_bytes_n(uint64_t points) {
    const uint64_t chunks = points >= CARRY_CHUNK ? points / CARRY_CHUNK : 1;
    return chunks * sizeof(LookbackSlot) + 256;
}

uint64_t workspace_bytes_plan(const Plan& p) {
    if (p.npass == 0) return 256;
    const uint64_t n = plan_points(p);
    return 2 * 8 * n + carry_scratch_bytes_n(n);
}

void choose_length(uint64_t digits, int* logn, int* three) {
    int l = 2;
    while ((1ull << l) < digits) ++l;
    if (l - 2 >= RADIX3_MIN_LOG && (3ull << (l - 2)) >= digits) {
        *logn = l - 2;
        *three = 1;
    } else {
        *logn = l;
        *three = 0;
    }
}

// Pass k's geometry; radix-3 plans run it over the three sub-transforms.
static PassGeo geo(const Plan& p, int k) {
    PassGeo g = pass_geo(p, k);
    if (p.three) {
        g.zdim = 3;
        g.zstride = 1ull << p.logn;
    }
    return g;
}

// Geometry of inverse pass k. For pass 0 with a scaled inverse table
// (PassGeo::tinv0) the pass applies 2^-logn with its twiddles, and
// *carry_scale, the factor the carry kernel divides by, drops to what is
// left (3 for a 3 * 2^logn transform, else 1). The table is looked up once
// here, so the pass and the carry agree.
static PassGeo inverse_geo(const Plan& p, int k, uint64_t* carry_scale) {
    PassGeo g = geo(p, k);
    if (k == 0 && g.tinv0) {
        g.tinv = g.tinv0;
        *carry_scale = p.three ? 3 : 1;
    }
    return g;
}

uint64_t workspace_bytes_for(int logn) {
    if (logn <= SMALL_MAX_LOGN) return 256;
    return 2 * (8ull << logn) + carry_scratch_bytes(logn);
}

cudaError_t configure_kernels() {
    cudaError_t e = configure_first();
    if (e == cudaSuccess) e = configure_mid();
    if (e == cudaSuccess) e = configure_inv();
    if (e == cudaSuccess) e = configure_last();
    if (e == cudaSuccess) e = configure_fused();
    if (e == cudaSuccess) e = configure_small();
    return e;
}

int plan_launches(const Plan& p) { return p.npass == 0 ? 1 : 3 * p.npass + (p.three ? 3 : 0); }

static cudaError_t launch_forward(const u32* limbs, uint64_t nlimbs, u64* buf, const Plan& p,
                                  const RootTables& tw, bool fused, const u64* aspec, u64 ninv,
                                  cudaStream_t s, Tracer* tr) {
    cudaError_t e;
    int k0 = 0;
    if (p.three) {
        // radix-3 step from the digits, then the sub-transforms from pass 0
        if (tr) tr->mark(s, B2M_K_R3_FWD, 0);
        e = launch_r3_fwd(s, limbs, 2 * nlimbs, buf, p.logn, tw);
    } else {
        if (tr) tr->mark(s, B2M_K_FWD_FIRST, p.logr[0]);
        e = launch_fwd_first(p.logr[0], geo(p, 0), s, limbs, 2 * nlimbs, buf, tw);
        k0 = 1;
    }
    for (int k = k0; e == cudaSuccess && k + 1 < p.npass; ++k) {
        if (tr) tr->mark(s, B2M_K_FWD_MID, p.logr[k]);
        e = launch_fwd_mid(p.logr[k], geo(p, k), s, buf, tw);
    }
    if (e != cudaSuccess) return e;
    const int last = p.npass - 1;
    if (tr) tr->mark(s, fused ? B2M_K_FUSED_LAST : B2M_K_FWD_LAST, p.logr[last]);
    return fused ? launch_fused_last(p.logr[last], geo(p, last), s, buf, aspec, ninv, tw)
                 : launch_fwd_last(p.logr[last], geo(p, last), s, buf, tw);
}

cudaError_t launch_product(const u32* a, uint64_t na, const u32* b, uint64_t nb, u32* out, uint64_t* out_len,
                           void* ws, const Plan& p, const RootTables& tw, u32* err, cudaStream_t s, Tracer* tr,
                           cudaEvent_t b_ready) {
    const int logn = p.logn;
    const uint64_t n = plan_points(p);
    const u64 ninv = gl_inv(n);
    const u64 nout = na + nb;
    if (p.npass == 0) {
        PassGeo g{};
        const int T = logn >= 4 ? (1 << (logn - 4)) : 1;
        const size_t rp = (size_t)(1 << logn) + (size_t)((1 << logn) >> 6);
        g.grid = 1;
        g.block = (unsigned)T;
        g.smem = 2 * rp * sizeof(u64) + (size_t)T * 2 * sizeof(u64);
        if (b_ready) {
            cudaError_t e = cudaStreamWaitEvent(s, b_ready, 0);
            if (e != cudaSuccess) return e;
        }
        if (tr) tr->mark(s, B2M_K_SMALL, logn);
        cudaError_t e = launch_mul_small(logn, g, s, a, na, b, nb, out, nout,
                                         reinterpret_cast<unsigned long long*>(out_len), ninv, tw);
        if (tr) tr->end(s);
        return e;
    }
    u64* bufA = static_cast<u64*>(ws);
    u64* bufB = bufA + n;
    unsigned char* scratch = reinterpret_cast<unsigned char*>(bufB + n);
    const uint64_t nchunks = n / CARRY_CHUNK;
    LookbackSlot* slots = reinterpret_cast<LookbackSlot*>(scratch);
    u32* ticket = reinterpret_cast<u32*>(scratch + nchunks * sizeof(LookbackSlot));
    unsigned long long* len_tmp = reinterpret_cast<unsigned long long*>(ticket + 2);
    cudaError_t e = cudaMemsetAsync(scratch, 0, carry_scratch_bytes_n(n), s);
    if (e != cudaSuccess) return e;
    unsigned long long* ol = out_len ? reinterpret_cast<unsigned long long*>(out_len) : len_tmp;
    if (out_len && (e = cudaMemsetAsync(out_len, 0, sizeof(uint64_t), s)) != cudaSuccess) return e;

    if (a == b && na == nb) {
        // a square: one forward transform, its spectrum squared in the fused pass
        if (b_ready && (e = cudaStreamWaitEvent(s, b_ready, 0)) != cudaSuccess) return e;
        if ((e = launch_forward(b, nb, bufB, p, tw, true, nullptr, 1, s, tr)) != cudaSuccess) return e;
    } else {
        if ((e = launch_forward(a, na, bufA, p, tw, false, nullptr, 0, s, tr)) != cudaSuccess) return e;
        if (b_ready && (e = cudaStreamWaitEvent(s, b_ready, 0)) != cudaSuccess) return e;
        if ((e = launch_forward(b, nb, bufB, p, tw, true, bufA, 1, s, tr)) != cudaSuccess) return e;
    }
    uint64_t carry_scale = n;  // the factor the carry still divides by
    for (int k = p.npass - 2; k >= 0; --k) {
        if (tr) tr->mark(s, B2M_K_INV_MID, p.logr[k]);
        if ((e = launch_inv_mid(p.logr[k], inverse_geo(p, k, &carry_scale), s, bufB, tw)) != cudaSuccess) return e;
    }
    if (p.three) {
        if (tr) tr->mark(s, B2M_K_R3_INV, 0);
        if ((e = launch_r3_inv(s, bufB, logn, tw)) != cudaSuccess) return e;
    }
    if (tr) tr->mark(s, B2M_K_CARRY, 0);
    e = launch_carry((unsigned)nchunks, s, bufB, out, nout, slots, ticket, ol, err, nullptr, 1, carry_scale);
    if (tr) tr->end(s);
    return e;
}

// Forward transform of operand `op` of every job (op 1 ends in the fused
// pass: pointwise product with bufA and the first inverse pass).
static cudaError_t bucket_forward(const Plan& p, const ProdJob* jobs, unsigned njobs, const RootTables& tw,
                                  cudaStream_t s, int op, u64 ninv) {
    const int logn = p.logn;
    cudaError_t e = cudaSuccess;
    int k0 = 0;
    if (p.three) {
        e = launch_r3_fwd(s, nullptr, 0, nullptr, logn, tw, jobs, njobs, op);
    } else {
        e = launch_fwd_first(p.logr[0], geo(p, 0), s, nullptr, 0, nullptr, tw, jobs, njobs, op);
        k0 = 1;
    }
    for (int k = k0; e == cudaSuccess && k + 1 < p.npass; ++k)
        e = launch_fwd_mid(p.logr[k], geo(p, k), s, nullptr, tw, jobs, njobs, op);
    if (e != cudaSuccess) return e;
    const int last = p.npass - 1;
    return op == 0 ? launch_fwd_last(p.logr[last], geo(p, last), s, nullptr, tw, jobs, njobs)
                   : launch_fused_last(p.logr[last], geo(p, last), s, nullptr, nullptr, ninv, tw, jobs, njobs);
}

cudaError_t launch_bucket_spectrum(const Plan& p, const ProdJob* jobs, unsigned njobs, const RootTables& tw,
                                   cudaStream_t s) {
    if (p.npass == 0) return cudaErrorInvalidValue;
    return bucket_forward(p, jobs, njobs, tw, s, 0, 0);
}

cudaError_t launch_bucket(const Plan& p, const ProdJob* jobs, unsigned njobs, const RootTables& tw, u32* err,
                          cudaStream_t s, bool a_ready) {
    const int logn = p.logn;
    const u64 ninv = gl_inv(plan_points(p));
    if (p.npass == 0) {
        PassGeo g{};
        const int T = logn >= 4 ? (1 << (logn - 4)) : 1;
        const size_t rp = (size_t)(1 << logn) + (size_t)((1 << logn) >> 6);
        g.grid = 1;
        g.block = (unsigned)T;
        g.smem = 2 * rp * sizeof(u64) + (size_t)T * 2 * sizeof(u64);
        return launch_mul_small(logn, g, s, nullptr, 0, nullptr, 0, nullptr, 0, nullptr, ninv, tw, jobs, njobs);
    }
    cudaError_t e = cudaSuccess;
    for (int op = a_ready ? 1 : 0; op < 2 && e == cudaSuccess; ++op)
        e = bucket_forward(p, jobs, njobs, tw, s, op, 1);  // N^-1: in the carry
    uint64_t carry_scale = plan_points(p);
    for (int k = p.npass - 2; e == cudaSuccess && k >= 0; --k)
        e = launch_inv_mid(p.logr[k], inverse_geo(p, k, &carry_scale), s, nullptr, tw, jobs, njobs);
    if (e == cudaSuccess && p.three) e = launch_r3_inv(s, nullptr, logn, tw, jobs, njobs);
    if (e != cudaSuccess) return e;
    const unsigned nchunks = (unsigned)(plan_points(p) / CARRY_CHUNK);
    return launch_carry(nchunks, s, nullptr, nullptr, 0, nullptr, nullptr, nullptr, err, jobs, njobs, carry_scale);
}

// Zero a contiguous carry-scratch region and every job's out_len
// (multi-pass products accumulate it with atomicMax; empty jobs report 0).
__global__ void k_batch_prep(const ProdJob* __restrict__ jobs, unsigned njobs, unsigned long long* scratch,
                             u64 nwords) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += stride) scratch[i] = 0;
    for (u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += stride)
        if (jobs[j].out_len) *jobs[j].out_len = 0;
}

cudaError_t launch_batch_prep(cudaStream_t s, const ProdJob* jobs, unsigned njobs, unsigned long long* scratch,
                              u64 nwords) {
    const uint64_t work = nwords > njobs ? nwords : njobs;
    const unsigned blocks = (unsigned)(work / 256 + 1 < 1024 ? work / 256 + 1 : 1024);
    k_batch_prep<<<blocks, 256, 0, s>>>(jobs, njobs, scratch, nwords);
    return cudaGetLastError();
}

// Seeded operands: limb i = high half of splitmix64's output function at
// seed + (i + 1) * 0x9E3779B97F4A7C15, top limb forced non-zero; kind 1 gives
// all-0xFFFFFFFF limbs.
__device__ __forceinline__ u32 gen_limb(u64 seed, u64 i) {
    u64 z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (u32)(z >> 32);
}

__global__ void k_gen_operand(u64 seed, u64 n, u32 kind, u32* out) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        u32 v = kind == 1 ? 0xFFFFFFFFu : gen_limb(seed, i);
        if (i == n - 1 && v == 0) v = 1;
        out[i] = v;
    }
}

cudaError_t launch_gen_operand(cudaStream_t s, u64 seed, u64 n, u32 kind, u32* out) {
    if (n == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    k_gen_operand<<<blocks, 256, 0, s>>>(seed, n, kind, out);
    return cudaGetLastError();
}

}  // namespace b2m
