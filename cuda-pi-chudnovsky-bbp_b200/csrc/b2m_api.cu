// b2m_api.cu -- library context and the single-product C ABI (include/b2m.h).
//
// Replaces the per-call setup and teardown of src/ntt_cuda.cu:179-243 (device
// probe, 4x cudaMalloc, 2x twiddle build, blocking copies, cudaFree, CPU
// fallback) with: one context per process bound to one device, root tables
// uploaded once, workspaces from a stream-ordered pool under an HBM budget,
// and status codes instead of a fallback.
#include <cuda_runtime.h>

#include <algorithm>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "b2m.h"
#include "b2m_internal.h"
#include "b2m_context.h"

namespace b2m {

Context* g_ctx = nullptr;
std::mutex g_ctx_mu;
static thread_local std::string t_err;

void set_error(const std::string& msg) { t_err = msg; }

b2m_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return B2M_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return B2M_ERR_OUT_OF_MEMORY;
    return B2M_ERR_CUDA;
}

int ilog2_pow2(uint64_t n) {
    int l = 0;
    while ((1ull << l) < n) ++l;
    return l;
}

uint64_t ntt_length_of(uint64_t na, uint64_t nb) {
    const uint64_t x = 2 * na + 2 * nb;
    uint64_t n = 1;
    while (n < x) n <<= 1;
    return n;
}

// Host construction of the resident root tables (see RootTables).
static std::vector<u64> build_tables() {
    std::vector<u64> t((1u << 15) + (2u << 16));
    u64* dtw = t.data();
    for (int l = 0; l <= 14; ++l) {
        const u64 w = gl_root2(l);
        u64 x = 1;
        for (uint64_t e = 0; e < (1ull << l); ++e) {
            dtw[(1ull << l) + e] = x;
            x = gl_mul(x, w);
        }
    }
    dtw[0] = 1;
    u64* u1 = dtw + (1u << 15);
    u64* u2 = u1 + (1u << 16);
    const u64 step2 = gl_pow(GL_RHO, 1ull << 16);
    u64 x1 = 1, x2 = 1;
    for (uint64_t e = 0; e < (1ull << 16); ++e) {
        u1[e] = x1;
        u2[e] = x2;
        x1 = gl_mul(x1, GL_RHO);
        x2 = gl_mul(x2, step2);
    }
    return t;
}

static void destroy_context(Context* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->hstream) cudaStreamSynchronize(c->hstream);
    if (c->hcopy) cudaStreamSynchronize(c->hcopy);
    if (c->host_dev) cudaFree(c->host_dev);
    twtable_free_all(c);
    if (c->d_tables) cudaFree(c->d_tables);
    if (c->d_err) cudaFree(c->d_err);
    if (c->hstream) cudaStreamDestroy(c->hstream);
    if (c->hcopy) cudaStreamDestroy(c->hcopy);
    if (c->hev_a) cudaEventDestroy(c->hev_a);
    if (c->hev_b) cudaEventDestroy(c->hev_b);
    delete c;
}

Context* ctx() { return g_ctx; }

// Budget accounting: reserve before an allocation, release after a free.
bool budget_reserve(Context* c, uint64_t bytes) {
    uint64_t cur = c->in_use.load();
    do {
        if (cur + bytes > c->budget) return false;
    } while (!c->in_use.compare_exchange_weak(cur, cur + bytes));
    return true;
}
void budget_release(Context* c, uint64_t bytes) { c->in_use.fetch_sub(bytes); }

b2m_status check_sizes(uint64_t na, uint64_t nb, int* logn) {
    if (na > (1ull << 29) || nb > (1ull << 29)) {
        set_error("operand longer than 2^29 limbs");
        return B2M_ERR_TOO_LARGE;
    }
    const int l = ilog2_pow2(ntt_length_of(na, nb));
    if (l > MAX_LOGN) {
        set_error("transform length above 2^30 (na + nb > 2^28 limbs)");
        return B2M_ERR_TOO_LARGE;
    }
    *logn = l;
    return B2M_OK;
}

}  // namespace b2m

using namespace b2m;

extern "C" {

b2m_status b2m_init(int device, uint64_t hbm_budget_bytes) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (g_ctx && g_ctx->device == device) {
        if (hbm_budget_bytes) g_ctx->budget = hbm_budget_bytes;
        return B2M_OK;
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0) {
        set_error(e != cudaSuccess ? cudaGetErrorString(e) : "no CUDA device");
        return B2M_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) {
        set_error("device index out of range");
        return B2M_ERR_INVALID_ARGUMENT;
    }
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return cuda_status(e, "cudaGetDeviceProperties");
    if (prop.major != 10 || prop.minor != 0) {
        set_error("this build targets sm_100a (B200); device is sm_" + std::to_string(prop.major) +
                  std::to_string(prop.minor));
        return B2M_ERR_NO_DEVICE;
    }
    if (g_ctx) {
        destroy_context(g_ctx);
        g_ctx = nullptr;
    }
    if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    if ((e = configure_kernels()) != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute");
    Context* c = new Context();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    std::vector<u64> tables = build_tables();
    const size_t tbytes = tables.size() * sizeof(u64);
    if ((e = cudaMalloc(&c->d_tables, tbytes)) != cudaSuccess) {
        delete c;
        return cuda_status(e, "cudaMalloc(tables)");
    }
    if ((e = cudaMemcpy(c->d_tables, tables.data(), tbytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&c->d_err, 256)) != cudaSuccess || (e = cudaMemset(c->d_err, 0, 256)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->hstream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->hcopy, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->hev_a, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->hev_b, cudaEventDisableTiming)) != cudaSuccess) {
        destroy_context(c);
        return cuda_status(e, "context setup");
    }
    c->tw.dtw = c->d_tables;
    c->tw.u1 = c->d_tables + (1u << 15);
    c->tw.u2 = c->tw.u1 + (1u << 16);
    // Keep freed pool memory cached so steady-state calls never hit cudaMalloc.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    c->budget = hbm_budget_bytes ? hbm_budget_bytes : (uint64_t)(0.9 * (double)free_b);
    g_ctx = c;
    return B2M_OK;
}

b2m_status b2m_shutdown(void) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    destroy_context(g_ctx);
    g_ctx = nullptr;
    return B2M_OK;
}

int b2m_cuda_available(void) {
    static std::atomic<int> cached{-1};
    int v = cached.load();
    if (v < 0) {
        v = (g_ctx != nullptr || b2m_init(0, 0) == B2M_OK) ? 1 : 0;
        cached.store(v);
    }
    return v;
}

const char* b2m_strerror(b2m_status s) {
    switch (s) {
        case B2M_OK: return "ok";
        case B2M_ERR_INVALID_ARGUMENT: return "invalid argument";
        case B2M_ERR_NO_DEVICE: return "no usable sm_100 CUDA device";
        case B2M_ERR_NOT_INITIALIZED: return "library not initialised (call b2m_init)";
        case B2M_ERR_CUDA: return "CUDA runtime error";
        case B2M_ERR_OUT_OF_MEMORY: return "out of device memory or HBM budget";
        case B2M_ERR_TOO_LARGE: return "operands too large (transform length above 2^30)";
        case B2M_ERR_OUTPUT_TOO_SMALL: return "output buffer smaller than na + nb limbs";
        case B2M_ERR_DEVICE_TIMEOUT: return "a bounded device-side wait timed out";
        case B2M_ERR_QUEUE_FULL: return "request table full";
        case B2M_ERR_NOT_FOUND: return "unknown ticket";
        case B2M_ERR_SHUTDOWN: return "server stopping";
        case B2M_ERR_INTERNAL: return "internal check failed";
    }
    return "unknown status";
}

const char* b2m_last_error(void) { return t_err.c_str(); }

uint64_t b2m_ntt_length(uint64_t na, uint64_t nb) { return ntt_length_of(na, nb); }

uint64_t b2m_workspace_bytes(uint64_t na, uint64_t nb) {
    if (na == 0 || nb == 0) return 0;
    Context* c = ctx();
    int logn = 0, three = 0;
    choose_length(2 * (na + nb), &logn, &three);
    Plan p = c ? plan_for(c, logn, three) : make_plan(logn, three);
    p.three = three;
    return workspace_bytes_plan(p);
}

b2m_status b2m_mul_device(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                          uint32_t* d_out, uint64_t out_cap, uint64_t* d_out_len, b2m_stream stream) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if ((na && !d_a) || (nb && !d_b)) return B2M_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (na == 0 || nb == 0) {
        if (d_out_len) return cuda_status(cudaMemsetAsync(d_out_len, 0, sizeof(uint64_t), s), "memset");
        return B2M_OK;
    }
    if (!d_out) return B2M_ERR_INVALID_ARGUMENT;
    if (out_cap < na + nb) return B2M_ERR_OUTPUT_TOO_SMALL;
    int logn;
    b2m_status st = check_sizes(na, nb, &logn);
    if (st != B2M_OK) return st;
    cudaSetDevice(c->device);
    const Plan p = product_plan(c, na, nb);
    if (cudaError_t te = twtable_ensure(c, p, s)) return cuda_status(te, "twiddle table");
    const uint64_t wsb = workspace_bytes_plan(p);
    if (!budget_reserve(c, wsb)) {
        set_error("HBM budget exhausted");
        return B2M_ERR_OUT_OF_MEMORY;
    }
    void* ws = nullptr;
    cudaError_t e = cudaMallocAsync(&ws, wsb, s);
    if (e != cudaSuccess) {
        budget_release(c, wsb);
        return cuda_status(e, "cudaMallocAsync(workspace)");
    }
    e = launch_product(d_a, na, d_b, nb, d_out, d_out_len, ws, p, c->tw, c->d_err, s);
    cudaError_t e2 = cudaFreeAsync(ws, s);
    budget_release(c, wsb);
    if (e != cudaSuccess) return cuda_status(e, "kernel launch");
    return cuda_status(e2, "cudaFreeAsync(workspace)");
}

b2m_status b2m_plan_describe(uint64_t na, uint64_t nb, b2m_plan_desc* d) {
    if (!d || na == 0 || nb == 0) return B2M_ERR_INVALID_ARGUMENT;
    int logn;
    b2m_status st = check_sizes(na, nb, &logn);
    if (st != B2M_OK) return st;
    Context* c = ctx();
    int l = 0, three = 0;
    choose_length(2 * (na + nb), &l, &three);
    Plan p = c ? plan_for(c, l, three) : make_plan(l, three);
    p.three = three;
    d->ntt_log2 = (uint32_t)l;
    d->three = (uint32_t)three;
    d->npass = (uint32_t)p.npass;
    for (int k = 0; k < 3; ++k) {
        d->logr[k] = (uint32_t)p.logr[k];
        d->logc[k] = (uint32_t)p.logc[k];
    }
    d->launches = (uint32_t)plan_launches(p);
    return B2M_OK;
}

b2m_status b2m_selftest_wait_timeout(b2m_stream stream) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    cudaSetDevice(c->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // Two chunks of (zero) coefficients and their lookback slots, the ticket
    // starting at 1: the CTA that takes chunk 1 waits for chunk 0's flag,
    // which nothing ever sets (no CTA is left to take ticket 0).
    const uint64_t n = 2 * (uint64_t)CARRY_CHUNK;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    const uint64_t bc = al(8 * n), bo = al(4 * (n / 2)), bs = al(2 * sizeof(LookbackSlot)), bt = 256;
    void* mem = nullptr;
    cudaError_t e = cudaMallocAsync(&mem, bc + bo + bs + bt, s);
    if (e != cudaSuccess) return cuda_status(e, "cudaMallocAsync(self-test)");
    unsigned char* b = static_cast<unsigned char*>(mem);
    u32* ticket = reinterpret_cast<u32*>(b + bc + bo + bs);
    static const u32 one = 1;
    e = cudaMemsetAsync(mem, 0, bc + bo + bs + bt, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ticket, &one, 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = launch_carry(2, s, reinterpret_cast<const u64*>(b), reinterpret_cast<u32*>(b + bc), n / 2,
                         reinterpret_cast<LookbackSlot*>(b + bc + bo), ticket,
                         reinterpret_cast<unsigned long long*>(ticket + 2), c->d_err);
    cudaFreeAsync(mem, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_status(e, "self-test launch");
    return take_device_error(c);
}

b2m_status b2m_set_plan(const b2m_plan_desc* desc) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (!desc || desc->ntt_log2 < 2 || desc->ntt_log2 > (uint32_t)MAX_LOGN) return B2M_ERR_INVALID_ARGUMENT;
    const int logn = (int)desc->ntt_log2;
    // only plans the library can launch: one of the autotuner's candidates
    for (const Plan& p : plan_candidates(logn)) {
        bool same = p.npass == (int)desc->npass;
        for (int k = 0; same && k < p.npass; ++k)
            same = p.logr[k] == (int)desc->logr[k] && p.logc[k] == (int)desc->logc[k];
        if (same) {
            set_tuned(c, logn, p);
            return B2M_OK;
        }
    }
    set_error("b2m_set_plan: not one of the candidate plans for this length");
    return B2M_ERR_INVALID_ARGUMENT;
}

b2m_status b2m_autotune(uint64_t na, uint64_t nb, b2m_stream stream, b2m_tune_entry* out, uint32_t cap,
                        uint32_t* n) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (na == 0 || nb == 0 || (cap && !out)) return B2M_ERR_INVALID_ARGUMENT;
    int logn;
    b2m_status st = check_sizes(na, nb, &logn);
    if (st != B2M_OK) return st;
    cudaSetDevice(c->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int three = 0;
    choose_length(2 * (na + nb), &logn, &three);  // candidates for the (sub-)transform length
    std::vector<Plan> cands = plan_candidates(logn);
    for (Plan& cp : cands) cp.three = three;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    const uint64_t ba = al(4 * na), bb = al(4 * nb), bo = al(4 * (na + nb)), wsb = al(workspace_bytes_plan(cands[0]));
    const uint64_t need = ba + bb + bo + 256 + wsb;
    if (!budget_reserve(c, need)) {
        set_error("HBM budget exhausted");
        return B2M_ERR_OUT_OF_MEMORY;
    }
    void* mem = nullptr;
    cudaError_t e = cudaMallocAsync(&mem, need, s);
    if (e != cudaSuccess) {
        budget_release(c, need);
        return cuda_status(e, "cudaMallocAsync(autotune)");
    }
    unsigned char* base = static_cast<unsigned char*>(mem);
    u32* da = reinterpret_cast<u32*>(base);
    u32* db = reinterpret_cast<u32*>(base + ba);
    u32* dout = reinterpret_cast<u32*>(base + ba + bb);
    uint64_t* dlen = reinterpret_cast<uint64_t*>(base + ba + bb + bo);
    void* ws = base + ba + bb + bo + 256;
    e = launch_gen_operand(s, 12345, na, 0, da);
    if (e == cudaSuccess) e = launch_gen_operand(s, 67890, nb, 0, db);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    float best = 1e30f;
    size_t best_i = 0;
    uint32_t cnt = 0;
    for (size_t i = 0; i < cands.size() && e == cudaSuccess; ++i) {
        // one warm-up, then the median of three timed products
        float ms[3];
        e = twtable_ensure(c, cands[i], s);
        for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
            e = cudaEventRecord(t0, s);
            if (e == cudaSuccess) e = launch_product(da, na, db, nb, dout, dlen, ws, cands[i], c->tw, c->d_err, s);
            if (e == cudaSuccess) e = cudaEventRecord(t1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(t1);
            if (e == cudaSuccess && rep > 0) cudaEventElapsedTime(&ms[rep - 1], t0, t1);
        }
        if (e != cudaSuccess) break;
        std::sort(ms, ms + 3);
        if (ms[1] < best) {
            best = ms[1];
            best_i = i;
        }
        if (cnt < cap) {
            b2m_tune_entry& o = out[cnt++];
            const Plan& p = cands[i];
            o.plan.ntt_log2 = (uint32_t)logn;
            o.plan.npass = (uint32_t)p.npass;
            for (int k = 0; k < 3; ++k) {
                o.plan.logr[k] = (uint32_t)p.logr[k];
                o.plan.logc[k] = (uint32_t)p.logc[k];
            }
            o.plan.launches = (uint32_t)plan_launches(p);
            o.plan.three = (uint32_t)p.three;
            o.ms = ms[1];
            o.chosen = 0;
        }
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFreeAsync(mem, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    budget_release(c, need);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_status(e, "autotune");
    st = take_device_error(c);
    if (st != B2M_OK) return st;
    Plan kept = cands[best_i];
    kept.three = 0;  // tuned plans are kept per power-of-two length
    set_tuned(c, logn, kept);
    if (best_i < cnt) out[best_i].chosen = 1;
    if (n) *n = cnt;
    return B2M_OK;
}

b2m_status b2m_mul_device_traced(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                                 uint32_t* d_out, uint64_t out_cap, uint64_t* d_out_len, b2m_stream stream,
                                 b2m_kernel_time* times, uint32_t cap, uint32_t* n) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (!d_a || !d_b || !d_out || !times || !n || na == 0 || nb == 0) return B2M_ERR_INVALID_ARGUMENT;
    if (out_cap < na + nb) return B2M_ERR_OUTPUT_TOO_SMALL;
    int logn;
    b2m_status st = check_sizes(na, nb, &logn);
    if (st != B2M_OK) return st;
    cudaSetDevice(c->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const Plan p = product_plan(c, na, nb);
    if (cudaError_t te = twtable_ensure(c, p, s)) return cuda_status(te, "twiddle table");
    const uint64_t wsb = workspace_bytes_plan(p);
    if (!budget_reserve(c, wsb)) {
        set_error("HBM budget exhausted");
        return B2M_ERR_OUT_OF_MEMORY;
    }
    void* ws = nullptr;
    cudaError_t e = cudaMallocAsync(&ws, wsb, s);
    if (e != cudaSuccess) {
        budget_release(c, wsb);
        return cuda_status(e, "cudaMallocAsync(workspace)");
    }
    Tracer tr;
    for (int i = 0; i <= Tracer::CAP; ++i) cudaEventCreate(&tr.ev[i]);
    e = launch_product(d_a, na, d_b, nb, d_out, d_out_len, ws, p, c->tw, c->d_err, s, &tr);
    cudaFreeAsync(ws, s);
    budget_release(c, wsb);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) {
        uint32_t k = 0;
        for (int i = 0; i < tr.n && k < cap; ++i, ++k) {
            float ms = 0;
            cudaEventElapsedTime(&ms, tr.ev[i], tr.ev[i + 1]);
            times[k].kind = tr.kind[i];
            times[k].logr = tr.logr[i];
            times[k].ms = ms;
        }
        *n = k;
    }
    for (int i = 0; i <= Tracer::CAP; ++i) cudaEventDestroy(tr.ev[i]);
    if (e != cudaSuccess) return cuda_status(e, "traced product");
    return take_device_error(c);
}

b2m_status b2m_stream_check(b2m_stream stream) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    cudaError_t e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamSynchronize");
    return take_device_error(c);
}

b2m_status b2m_mul_host(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb, uint32_t* out,
                        uint64_t out_cap, uint64_t* out_len) {
    if (!out_len || (na && !a) || (nb && !b)) return B2M_ERR_INVALID_ARGUMENT;
    if (na == 0 || nb == 0) {  // x * 0 = 0 needs no device (src/ntt_cuda.cu:181)
        *out_len = 0;
        return B2M_OK;
    }
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (!out) return B2M_ERR_INVALID_ARGUMENT;
    if (out_cap < na + nb) return B2M_ERR_OUTPUT_TOO_SMALL;
    int logn;
    b2m_status st = check_sizes(na, nb, &logn);
    if (st != B2M_OK) return st;
    std::lock_guard<std::mutex> lk(c->host_mu);
    cudaSetDevice(c->device);
    const Plan p = product_plan(c, na, nb);
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    const uint64_t ba = al(4 * na), bb = al(4 * nb), bo = al(4 * (na + nb)), bl = 256;
    const uint64_t wsb = workspace_bytes_plan(p);
    const uint64_t need = ba + bb + bo + bl + wsb;
    if (need > c->host_dev_cap) {
        if (c->host_dev) {
            cudaStreamSynchronize(c->hstream);
            cudaFree(c->host_dev);
            budget_release(c, c->host_dev_cap);
            c->host_dev = nullptr;
            c->host_dev_cap = 0;
        }
        if (!budget_reserve(c, need)) {
            set_error("HBM budget exhausted");
            return B2M_ERR_OUT_OF_MEMORY;
        }
        cudaError_t e = cudaMalloc(&c->host_dev, need);
        if (e != cudaSuccess) {
            budget_release(c, need);
            return cuda_status(e, "cudaMalloc(host-call buffers)");
        }
        c->host_dev_cap = need;
    }
    unsigned char* base = static_cast<unsigned char*>(c->host_dev);
    u32* da = reinterpret_cast<u32*>(base);
    u32* db = reinterpret_cast<u32*>(base + ba);
    u32* dout = reinterpret_cast<u32*>(base + ba + bb);
    uint64_t* dlen = reinterpret_cast<uint64_t*>(base + ba + bb + bo);
    void* ws = base + ba + bb + bo + bl;
    cudaStream_t s = c->hstream;
    cudaError_t e;
    if ((e = twtable_ensure(c, p, s)) != cudaSuccess) return cuda_status(e, "twiddle table");
    if (a == b && na == nb) {
        // a square (the reference's x * x passes one vector twice): one copy,
        // one forward transform (launch_product's squaring path)
        if ((e = cudaMemcpyAsync(da, a, 4 * na, cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return cuda_status(e, "cudaMemcpyAsync(H2D)");
        if ((e = launch_product(da, na, da, na, dout, dlen, ws, p, c->tw, c->d_err, s, nullptr, nullptr)) !=
            cudaSuccess)
            return cuda_status(e, "kernel launch");
    } else {
        // Operand B crosses the bus after A, on a second stream, while A's
        // forward transform runs: the product waits for B only before B's
        // transform.
        if ((e = cudaMemcpyAsync(da, a, 4 * na, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaEventRecord(c->hev_a, s)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(c->hcopy, c->hev_a, 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(db, b, 4 * nb, cudaMemcpyHostToDevice, c->hcopy)) != cudaSuccess ||
            (e = cudaEventRecord(c->hev_b, c->hcopy)) != cudaSuccess)
            return cuda_status(e, "cudaMemcpyAsync(H2D)");
        if ((e = launch_product(da, na, db, nb, dout, dlen, ws, p, c->tw, c->d_err, s, nullptr, c->hev_b)) !=
            cudaSuccess) {
            cudaStreamSynchronize(c->hcopy);
            return cuda_status(e, "kernel launch");
        }
    }
    uint64_t hlen = 0;
    if ((e = cudaMemcpyAsync(out, dout, 4 * (na + nb), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&hlen, dlen, sizeof(uint64_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_status(e, "cudaMemcpyAsync(D2H)");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_status(e, "cudaStreamSynchronize");
    st = take_device_error(c);
    if (st != B2M_OK) return st;
    *out_len = hlen;
    return B2M_OK;
}

}  // extern "C"
