// b2m_server.cu -- continuous-batching multiply server (include/b2m.h, b2m_server_*).
//
// No counterpart in the reference, whose multiply is a blocking library call.
// Requests of mixed sizes arrive at any time (b2m_server_submit). A native
// scheduler thread admits them in arrival order while the HBM budget allows
// (operands it generates, outputs it owns, and each product's transform
// workspace all count), and whenever one of its stream slots is free it turns
// everything admitted so far into one dispatch: the dispatch's products are
// bucketed by transform length and launched bucket by bucket (b2m_batch's
// launch_bucket) on that slot's stream. Several dispatches run at once on
// different streams, so requests that arrive while others are on the GPU are
// admitted as slots and memory free up and their work overlaps on the device.
// Every product is checked on the device modulo 2^32 - 1 and 2^32 + 1 (limb
// sums and alternating sums of operands and product) before it is reported
// done; workspace returns to the budget at completion, owned buffers at
// b2m_server_release. Each slot keeps its dispatch blocks (job tables and
// transform workspaces) in one device arena that only grows, so steady-state
// dispatches allocate nothing large. The scheduler never waits on the device:
// it polls completion events.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "b2m.h"
#include "b2m_context.h"
#include "b2m_internal.h"

namespace b2m {

constexpr int RES_WORDS = 9;  // per job: (sum, even, odd) of a, b and the product

// res[j*9 + 3*w + k]: array w (a, b, out) limb sum (k=0), even-index sum (1),
// odd-index sum (2). Grid: x over 4096-limb chunks, y over jobs.
__global__ void k_residues(const ProdJob* __restrict__ jobs, unsigned long long* res) {
    const ProdJob& J = jobs[blockIdx.y];
    const u64 base = (u64)blockIdx.x * 4096;
    __shared__ unsigned long long s[RES_WORDS];
    if (threadIdx.x < RES_WORDS) s[threadIdx.x] = 0;
    __syncthreads();
    for (int w = 0; w < 3; ++w) {
        const u32* p = w == 0 ? J.a : (w == 1 ? J.b : J.out);
        const u64 n = w == 0 ? J.na : (w == 1 ? J.nb : J.na + J.nb);
        unsigned long long even = 0, odd = 0;
        for (u64 i = base + threadIdx.x; i < n && i < base + 4096; i += blockDim.x) {
            const u32 v = p[i];
            if (i & 1) odd += v;
            else even += v;
        }
        for (int off = 16; off > 0; off >>= 1) {
            even += __shfl_xor_sync(0xFFFFFFFFu, even, off);
            odd += __shfl_xor_sync(0xFFFFFFFFu, odd, off);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&s[3 * w + 0], even + odd);
            atomicAdd(&s[3 * w + 1], even);
            atomicAdd(&s[3 * w + 2], odd);
        }
    }
    __syncthreads();
    if (threadIdx.x < RES_WORDS && s[threadIdx.x]) atomicAdd(res + (u64)blockIdx.y * RES_WORDS + threadIdx.x, s[threadIdx.x]);
}

static bool residues_match(const unsigned long long* r) {
    typedef unsigned __int128 u128;
    const u64 m1 = 0xFFFFFFFFull, m2 = 0x100000001ull;
    auto mod1 = [&](int w) { return (u64)(r[3 * w] % m1); };
    auto mod2 = [&](int w) {  // sum of even-index limbs minus odd-index limbs, mod 2^32 + 1
        const u64 e = r[3 * w + 1] % m2, o = r[3 * w + 2] % m2;
        return (e + m2 - o) % m2;
    };
    const bool ok1 = (u64)(((u128)mod1(0) * mod1(1)) % m1) == mod1(2);
    const bool ok2 = (u64)(((u128)mod2(0) * mod2(1)) % m2) == mod2(2);
    return ok1 && ok2;
}

static uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Req {
    b2m_request r{};
    int logn = 0;       // log2 of the (sub-)transform length
    int three = 0;      // 1: 3 * 2^logn points
    uint64_t pts = 0;   // transform points
    int32_t state = 0;  // 0 queued, 1 on the GPU, 2 done, 3 failed
    b2m_status status = B2M_OK;
    u32* a = nullptr;  // device operands (owned when generated)
    u32* b = nullptr;
    u32* out = nullptr;
    bool own_a = false, own_b = false, own_out = false;
    uint64_t own_bytes = 0;  // budget held until release
    uint64_t ws_bytes = 0;   // budget held until completion
    uint64_t out_len = 0;
    int32_t residues_ok = 0;
    uint64_t t_submit = 0, t_admit = 0, t_done = 0;
};

struct Slot {
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    bool busy = false;
    std::vector<uint64_t> ids;
    void* block = nullptr;        // dispatch block: job table, lengths, residues, workspaces
    uint64_t block_bytes = 0;
    // The slot's dispatch blocks live in one arena that only grows: a slot
    // runs one dispatch at a time, and a fresh multi-GB stream-ordered
    // allocation per dispatch cost the scheduler thread ~80 ms of mapping.
    void* arena = nullptr;
    uint64_t arena_cap = 0;
    void* host = nullptr;         // pinned: lengths + residues + error word
    uint64_t host_cap = 0;
    uint64_t t_start = 0;         // when the running dispatch was enqueued
};

}  // namespace b2m

using namespace b2m;

struct b2m_server {
    Context* c = nullptr;
    b2m_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> pending;
    std::unordered_map<uint64_t, Req> reqs;
    uint64_t next_id = 1;
    uint64_t used = 0;  // budget bytes held
    bool stopping = false;
    std::vector<Slot> slots;
    cudaStream_t release_stream = nullptr;
    std::thread th;
    b2m_server_stats st{};
};

namespace b2m {

// Launch one dispatch of the given requests on slot k (requests already admitted).
// `rs` are copies of the admitted requests; the owned buffers allocated here
// are written into the copies and published by the caller under the lock.
static cudaError_t launch_dispatch(b2m_server* S, Slot& sl, std::vector<Req>& rv) {
    std::vector<Req*> rs(rv.size());
    for (size_t i = 0; i < rv.size(); ++i) rs[i] = &rv[i];
    cudaStream_t s = sl.s;
    cudaError_t e = cudaSuccess;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    const size_t n = rs.size();
    // Owned buffers (generated operands, server-side outputs).
    for (Req* q : rs) {
        if (q->own_a && (e = cudaMallocAsync(&q->a, 4 * q->r.na, s)) != cudaSuccess) return e;
        if (q->own_b && (e = cudaMallocAsync(&q->b, 4 * q->r.nb, s)) != cudaSuccess) return e;
        if (q->own_out && (e = cudaMallocAsync(&q->out, 4 * (q->r.na + q->r.nb), s)) != cudaSuccess) return e;
        if (q->own_a && (e = launch_gen_operand(s, q->r.seed_a, q->r.na, q->r.kind, q->a)) != cudaSuccess) return e;
        if (q->own_b && (e = launch_gen_operand(s, q->r.seed_b, q->r.nb, q->r.kind, q->b)) != cudaSuccess) return e;
    }
    // Dispatch block: [job table][lengths][residues][buffers][carry scratch].
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return rs[x]->pts > rs[y]->pts; });
    const uint64_t tab = al(n * sizeof(ProdJob)), lens = al(n * 8), res = al(n * RES_WORDS * 8);
    uint64_t bufs = 0, scr = 0;
    for (Req* q : rs)
        if (q->pts > (1ull << SMALL_MAX_LOGN)) {
            bufs += 2 * 8 * q->pts;
            scr += al(carry_scratch_bytes_n(q->pts));
        }
    sl.block_bytes = tab + lens + res + bufs + scr;
    if (sl.block_bytes > sl.arena_cap) {
        // grow to at least twice the old size (256 MiB granules; the previous
        // dispatch on this slot has completed, so its arena can go): every
        // growth maps fresh device memory, which costs the scheduler thread
        // time proportional to its size, so growth steps must be few
        const uint64_t gran = 256ull << 20;
        const uint64_t cap = (std::max<uint64_t>(sl.block_bytes, 2 * sl.arena_cap) + gran - 1) & ~(gran - 1);
        if (sl.arena) {
            cudaFreeAsync(sl.arena, s);
            budget_release(S->c, sl.arena_cap);
            sl.arena = nullptr;
            sl.arena_cap = 0;
        }
        if (!budget_reserve(S->c, cap)) return cudaErrorMemoryAllocation;
        if ((e = cudaMallocAsync(&sl.arena, cap, s)) != cudaSuccess) {
            budget_release(S->c, cap);
            return e;
        }
        sl.arena_cap = cap;
    }
    sl.block = sl.arena;
    unsigned char* base = static_cast<unsigned char*>(sl.block);
    ProdJob* djobs = reinterpret_cast<ProdJob*>(base);
    u64* dlens = reinterpret_cast<u64*>(base + tab);
    unsigned long long* dres = reinterpret_cast<unsigned long long*>(base + tab + lens);
    unsigned char* pbuf = base + tab + lens + res;
    unsigned char* pscr = pbuf + bufs;
    const uint64_t host_need = lens + res + 256;
    if (sl.host_cap < host_need) {
        if (sl.host) cudaFreeHost(sl.host);
        sl.host_cap = std::max<uint64_t>(host_need, 1 << 16);
        if ((e = cudaMallocHost(&sl.host, sl.host_cap)) != cudaSuccess) {
            sl.host = nullptr;
            sl.host_cap = 0;
            return e;
        }
    }
    // Host job table, sorted by transform length.
    std::vector<ProdJob> hj(n);
    for (size_t k = 0; k < n; ++k) {
        Req* q = rs[order[k]];
        ProdJob J{};
        J.a = q->a;
        J.b = q->b;
        J.out = q->out;
        J.na = q->r.na;
        J.nb = q->r.nb;
        J.out_len = reinterpret_cast<unsigned long long*>(dlens + k);
        if (q->pts > (1ull << SMALL_MAX_LOGN)) {
            const uint64_t nn = q->pts;
            J.bufA = reinterpret_cast<u64*>(pbuf);
            J.bufB = J.bufA + nn;
            pbuf += 16 * nn;
            J.slots = reinterpret_cast<LookbackSlot*>(pscr);
            J.ticket = reinterpret_cast<u32*>(pscr + (nn / CARRY_CHUNK) * sizeof(LookbackSlot));
            pscr += al(carry_scratch_bytes_n(nn));
        }
        hj[k] = J;
    }
    // The table is copied from pageable memory (the driver stages it).
    if ((e = cudaMemcpyAsync(djobs, hj.data(), n * sizeof(ProdJob), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(dres, 0, res, s)) != cudaSuccess) return e;
    if ((e = launch_batch_prep(s, djobs, (unsigned)n, reinterpret_cast<unsigned long long*>(pbuf), scr / 8)) !=
        cudaSuccess)
        return e;
    // Buckets: consecutive equal transform lengths.
    for (size_t k0 = 0; k0 < n;) {
        const uint64_t pts = rs[order[k0]]->pts;
        size_t k1 = k0;
        while (k1 < n && rs[order[k1]]->pts == pts && k1 - k0 < 65535) ++k1;
        Plan p = plan_for(S->c, rs[order[k0]]->logn, rs[order[k0]]->three);
        if ((e = twtable_ensure(S->c, p, s)) != cudaSuccess) return e;
        if ((e = launch_bucket(p, djobs + k0, (unsigned)(k1 - k0), S->c->tw, S->c->d_err, s)) != cudaSuccess) return e;
        // Residue check of the bucket's products, its grid sized to the
        // bucket's longest operands (not the dispatch's).
        uint64_t maxlen = 0;
        for (size_t k = k0; k < k1; ++k) maxlen = std::max<uint64_t>(maxlen, rs[order[k]]->r.na + rs[order[k]]->r.nb);
        const unsigned gx = (unsigned)((maxlen + 4095) / 4096);
        k_residues<<<dim3(gx, (unsigned)(k1 - k0)), 256, 0, s>>>(djobs + k0, dres + k0 * RES_WORDS);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        k0 = k1;
    }
    // Results to pinned host memory.
    unsigned char* h = static_cast<unsigned char*>(sl.host);
    if ((e = cudaMemcpyAsync(h, dlens, n * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(h + lens, dres, n * RES_WORDS * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(h + lens + res, S->c->d_err, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    sl.block = nullptr;  // the arena stays with the slot
    return cudaEventRecord(sl.ev, s);
}

static void scheduler(b2m_server* S) {
    cudaSetDevice(S->c->device);
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    while (true) {
        bool progressed = false;
        // 1. completions
        for (Slot& sl : S->slots) {
            if (!sl.busy) continue;
            cudaError_t q = cudaEventQuery(sl.ev);
            if (q == cudaErrorNotReady) continue;
            const unsigned char* h = static_cast<const unsigned char*>(sl.host);
            const size_t n = sl.ids.size();
            const uint64_t lens = al(n * 8);
            const uint64_t res = al(n * RES_WORDS * 8);
            const u32 derr = q == cudaSuccess ? *reinterpret_cast<const u32*>(h + lens + res) : 0;
            const uint64_t t = now_ns();
            std::lock_guard<std::mutex> lk(S->mu);
            for (size_t k = 0; k < n; ++k) {
                Req& r = S->reqs[sl.ids[k]];
                S->used -= r.ws_bytes;  // the slot's arena holds the device memory itself
                r.ws_bytes = 0;
                r.t_done = t;
                if (q != cudaSuccess) {
                    r.state = 3;
                    r.status = B2M_ERR_CUDA;
                    ++S->st.failed;
                    continue;
                }
                r.out_len = reinterpret_cast<const u64*>(h)[k];
                r.residues_ok = residues_match(reinterpret_cast<const unsigned long long*>(h + lens) + k * RES_WORDS);
                r.state = (derr || !r.residues_ok) ? 3 : 2;
                r.status = derr ? B2M_ERR_DEVICE_TIMEOUT : (r.residues_ok ? B2M_OK : B2M_ERR_CUDA);
                if (r.state == 2) ++S->st.completed;
                else ++S->st.failed;
            }
            sl.busy = false;
            sl.ids.clear();
            S->st.slot_busy_ns += t - sl.t_start;
            --S->st.inflight_dispatches;
            progressed = true;
            S->cv_done.notify_all();
        }
        // 2. admissions + dispatch on free slots
        for (Slot& sl : S->slots) {
            if (sl.busy) continue;
            std::vector<Req> rs;
            std::vector<uint64_t> ids;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                while (!S->pending.empty() && rs.size() < S->cfg.max_batch) {
                    Req& r = S->reqs[S->pending.front()];
                    const uint64_t need = r.own_bytes + r.ws_bytes;
                    if (S->used + need > S->cfg.hbm_budget_bytes) break;  // FIFO: wait for memory
                    if (!budget_reserve(S->c, r.own_bytes)) break;  // workspace: reserved by the arenas
                    S->used += need;
                    S->st.peak_bytes = std::max<uint64_t>(S->st.peak_bytes, S->used);
                    r.state = 1;
                    r.t_admit = now_ns();
                    ids.push_back(S->pending.front());
                    rs.push_back(r);
                    S->pending.pop_front();
                }
            }
            if (rs.empty()) break;
            const uint64_t t_enq = now_ns();
            cudaError_t e = launch_dispatch(S, sl, rs);
            const uint64_t t_enq_end = now_ns();
            std::lock_guard<std::mutex> lk(S->mu);
            for (size_t k = 0; k < rs.size(); ++k) {  // publish the owned buffers
                Req& r = S->reqs[ids[k]];
                r.a = rs[k].a;
                r.b = rs[k].b;
                r.out = rs[k].out;
            }
            if (e != cudaSuccess) {
                for (size_t k = 0; k < rs.size(); ++k) {
                    Req& r = S->reqs[ids[k]];
                    r.state = 3;
                    r.status = e == cudaErrorMemoryAllocation ? B2M_ERR_OUT_OF_MEMORY : B2M_ERR_CUDA;
                    r.t_done = now_ns();
                    S->used -= r.ws_bytes;
                    r.ws_bytes = 0;
                    ++S->st.failed;
                }
                cudaStreamSynchronize(sl.s);
                cudaGetLastError();
                S->cv_done.notify_all();
                continue;
            }
            // launch_dispatch sorted the jobs by size: record ids in that order
            std::vector<size_t> order(rs.size());
            for (size_t i = 0; i < order.size(); ++i) order[i] = i;
            std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return rs[x].pts > rs[y].pts; });
            sl.ids.resize(rs.size());
            for (size_t k = 0; k < order.size(); ++k) sl.ids[k] = ids[order[k]];
            sl.busy = true;
            sl.t_start = t_enq;
            S->st.host_dispatch_ns += t_enq_end - t_enq;
            ++S->st.inflight_dispatches;
            S->st.max_inflight_dispatches = std::max(S->st.max_inflight_dispatches, S->st.inflight_dispatches);
            ++S->st.dispatches;
            progressed = true;
        }
        std::unique_lock<std::mutex> lk(S->mu);
        bool any_busy = false;
        for (const Slot& sl : S->slots) any_busy |= sl.busy;
        if (S->stopping && S->pending.empty() && !any_busy) break;
        if (!progressed) S->cv_work.wait_for(lk, std::chrono::microseconds(any_busy ? 20 : 2000));
    }
}

}  // namespace b2m

extern "C" {

b2m_status b2m_gen_operand(uint64_t seed, uint64_t n, uint32_t kind, uint32_t* d_out, b2m_stream stream) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if ((n && !d_out) || kind > 1) return B2M_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    return cuda_status(launch_gen_operand(reinterpret_cast<cudaStream_t>(stream), seed, n, kind, d_out),
                       "operand generator");
}

b2m_status b2m_server_start(const b2m_server_config* cfg, b2m_server** out) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (!out) return B2M_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    b2m_server* S = new b2m_server();
    S->c = c;
    if (cfg) S->cfg = *cfg;
    if (S->cfg.hbm_budget_bytes == 0) S->cfg.hbm_budget_bytes = c->budget / 2;
    if (S->cfg.streams == 0) S->cfg.streams = 4;
    if (S->cfg.max_batch == 0) S->cfg.max_batch = 256;
    if (S->cfg.max_pending == 0) S->cfg.max_pending = 1u << 20;
    S->slots.resize(S->cfg.streams);
    for (Slot& sl : S->slots) {
        cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
    }
    cudaStreamCreateWithFlags(&S->release_stream, cudaStreamNonBlocking);
    // Twiddle tables of every transform length the budget can admit, built
    // now: building one later means a cudaMalloc (which synchronises the
    // device) and a stream wait inside the scheduler, stalling every
    // dispatch in flight.
    for (int logn = SMALL_MAX_LOGN + 1; logn <= MAX_LOGN; ++logn) {
        const uint64_t pts = 1ull << logn;
        if (2 * 8 * pts > S->cfg.hbm_budget_bytes) break;
        if (twtable_ensure(c, plan_for(c, logn), S->release_stream) != cudaSuccess) break;
        // the sub-transform plan of 3 * 2^logn points may differ
        if (6 * 8 * pts <= S->cfg.hbm_budget_bytes &&
            twtable_ensure(c, plan_for(c, logn, 1), S->release_stream) != cudaSuccess)
            break;
    }
    // Each slot's arena starts at an equal share of half the budget (at most
    // 4 GiB), so that typical dispatches never grow it.
    {
        const uint64_t gran = 256ull << 20;
        uint64_t share = std::min<uint64_t>(S->cfg.hbm_budget_bytes / (2 * S->cfg.streams), 4ull << 30) & ~(gran - 1);
        for (Slot& sl : S->slots) {
            if (share == 0 || !budget_reserve(c, share)) break;
            if (cudaMallocAsync(&sl.arena, share, sl.s) != cudaSuccess) {
                budget_release(c, share);
                sl.arena = nullptr;
                cudaGetLastError();
                break;
            }
            sl.arena_cap = share;
        }
    }
    S->th = std::thread(scheduler, S);
    *out = S;
    return B2M_OK;
}

b2m_status b2m_server_submit(b2m_server* S, const b2m_request* req, uint64_t* ticket) {
    if (!S || !req || !ticket) return B2M_ERR_INVALID_ARGUMENT;
    const b2m_request& r = *req;
    if (r.na == 0 || r.nb == 0 || r.kind > 1 || (r.out && r.out_cap < r.na + r.nb)) return B2M_ERR_INVALID_ARGUMENT;
    int logn;
    b2m_status st = check_sizes(r.na, r.nb, &logn);
    if (st != B2M_OK) return st;
    Req q;
    q.r = r;
    choose_length(2 * (r.na + r.nb), &q.logn, &q.three);
    q.pts = (q.three ? 3ull : 1ull) << q.logn;
    q.own_a = r.a == nullptr;
    q.own_b = r.b == nullptr;
    q.own_out = r.out == nullptr;
    q.a = const_cast<u32*>(r.a);
    q.b = const_cast<u32*>(r.b);
    q.out = r.out;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    q.own_bytes = (q.own_a ? al(4 * r.na) : 0) + (q.own_b ? al(4 * r.nb) : 0) + (q.own_out ? al(4 * (r.na + r.nb)) : 0);
    q.ws_bytes = (q.pts > (1ull << SMALL_MAX_LOGN) ? 2 * 8 * q.pts + al(carry_scratch_bytes_n(q.pts)) : 0) + 256;
    if (q.own_bytes + q.ws_bytes > S->cfg.hbm_budget_bytes) {
        set_error("request larger than the server's HBM budget");
        return B2M_ERR_OUT_OF_MEMORY;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) return B2M_ERR_SHUTDOWN;
    if (S->pending.size() >= S->cfg.max_pending) return B2M_ERR_QUEUE_FULL;
    q.t_submit = now_ns();
    const uint64_t id = S->next_id++;
    S->reqs.emplace(id, q);
    S->pending.push_back(id);
    ++S->st.submitted;
    S->st.max_queue = std::max<uint64_t>(S->st.max_queue, S->pending.size());
    *ticket = id;
    S->cv_work.notify_one();
    return B2M_OK;
}

static void fill_result(const Req& r, b2m_result* res) {
    res->state = r.state;
    res->status = r.status;
    res->out = r.out;
    res->out_len = r.out_len;
    res->t_submit_ns = r.t_submit;
    res->t_admit_ns = r.t_admit;
    res->t_done_ns = r.t_done;
    res->residues_ok = r.residues_ok;
}

b2m_status b2m_server_poll(b2m_server* S, uint64_t ticket, b2m_result* res) {
    if (!S || !res) return B2M_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return B2M_ERR_NOT_FOUND;
    fill_result(it->second, res);
    return B2M_OK;
}

b2m_status b2m_server_wait(b2m_server* S, uint64_t ticket, double timeout_s, b2m_result* res) {
    if (!S || !res) return B2M_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(S->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    while (true) {
        auto it = S->reqs.find(ticket);
        if (it == S->reqs.end()) return B2M_ERR_NOT_FOUND;
        if (it->second.state >= 2) {
            fill_result(it->second, res);
            return B2M_OK;
        }
        if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
            fill_result(S->reqs[ticket], res);
            return res->state >= 2 ? B2M_OK : B2M_ERR_DEVICE_TIMEOUT;
        }
    }
}

b2m_status b2m_server_release(b2m_server* S, uint64_t ticket) {
    if (!S) return B2M_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return B2M_ERR_NOT_FOUND;
    Req& r = it->second;
    if (r.state < 2) return B2M_ERR_INVALID_ARGUMENT;  // still queued or on the GPU
    cudaSetDevice(S->c->device);
    if (r.own_a && r.a) cudaFreeAsync(r.a, S->release_stream);
    if (r.own_b && r.b) cudaFreeAsync(r.b, S->release_stream);
    if (r.own_out && r.out) cudaFreeAsync(r.out, S->release_stream);
    if (r.state == 2 || r.state == 3) {
        S->used -= r.own_bytes;
        budget_release(S->c, r.own_bytes);
    }
    S->reqs.erase(it);
    S->cv_work.notify_one();
    return B2M_OK;
}

b2m_status b2m_server_get_stats(b2m_server* S, b2m_server_stats* out) {
    if (!S || !out) return B2M_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->queued = S->pending.size();
    out->bytes_in_use = S->used;
    return B2M_OK;
}

b2m_status b2m_server_stop(b2m_server* S) {
    if (!S) return B2M_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        S->cv_work.notify_all();
    }
    if (S->th.joinable()) S->th.join();
    cudaSetDevice(S->c->device);
    for (auto& kv : S->reqs) {
        Req& r = kv.second;
        if (r.own_a && r.a) cudaFreeAsync(r.a, S->release_stream);
        if (r.own_b && r.b) cudaFreeAsync(r.b, S->release_stream);
        if (r.own_out && r.out) cudaFreeAsync(r.out, S->release_stream);
        budget_release(S->c, r.own_bytes);
    }
    cudaStreamSynchronize(S->release_stream);
    for (Slot& sl : S->slots) {
        cudaStreamSynchronize(sl.s);
        if (sl.arena) {
            cudaFree(sl.arena);
            budget_release(S->c, sl.arena_cap);
        }
        if (sl.host) cudaFreeHost(sl.host);
        cudaEventDestroy(sl.ev);
        cudaStreamDestroy(sl.s);
    }
    cudaStreamDestroy(S->release_stream);
    delete S;
    return B2M_OK;
}

}  // extern "C"
