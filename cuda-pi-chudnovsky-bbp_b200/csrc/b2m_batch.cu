// b2m_batch.cu -- batched products of mixed sizes (include/b2m.h, b2m_batch_*).
//
// Reference counterpart: none as an API. The reference's binary-splitting
// tree (src/chudnovsky.cpp:64-102) issues its products one at a time through
// mul_dispatch (src/bignum.cpp:204-232), each GPU product paying its own
// allocation, copies and ~2 log2 N launches (src/ntt_cuda.cu:179-243).
//
// A batch buckets its jobs by transform length. A bucket is one set of
// launches whose grid's second dimension runs over the bucket's jobs (one CTA
// per job for transform lengths <= 2^13), so thousands of small products fill
// the GPU instead of one SM each. Buckets are independent and run on forked
// streams; the whole sequence (prep kernel, buckets, join) can be captured
// once into a CUDA graph and replayed. With B2M_BATCH_AUTOTUNE the pass split
// and tile size of every multi-pass bucket is chosen by timing the candidates
// on the bucket itself; choices are remembered per transform length.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <vector>

#include "b2m.h"
#include "b2m_context.h"
#include "b2m_internal.h"

namespace b2m {

struct Bucket {
    int logn = 0;
    Plan plan;
    unsigned first = 0;  // index of the bucket's first job in the device table
    unsigned njobs = 0;
};

}  // namespace b2m

using namespace b2m;

struct b2m_batch {
    Context* ctx = nullptr;
    std::vector<Bucket> buckets;
    unsigned njobs_all = 0;           // jobs in the device table (incl. empty ones)
    void* dmem = nullptr;
    uint64_t dbytes = 0;
    ProdJob* djobs = nullptr;
    unsigned long long* scratch = nullptr;
    uint64_t scratch_words = 0;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev;      // ev[0]: fork, ev[1..]: per side stream join
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace b2m {

static cudaError_t enqueue_batch(b2m_batch* bt, cudaStream_t s) {
    Context* c = bt->ctx;
    cudaError_t e;
    if ((e = launch_batch_prep(s, bt->djobs, bt->njobs_all, bt->scratch, bt->scratch_words)) != cudaSuccess)
        return e;
    if ((e = cudaEventRecord(bt->ev[0], s)) != cudaSuccess) return e;
    const size_t ns = bt->side.size();
    for (size_t i = 0; i < ns; ++i)
        if ((e = cudaStreamWaitEvent(bt->side[i], bt->ev[0], 0)) != cudaSuccess) return e;
    // Largest buckets first, spread round-robin over the side streams.
    for (size_t i = 0; i < bt->buckets.size(); ++i) {
        const Bucket& b = bt->buckets[i];
        cudaStream_t st = bt->side[i % ns];
        if ((e = launch_bucket(b.plan, bt->djobs + b.first, b.njobs, c->tw, c->d_err, st)) != cudaSuccess) return e;
    }
    for (size_t i = 0; i < ns; ++i) {
        if ((e = cudaEventRecord(bt->ev[1 + i], bt->side[i])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, bt->ev[1 + i], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

static void free_batch(b2m_batch* bt) {
    if (!bt) return;
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    for (cudaStream_t s : bt->side) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    for (cudaEvent_t e : bt->ev) cudaEventDestroy(e);
    if (bt->dmem) {
        cudaFree(bt->dmem);
        budget_release(bt->ctx, bt->dbytes);
    }
    delete bt;
}

// Time every candidate plan of bucket b on its own jobs; keep the fastest.
static cudaError_t autotune_bucket(b2m_batch* bt, Bucket& b, cudaStream_t s) {
    Context* c = bt->ctx;
    if (b.plan.three) return cudaSuccess;  // radix-3 buckets run the sub-length's current plan
    {
        std::lock_guard<std::mutex> lk(c->tune_mu);
        if (c->has_tuned[b.logn]) {
            b.plan = c->tuned[b.logn];
            return cudaSuccess;
        }
    }
    std::vector<Plan> cands = plan_candidates(b.logn);
    if (cands.size() < 2) return cudaSuccess;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best = 1e30f;
    Plan best_p = b.plan;
    cudaError_t e = cudaSuccess;
    for (const Plan& p : cands) {
        float ms_sum = 0;
        if ((e = twtable_ensure(c, p, s)) != cudaSuccess) break;
        for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
            launch_batch_prep(s, bt->djobs, bt->njobs_all, bt->scratch, bt->scratch_words);
            cudaEventRecord(t0, s);
            e = launch_bucket(p, bt->djobs + b.first, b.njobs, c->tw, c->d_err, s);
            cudaEventRecord(t1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(t1);
            float ms = 0;
            cudaEventElapsedTime(&ms, t0, t1);
            if (rep > 0) ms_sum += ms;  // first run warms up
        }
        if (e != cudaSuccess) break;
        if (ms_sum < best) {
            best = ms_sum;
            best_p = p;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (e != cudaSuccess) return e;
    b.plan = best_p;
    set_tuned(c, b.logn, best_p);
    return cudaSuccess;
}

}  // namespace b2m

extern "C" {

b2m_status b2m_batch_create(const b2m_job* jobs, uint64_t njobs, uint32_t flags, b2m_batch** out) {
    Context* c = ctx();
    if (!c) return B2M_ERR_NOT_INITIALIZED;
    if (!out || (njobs && !jobs) || njobs > (1u << 24) || (flags & ~(B2M_BATCH_GRAPH | B2M_BATCH_AUTOTUNE)))
        return B2M_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    // Validate and bucket.
    std::map<uint64_t, std::vector<unsigned>> by_pts;  // transform points -> job indices
    std::vector<unsigned> empty;
    for (uint64_t i = 0; i < njobs; ++i) {
        const b2m_job& j = jobs[i];
        if ((j.na && !j.a) || (j.nb && !j.b)) return B2M_ERR_INVALID_ARGUMENT;
        if (j.na == 0 || j.nb == 0) {
            empty.push_back((unsigned)i);
            continue;
        }
        if (!j.out) return B2M_ERR_INVALID_ARGUMENT;
        if (j.out_cap < j.na + j.nb) return B2M_ERR_OUTPUT_TOO_SMALL;
        int logn, three;
        b2m_status st = check_sizes(j.na, j.nb, &logn);
        if (st != B2M_OK) return st;
        choose_length(2 * (j.na + j.nb), &logn, &three);
        by_pts[(three ? 3ull : 1ull) << logn].push_back((unsigned)i);
    }
    cudaSetDevice(c->device);
    b2m_batch* bt = new b2m_batch();
    bt->ctx = c;
    // Device layout: [job table][len slots][transform buffers][carry scratch].
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    const uint64_t tab = al(njobs * sizeof(ProdJob));
    const uint64_t lens = al(njobs * sizeof(uint64_t));
    uint64_t bufs = 0, scr = 0;
    for (auto& kv : by_pts) {
        if (kv.first <= (1ull << SMALL_MAX_LOGN)) continue;
        bufs += kv.second.size() * 2 * 8 * kv.first;
        scr += kv.second.size() * al(carry_scratch_bytes_n(kv.first));
    }
    bt->dbytes = tab + lens + bufs + scr;
    if (!budget_reserve(c, bt->dbytes)) {
        delete bt;
        set_error("HBM budget exhausted by the batch workspace");
        return B2M_ERR_OUT_OF_MEMORY;
    }
    cudaError_t e = cudaMalloc(&bt->dmem, bt->dbytes);
    if (e != cudaSuccess) {
        budget_release(c, bt->dbytes);
        bt->dmem = nullptr;
        free_batch(bt);
        return cuda_status(e, "cudaMalloc(batch workspace)");
    }
    unsigned char* base = static_cast<unsigned char*>(bt->dmem);
    bt->djobs = reinterpret_cast<ProdJob*>(base);
    uint64_t* dlens = reinterpret_cast<uint64_t*>(base + tab);
    unsigned char* pbuf = base + tab + lens;
    unsigned char* pscr = pbuf + bufs;
    bt->scratch = reinterpret_cast<unsigned long long*>(pscr);
    bt->scratch_words = scr / 8;
    // Host job table in bucket order (largest transforms first), then empties.
    std::vector<ProdJob> hj;
    hj.reserve(njobs);
    auto mk = [&](unsigned i) {
        const b2m_job& j = jobs[i];
        ProdJob p{};
        p.a = j.a;
        p.b = j.b;
        p.out = j.out;
        p.na = j.na;
        p.nb = j.nb;
        p.out_len = reinterpret_cast<unsigned long long*>(j.out_len ? j.out_len : dlens + hj.size());
        return p;
    };
    constexpr unsigned MAX_GRID_Y = 65535;  // a bucket launch covers at most this many jobs
    for (auto it = by_pts.rbegin(); it != by_pts.rend(); ++it) {
      const uint64_t n = it->first;
      const int three = (n & (n - 1)) ? 1 : 0;  // 3 * 2^k is no power of two
      const uint64_t sub = three ? n / 3 : n;      // the (sub-)transform length 2^k
      int lg = 0;
      while ((1ull << lg) < sub) ++lg;
      for (size_t off = 0; off < it->second.size(); off += MAX_GRID_Y) {
        Bucket b;
        b.logn = lg;
        b.plan = plan_for(c, b.logn, three);
        b.first = (unsigned)hj.size();
        b.njobs = (unsigned)std::min<size_t>(MAX_GRID_Y, it->second.size() - off);
        for (size_t k = off; k < off + b.njobs; ++k) {
            const unsigned i = it->second[k];
            ProdJob p = mk(i);
            if (n > (1ull << SMALL_MAX_LOGN)) {
                p.bufA = reinterpret_cast<u64*>(pbuf);
                p.bufB = p.bufA + n;
                pbuf += 2 * 8 * n;
                p.slots = reinterpret_cast<LookbackSlot*>(pscr);
                p.ticket = reinterpret_cast<u32*>(pscr + (n / CARRY_CHUNK) * sizeof(LookbackSlot));
                pscr += al(carry_scratch_bytes_n(n));
            }
            hj.push_back(p);
        }
        bt->buckets.push_back(b);
      }
    }
    for (unsigned i : empty) hj.push_back(mk(i));
    bt->njobs_all = (unsigned)hj.size();
    if (!hj.empty() && (e = cudaMemcpy(bt->djobs, hj.data(), hj.size() * sizeof(ProdJob), cudaMemcpyHostToDevice)) != cudaSuccess) {
        free_batch(bt);
        return cuda_status(e, "cudaMemcpy(job table)");
    }
    const size_t nside = std::max<size_t>(1, std::min<size_t>(4, bt->buckets.size()));
    bt->side.resize(nside);
    bt->ev.resize(nside + 1);
    for (auto& s : bt->side) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    for (auto& ev : bt->ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (flags & B2M_BATCH_AUTOTUNE) {
        for (Bucket& b : bt->buckets)
            if ((e = autotune_bucket(bt, b, bt->side[0])) != cudaSuccess) {
                free_batch(bt);
                return cuda_status(e, "autotune");
            }
    }
    for (Bucket& b : bt->buckets)  // twiddle tables exist before any capture
        if ((e = twtable_ensure(c, b.plan, bt->side[0])) != cudaSuccess) {
            free_batch(bt);
            return cuda_status(e, "twiddle table");
        }
    if (flags & B2M_BATCH_GRAPH) {
        cudaStream_t cs;
        cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t e2 = enqueue_batch(bt, cs);
            e = cudaStreamEndCapture(cs, &bt->graph);
            if (e2 != cudaSuccess) e = e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&bt->exec, bt->graph, 0);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) {
            free_batch(bt);
            return cuda_status(e, "graph capture");
        }
    }
    *out = bt;
    return B2M_OK;
}

b2m_status b2m_batch_launch(b2m_batch* bt, b2m_stream stream) {
    if (!bt) return B2M_ERR_INVALID_ARGUMENT;
    cudaSetDevice(bt->ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = bt->exec ? cudaGraphLaunch(bt->exec, s) : enqueue_batch(bt, s);
    return cuda_status(e, "batch launch");
}

b2m_status b2m_batch_destroy(b2m_batch* bt) {
    if (!bt) return B2M_OK;
    cudaSetDevice(bt->ctx->device);
    cudaDeviceSynchronize();
    free_batch(bt);
    return B2M_OK;
}

b2m_status b2m_mul_batch(const b2m_job* jobs, uint64_t njobs, b2m_stream stream) {
    b2m_batch* bt = nullptr;
    b2m_status st = b2m_batch_create(jobs, njobs, 0, &bt);
    if (st != B2M_OK) return st;
    st = b2m_batch_launch(bt, stream);
    cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
    b2m_batch_destroy(bt);
    return st;
}

}  // extern "C"
