// b2m_context.h -- the process-wide library context (one device).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "b2m.h"
#include "b2m_internal.h"

namespace b2m {

struct Context {
    int device = -1;
    int sm_count = 0;
    uint64_t budget = 0;                 // bytes the library may hold on the device
    std::atomic<uint64_t> in_use{0};     // bytes currently reserved against the budget
    u64* d_tables = nullptr;             // dtw | u1 | u2, resident
    RootTables tw{};
    u32* d_err = nullptr;                // sticky device error word (bounded waits)
    cudaStream_t hstream = nullptr;      // stream of the host-buffer entry point
    cudaStream_t hcopy = nullptr;        // its second operand's H2D copy (overlaps operand A's transform)
    cudaEvent_t hev_a = nullptr, hev_b = nullptr;  // operand A / operand B resident
    std::mutex host_mu;                  // serialises b2m_mul_host (shared buffers)
    void* host_dev = nullptr;            // device buffers of b2m_mul_host, grown on demand
    uint64_t host_dev_cap = 0;
    // Inter-pass twiddle tables (twtable_ensure), keyed by (logm, logr).
    struct TwTable {
        int logm, logr;
        u64* fwd;
        u64* inv;
        uint64_t bytes;
        // inv times 2^-logm, for the table's use as pass 0 of a 2^logm-point
        // transform (the inverse pass 0 then applies N^-1 for free); built by
        // twtable_ensure for pass 0, null until then or if the budget is short
        u64* inv0 = nullptr;
        uint64_t inv0_bytes = 0;
    };
    std::mutex twt_mu;
    std::vector<TwTable> twt;
    // Autotuned plan per transform length (b2m_autotune, batch autotune);
    // used by every product of that length once set.
    std::mutex tune_mu;
    Plan tuned[MAX_LOGN + 1];
    bool has_tuned[MAX_LOGN + 1];
    Context() {
        for (int i = 0; i <= MAX_LOGN; ++i) has_tuned[i] = false;
    }
};

// The plan products of (sub-)transform length 2^logn use: the tuned one if
// any, else the default (three: the radix-3 products' default).
inline Plan plan_for(Context* c, int logn, int three = 0) {
    std::lock_guard<std::mutex> lk(c->tune_mu);
    Plan p = c->has_tuned[logn] ? c->tuned[logn] : make_plan(logn, three);
    p.three = three;
    return p;
}
// The plan of an na x nb product: 2^L points, or 3 * 2^(L-2) when that holds
// the 2(na + nb) digits (choose_length), its sub-transform the tuned or
// default plan of that length.
inline Plan product_plan(Context* c, uint64_t na, uint64_t nb) {
    int logn = 0, three = 0;
    choose_length(2 * (na + nb), &logn, &three);
    return plan_for(c, logn, three);
}
inline void set_tuned(Context* c, int logn, const Plan& p) {
    std::lock_guard<std::mutex> lk(c->tune_mu);
    c->tuned[logn] = p;
    c->has_tuned[logn] = true;
}

extern Context* g_ctx;
extern std::mutex g_ctx_mu;

Context* ctx();
void set_error(const std::string& msg);
b2m_status cuda_status(cudaError_t e, const char* what);
int ilog2_pow2(uint64_t n);
uint64_t ntt_length_of(uint64_t na, uint64_t nb);
bool budget_reserve(Context* c, uint64_t bytes);
void budget_release(Context* c, uint64_t bytes);
b2m_status check_sizes(uint64_t na, uint64_t nb, int* logn);

// Reads and clears the device error word (caller has synchronised).
inline b2m_status take_device_error(Context* c) {
    u32 h = 0;
    cudaError_t e = cudaMemcpy(&h, c->d_err, sizeof(u32), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemcpy(error word)");
    if (h) {
        cudaMemset(c->d_err, 0, sizeof(u32));
        set_error("carry lookback wait exceeded its bound");
        return B2M_ERR_DEVICE_TIMEOUT;
    }
    return B2M_OK;
}

}  // namespace b2m
