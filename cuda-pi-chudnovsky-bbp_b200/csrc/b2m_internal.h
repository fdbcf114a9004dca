// b2m_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "gl.cuh"

namespace b2m {

constexpr int MAX_LOGN = 30;      // coefficients stay below p for N <= 2^32
constexpr int SMALL_MAX_LOGN = 13; // one CTA holds both transforms up to here
constexpr int CARRY_THREADS = 256;
constexpr int CARRY_G = 16;       // coefficients per thread in the carry kernel
constexpr int CARRY_CHUNK = CARRY_THREADS * CARRY_G;
// Dynamic shared memory each kernel may request: the largest tile (2^14
// elements + padding, ~133 KB) fits, and the opt-in limit (227 KB on sm_100)
// leaves room for the kernels' static shared memory.
constexpr int kMaxDynSmem = 200 * 1024;

// Device root tables, built once per device and kept resident:
//   dtw[2^l + e] = w_{2^l}^e, l in [0, 14]          (2^15 entries)
//   u1[e] = RHO^e, u2[e] = RHO^(e * 2^16), e < 2^16  (2 x 2^16 entries)
struct RootTables {
    const u64* dtw;
    const u64* u1;
    const u64* u2;
};

// Pass plan of one transform length.
struct Plan {
    int logn = 0;
    int npass = 0;   // 0 = single-CTA multiply
    int logr[3] = {0, 0, 0};
    int logc[3] = {0, 0, 0};
    // 1: 3 * 2^logn points -- a radix-3 step (ntt_radix3.cu) around three
    // 2^logn-point transforms that run the passes above (npass >= 2).
    int three = 0;
};

// Points of a plan's transform, and the workspace and carry scratch a
// product with that plan needs.
inline uint64_t plan_points(const Plan& p) { return (p.three ? 3ull : 1ull) << p.logn; }
uint64_t carry_scratch_bytes_n(uint64_t points);
uint64_t workspace_bytes_plan(const Plan& p);
// A transform of 3 * 2^k points is used when k >= RADIX3_MIN_LOG and it still
// holds the product's digits (fewer points than the next power of two).
constexpr int RADIX3_MIN_LOG = 14;
// Log2 of the sub-transform and the radix-3 choice for `digits` points of
// convolution output (2na + 2nb): three = 1 when 3 * 2^(L-2) >= digits.
void choose_length(uint64_t digits, int* logn, int* three);

// The default plan of a 2^logn-point transform, or (three) of the 2^logn-point
// sub-transforms of a 3 * 2^logn-point product.
Plan make_plan(int logn, int three = 0);
Plan make_plan_custom(int logn, int r0, int tile);
Plan make_plan_split(int logn, const int* r, int npass, int tile);
std::vector<Plan> plan_candidates(int logn);

// Per-product workspace layout (bytes): two N-element u64 arrays plus the
// carry scratch (lookback slots, ticket, out_len staging).
// One chunk's published carry state. `word` is 0 until the chunk publishes;
// then (value << 2) | state, state 1: aggregate independent of the carry-in
// (value = its carry-out), 3: aggregate with threshold agg_t (value = the
// carry-out below it), 2: inclusive carry-out. Carry-outs are below 2^49.
struct LookbackSlot {
    u64 word, agg_t;
};
uint64_t workspace_bytes_for(int logn);

// One product's device pointers. Batched launches give kernels a table of
// these and each CTA reads jobs[blockIdx.y] (blockIdx.x for the single-CTA
// kernel); single products pass a null table and plain arguments.
struct ProdJob {
    const u32* a;
    const u32* b;
    u32* out;
    unsigned long long* out_len;  // may be null
    u64 na, nb;
    u64* bufA;                    // transform buffers of N elements each
    u64* bufB;
    LookbackSlot* slots;          // carry scratch: N / CARRY_CHUNK slots + ticket
    u32* ticket;
};
uint64_t carry_scratch_bytes(int logn);

// Optional tracing of a launch sequence: an event is recorded on the stream
// before every kernel and once after the last one.
struct Tracer {
    static constexpr int CAP = 16;
    cudaEvent_t ev[CAP + 1];
    uint32_t kind[CAP], logr[CAP];
    int n = 0;
    void mark(cudaStream_t s, uint32_t k, uint32_t r) {
        if (n < CAP) {
            kind[n] = k;
            logr[n] = r;
            cudaEventRecord(ev[n], s);
            ++n;
        }
    }
    void end(cudaStream_t s) { cudaEventRecord(ev[n], s); }
};

// Kernel launch sequence for one product on `stream`.
//   a, b: device limbs; out: na+nb limbs; out_len: device u64 (may be null).
//   ws: workspace of workspace_bytes_for(logn) bytes; err: device error word.
// All passes, the carry and the bookkeeping of one size bucket of a batch:
// `njobs` products of plan p whose pointers are in the device table `jobs`.
// a_ready: every job's bufA already holds the finished forward spectrum of
// its operand a under plan p (a spectrum several products share: the kernels
// only read bufA), so a's forward passes are skipped. Plans of one CTA
// (npass == 0) transform both operands themselves and ignore it.
cudaError_t launch_bucket(const Plan& p, const ProdJob* jobs, unsigned njobs, const RootTables& tw, u32* err,
                          cudaStream_t s, bool a_ready = false);
// Only the forward transform of operand a of each job, into its bufA
// (npass >= 1): the spectrum that later launch_bucket(..., a_ready) calls read.
cudaError_t launch_bucket_spectrum(const Plan& p, const ProdJob* jobs, unsigned njobs, const RootTables& tw,
                                   cudaStream_t s);

// Grid-wide passes over u32 limbs (b2m_bigops.cu), ordered on s:
// out = a +- b mod 2^(32 n) (limbs of a at or past la read as 0, likewise b;
// out may be a or b) with the carry or borrow out in *flag, using `scratch`
// of addsub_scratch_bytes(n) bytes; *out = the largest k + 1 with a[k] != 0
// (launch_top) or a[k] != b[k] (launch_top_diff) for k < n, into a word the
// caller zeroed.
uint64_t addsub_scratch_bytes(uint64_t n);
cudaError_t launch_addsub(const u32* a, uint64_t la, const u32* b, uint64_t lb, uint64_t n, int sub, u32* out,
                          void* scratch, u32* flag, cudaStream_t s);
cudaError_t launch_top(const u32* a, uint64_t n, unsigned long long* out, cudaStream_t s);
cudaError_t launch_top_diff(const u32* a, const u32* b, uint64_t n, unsigned long long* out, cudaStream_t s);

// Zero `nwords` u64 of carry scratch and every job's out_len.
cudaError_t launch_batch_prep(cudaStream_t s, const ProdJob* jobs, unsigned njobs, unsigned long long* scratch,
                              u64 nwords);
// Seeded operand generator (same sequence as b2m_gen_operand).
cudaError_t launch_gen_operand(cudaStream_t s, u64 seed, u64 n, u32 kind, u32* out);

cudaError_t launch_product(const u32* a, uint64_t na, const u32* b, uint64_t nb, u32* out,
                           uint64_t* out_len, void* ws, const Plan& plan, const RootTables& tw,
                           u32* err, cudaStream_t stream, Tracer* tr = nullptr,
                           cudaEvent_t b_ready = nullptr);  // operand B waited for just before its transform
// Kernels one product launches under plan p.
int plan_launches(const Plan& p);

// One-time per-device kernel attribute setup (dynamic shared memory limits).
cudaError_t configure_kernels();

// Launch geometry of one pass (see make_plan / pass_geo in ntt_launch.cu).
struct PassGeo {
    int logr = 0, logc = 0, logs = 0, logm = 0;
    unsigned grid = 0, block = 0;
    size_t smem = 0;
    // Inter-pass twiddles of this pass in data order (w_M^(bitrev(row) * c)
    // at (row << logs) + c), forward and inverse, when a table exists for
    // (logm, logr); null: the kernels build each twiddle from u1 * u2.
    const u64* tfwd = nullptr;
    const u64* tinv = nullptr;
    // Pass 0 only: the inverse table times 2^-logm (see Context::TwTable),
    // when it exists; an inverse pass 0 run with it leaves the coefficients
    // already scaled by the sub-transform's 2^-logn.
    const u64* tinv0 = nullptr;
    // Radix-3 plans: grid z runs over the three sub-transforms, zstride
    // elements apart (1 and 0 otherwise).
    unsigned zdim = 1;
    u64 zstride = 0;
};
PassGeo pass_geo(const Plan& p, int k);

// Inter-pass twiddle tables, per (logm, logr), kept for the context's life.
// twtable_ensure builds the ones plan p needs (only for M >= 2^TWT_MIN_LOGM,
// never while `s` is capturing, skipped if the budget is short); pass_geo
// only looks them up, so launch paths that must not allocate still use
// tables that exist.
constexpr int TWT_MIN_LOGM = 12;
struct Context;
cudaError_t twtable_ensure(Context* c, const Plan& p, cudaStream_t s);
void twtable_free_all(Context* c);

// Per-family launchers (ntt_fam_*.cu, ntt_carry.cu); each dispatches on the
// radix exponent to the matching template instantiation.
// `jobs` (device table, may be null) and `njobs` select batched launches:
// grid.y (grid.x for the single-CTA kernel) runs over the jobs.
cudaError_t launch_fwd_first(int logr, const PassGeo& g, cudaStream_t s, const u32* limbs, u64 ndig, u64* out,
                             const RootTables& tw, const ProdJob* jobs = nullptr, unsigned njobs = 1,
                             int operand = 0);
cudaError_t launch_fwd_mid(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw,
                           const ProdJob* jobs = nullptr, unsigned njobs = 1, int operand = 0);
cudaError_t launch_inv_mid(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw,
                           const ProdJob* jobs = nullptr, unsigned njobs = 1);
cudaError_t launch_fwd_last(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw,
                            const ProdJob* jobs = nullptr, unsigned njobs = 1);
cudaError_t launch_fused_last(int logr, const PassGeo& g, cudaStream_t s, u64* bbuf, const u64* aspec, u64 ninv,
                              const RootTables& tw, const ProdJob* jobs = nullptr, unsigned njobs = 1);
cudaError_t launch_r3_fwd(cudaStream_t s, const u32* limbs, u64 ndig, u64* out, int logm, const RootTables& tw,
                          const ProdJob* jobs = nullptr, unsigned njobs = 1, int operand = 0);
cudaError_t launch_r3_inv(cudaStream_t s, u64* buf, int logm, const RootTables& tw, const ProdJob* jobs = nullptr,
                          unsigned njobs = 1);
cudaError_t launch_mul_small(int logn, const PassGeo& g, cudaStream_t s, const u32* a, u64 na, const u32* b, u64 nb,
                             u32* out, u64 nout, unsigned long long* out_len, u64 ninv, const RootTables& tw,
                             const ProdJob* jobs = nullptr, unsigned njobs = 1);
// The coefficients in `coef` are the unscaled inverse transform of `points`
// points (N * c mod p); the carry scales them by points^-1 (points = 1: as
// they are).
cudaError_t launch_carry(unsigned nchunks, cudaStream_t s, const u64* coef, u32* out, u64 nout,
                         LookbackSlot* slots, u32* ticket, unsigned long long* out_len, u32* err,
                         const ProdJob* jobs = nullptr, unsigned njobs = 1, u64 points = 1);
cudaError_t configure_first();
cudaError_t configure_mid();
cudaError_t configure_inv();
cudaError_t configure_last();
cudaError_t configure_fused();
cudaError_t configure_small();

}  // namespace b2m
