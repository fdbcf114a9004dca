/*
 * b2m.h -- C ABI of the B200 Goldilocks-NTT big-integer multiply backend.
 *
 * Numbers are little-endian arrays of 32-bit limbs (value = sum limb[i] *
 * 2^(32 i)), exactly the magnitude layout of the reference's BigInt::mag
 * (include/bignum.h:21-44, 106-109). Products are bit-exact: the same integer
 * the reference's mul_ntt_cpu / mul_schoolbook return, trimmed of leading
 * zero limbs. No entry point ever falls back to a CPU multiply; failures are
 * reported as status codes.
 *
 * The reference exposes this path as C++ functions
 *   std::vector<uint32_t> pidigits::mul_ntt_cuda(const std::vector<uint32_t>&,
 *                                                const std::vector<uint32_t>&)
 *   bool pidigits::cuda_available()
 * (include/bignum.h:200-205, src/ntt_cuda.cu:165-243). The C++ shim
 * ntt_cuda_b200.cpp maps those two signatures onto b2m_mul_host and
 * b2m_cuda_available below, so the reference's own callers (mul_dispatch in
 * src/bignum.cpp:204-232, chudnovsky_bs in src/chudnovsky.cpp:64-102) run on
 * this backend unchanged.
 *
 * Threading: every entry point may be called from any host thread; library
 * state is guarded internally. Device work of the *_device / batch calls is
 * ordered on the caller's stream.
 */
#ifndef B2M_H
#define B2M_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2M_API_VERSION 1

/* A CUDA stream (cudaStream_t / CUstream); NULL is the legacy default stream. */
typedef struct CUstream_st* b2m_stream;

typedef enum b2m_status {
    B2M_OK = 0,
    B2M_ERR_INVALID_ARGUMENT = 1,  /* null pointer with a non-zero size, bad flag, ... */
    B2M_ERR_NO_DEVICE = 2,         /* no CUDA device, or not an sm_100 device */
    B2M_ERR_NOT_INITIALIZED = 3,   /* b2m_init was not called (or failed) */
    B2M_ERR_CUDA = 4,              /* a CUDA runtime call failed (detail: b2m_last_error) */
    B2M_ERR_OUT_OF_MEMORY = 5,     /* device allocation failed or the HBM budget is exhausted */
    B2M_ERR_TOO_LARGE = 6,         /* transform length above 2^30 (na + nb > 2^28 limbs) */
    B2M_ERR_OUTPUT_TOO_SMALL = 7,  /* out_cap < na + nb */
    B2M_ERR_DEVICE_TIMEOUT = 8,    /* a bounded device-side wait gave up (carry lookback) */
    B2M_ERR_QUEUE_FULL = 9,        /* serving: request table full */
    B2M_ERR_NOT_FOUND = 10,        /* serving: unknown ticket */
    B2M_ERR_SHUTDOWN = 11,         /* serving: the server is stopping */
    B2M_ERR_INTERNAL = 12          /* an exact-arithmetic check failed (a library bug; detail: b2m_last_error) */
} b2m_status;

/* ---- lifetime ------------------------------------------------------------ */

/* Replaces the implicit per-call setup of src/ntt_cuda.cu:179-214 (device
 * probe, cudaMalloc, twiddle build). Selects `device`, uploads the resident
 * root tables once and sets the HBM budget the library may allocate
 * (0 = 90% of the device's free memory at init). Idempotent for the same
 * device; a second call with another device re-initialises. */
b2m_status b2m_init(int device, uint64_t hbm_budget_bytes);

/* Frees every device resource the library holds. */
b2m_status b2m_shutdown(void);

/* Replaces pidigits::cuda_available() (src/ntt_cuda.cu:165-173): 1 when
 * b2m_init(0, 0) succeeds (or an earlier init succeeded), else 0. Cached. */
int b2m_cuda_available(void);

/* Human-readable name of a status; never NULL. */
const char* b2m_strerror(b2m_status status);

/* Detail of the last failure on the calling thread ("" if none). */
const char* b2m_last_error(void);

/* Replaces ntt_length (include/ntt.h:47-50): next power of two >= 2na + 2nb.
 * (The products may run on 3 * 2^k points instead; b2m_plan_describe tells.) */
uint64_t b2m_ntt_length(uint64_t na, uint64_t nb);

/* Device workspace in bytes that one product of na x nb limbs needs. */
uint64_t b2m_workspace_bytes(uint64_t na, uint64_t nb);

/* ---- single products ------------------------------------------------------- */

/* Replaces pidigits::mul_ntt_cuda (src/ntt_cuda.cu:179-243): host buffers in,
 * host buffer out, synchronous. a/b may carry leading zero limbs (their sizes
 * are taken as given, like the reference's .size()). out must hold
 * out_cap >= na + nb limbs; *out_len receives the trimmed length (0 for a
 * zero product or an empty input). Only out[0, *out_len) is defined. */
b2m_status b2m_mul_host(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb,
                        uint32_t* out, uint64_t out_cap, uint64_t* out_len);

/* The same product with operands already resident in device memory, ordered
 * on `stream` and asynchronous: d_out receives na + nb limbs (the limbs past
 * the trimmed length are zero) and *d_out_len (a device pointer, may be NULL)
 * the trimmed length. The workspace is taken from a stream-ordered pool.
 * Device-side failures surface through b2m_stream_check. */
b2m_status b2m_mul_device(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                          uint32_t* d_out, uint64_t out_cap, uint64_t* d_out_len,
                          b2m_stream stream);

/* No counterpart in the reference. The same product as b2m_mul_device, for
 * callers that cannot allocate device memory when they multiply (their HBM is
 * owned by another allocator, or a cudaMalloc's device-wide synchronisation
 * and latency are not acceptable in their loop): it allocates nothing. Its
 * scratch is one fixed static device array of about 16 MiB, present on every
 * GPU that loads the library until the process exits, so it accepts
 * transform lengths up to 2^20 only (na + nb <= 2^19 limbs) and returns
 * B2M_ERR_TOO_LARGE beyond that. Every call shares that array: calls whose
 * device work overlaps (other streams, other host threads) race, and the
 * caller must serialise them. The first call on a device looks up the
 * array's device address; make that first call before any stream capture.
 * Inputs, output and *d_out_len are the caller's device buffers, as for
 * b2m_mul_device. */
b2m_status b2m_mul_device_noalloc(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                                  uint32_t* d_out, uint64_t out_cap, uint64_t* d_out_len,
                                  b2m_stream stream);

/* Synchronises `stream` and reports (and clears) any device-side failure
 * raised by this library's kernels since the last check. */
b2m_status b2m_stream_check(b2m_stream stream);

/* No reference counterpart. Self-check of the device-side failure detection:
 * runs the carry kernel on a crafted job whose only block waits on a
 * predecessor that never publishes. The wait is bounded (a fixed number of
 * polls, about half a second), so the kernel flags the error word and
 * returns; the call reports B2M_ERR_DEVICE_TIMEOUT when that works as
 * designed (B2M_OK would mean the bound did not fire) and leaves the context
 * usable. Nothing faults, traps or hangs. */
b2m_status b2m_selftest_wait_timeout(b2m_stream stream);

/* Element-wise evaluation of the device field arithmetic that the transforms
 * are built from (the Goldilocks field of include/goldilocks.h:90-189, which
 * the reference's self-test checks in tests/self_test.cu:46-62): out[i] =
 * op(a[i], b[i]) computed on the device by exactly the device functions the
 * kernels inline. Host buffers of n elements, synchronous. Operands are field
 * elements in [0, p) (SHL: b[i] is the shift amount, taken mod 192; POW: b[i]
 * is the exponent; INV ignores b). DFT8 / IDFT8 transform each group of 8
 * consecutive elements of a (n a multiple of 8; b unused): the forward
 * 8-point DFT with root 2^24, natural order in, bit-reversed order out, and
 * its unscaled inverse (bit-reversed in, natural out, root 2^-24).
 * Results are canonical, in [0, p). */
typedef enum b2m_field_op {
    B2M_FIELD_ADD = 0,
    B2M_FIELD_SUB = 1,
    B2M_FIELD_MUL = 2,
    B2M_FIELD_SHL = 3,   /* a * 2^(b mod 192) */
    B2M_FIELD_POW = 4,
    B2M_FIELD_INV = 5,
    B2M_FIELD_DFT8 = 6,
    B2M_FIELD_IDFT8 = 7,
    B2M_FIELD_SHL_RT = 8,  /* a * 2^(b mod 192) by the run-time shift of the level-1 twiddles */
    B2M_FIELD_SHL_160 = 9, /* a * 2^(160 + (b mod 32)): the carry's scale by N^-1 = 2^(192 - log2 N) */
    B2M_FIELD_SHL_RT2 = 10 /* a[2k], a[2k+1] * 2^(b[2k] mod 192) by the paired run-time shift */
} b2m_field_op;
b2m_status b2m_field_eval_host(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, uint64_t n);

/* ---- batched products ---------------------------------------------------------
 * No counterpart in the reference, whose tree (src/chudnovsky.cpp:64-102)
 * multiplies one pair at a time, each call paying its own allocation, copies
 * and radix-2 launches. A batch runs many independent products of mixed sizes
 * together: jobs are bucketed by transform length, every bucket runs as one
 * set of launches covering all of its products (grid dimension over the
 * jobs), buckets run concurrently on forked streams, and the whole sequence
 * can be captured once into a CUDA graph and replayed. */

typedef struct b2m_job {
    const uint32_t* a;     /* device limbs */
    uint64_t na;
    const uint32_t* b;
    uint64_t nb;
    uint32_t* out;         /* device, out_cap >= na + nb limbs */
    uint64_t out_cap;
    uint64_t* out_len;     /* device pointer or NULL: trimmed product length */
} b2m_job;

typedef struct b2m_batch b2m_batch;

#define B2M_BATCH_GRAPH 1u     /* capture the launch sequence into a CUDA graph */
#define B2M_BATCH_AUTOTUNE 2u  /* time candidate pass splits and tile sizes per size
                                  bucket at creation and keep the fastest */

/* Plans a batch over `jobs` (copied; the device buffers they point to must
 * stay valid while the batch exists). Allocates the batch's workspace from
 * the HBM budget. The batch can be launched any number of times; each launch
 * recomputes every product from the current contents of the inputs. */
b2m_status b2m_batch_create(const b2m_job* jobs, uint64_t njobs, uint32_t flags, b2m_batch** batch);

/* Enqueues every product of the batch on `stream` (one graph launch when
 * created with B2M_BATCH_GRAPH). Launches of one batch must not overlap. */
b2m_status b2m_batch_launch(b2m_batch* batch, b2m_stream stream);

/* Releases the batch (after synchronising its last launch). */
b2m_status b2m_batch_destroy(b2m_batch* batch);

/* create + launch + destroy without a graph: for one-shot batches. */
b2m_status b2m_mul_batch(const b2m_job* jobs, uint64_t njobs, b2m_stream stream);

/* ---- Chudnovsky binary splitting ------------------------------------------------
 * Replaces chudnovsky_bs (src/chudnovsky.cpp:64-102) for the caller's
 * product tree: (P, Q, T) of the term range [a, b), built level by level on
 * the device with every value resident in HBM and every level's products
 * batched (see b2m_chudnovsky.cu). The root equals the reference's
 * (P and Q are products, T/Q the exact partial sum, so the tree shape does not
 * matter). Term indices must stay below 2,000,000 (about 28 million digits). */

typedef struct b2m_pqt b2m_pqt;  /* device-resident (P, Q, T) */

b2m_status b2m_chudnovsky_bs(uint64_t a, uint64_t b, b2m_stream stream, b2m_pqt** result);

/* Lengths (limbs) of P, Q, T, the sign of T (P, Q > 0), the number of tree
 * levels and of products computed. Any pointer may be NULL. */
b2m_status b2m_pqt_info(const b2m_pqt* r, uint64_t len[3], int32_t* t_sign, uint32_t* levels,
                        uint64_t* products);

/* Device pointer of P (which = 0), Q (1) or T's magnitude (2). */
const uint32_t* b2m_pqt_device(const b2m_pqt* r, int which);

/* Copies P, Q or |T| to host memory (cap limbs available). */
b2m_status b2m_pqt_copy(const b2m_pqt* r, int which, uint32_t* host, uint64_t cap);

b2m_status b2m_pqt_free(b2m_pqt* r);

/* (P, Q, T) of [a, c) from those of the adjacent ranges [a, b) (left) and
 * [b, c) (right): P = Pl*Pr, Q = Ql*Qr, T = Tl*Qr + Pl*Tr -- the merge step of
 * chudnovsky_bs (src/chudnovsky.cpp:96-100), one tree level of two nodes on
 * the device. Inputs are unchanged. Lets a tree be split into subtrees (on
 * several GPUs) and merged at the top. */
b2m_status b2m_pqt_merge(const b2m_pqt* left, const b2m_pqt* right, b2m_stream stream, b2m_pqt** result);

/* A node made from device limbs, copied (the caller keeps its buffers):
 * P, Q and |T| of len[0..2] trimmed limbs at d_limbs[0..2] (on this device),
 * and the sign of T (-1, 0, 1) -- e.g. a subtree root received from another
 * GPU. No reference counterpart (the reference has one process, one GPU). */
b2m_status b2m_pqt_import(const uint32_t* const d_limbs[3], const uint64_t len[3], int32_t t_sign,
                          b2m_stream stream, b2m_pqt** result);

/* ---- division, square root, decimal -------------------------------------------------
 * The big-integer steps after the tree in compute_pi_chudnovsky
 * (src/chudnovsky.cpp:107-164), on the device and sub-quadratic: the
 * reference's are schoolbook (div_fast forwards to divmod_knuth,
 * src/bignum_div.cpp:162-178; isqrt is Newton with a Knuth division per step,
 * :189-204; to_decimal divides by 10^9 repeatedly, :239-267). Results are the
 * same integers: Newton reciprocals and roots only seed estimates that an
 * exact correction against the remainder finishes. Operands are device
 * magnitudes (leading zero limbs allowed); calls are synchronous on `stream`
 * and write the trimmed lengths to host memory. */

/* q = floor(a / b), r = a mod b (b != 0). d_q / d_r may be NULL when not
 * wanted; q needs q_cap >= na - nb + 1 limbs, r needs r_cap >= nb. */
b2m_status b2m_divmod_device(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                             uint32_t* d_q, uint64_t q_cap, uint64_t* q_len,
                             uint32_t* d_r, uint64_t r_cap, uint64_t* r_len, b2m_stream stream);

/* floor(sqrt(a)); out needs cap >= (na + 1) / 2 limbs. */
b2m_status b2m_isqrt_device(const uint32_t* d_a, uint64_t na, uint32_t* d_out, uint64_t cap, uint64_t* out_len,
                            b2m_stream stream);

/* Decimal digits of a, no leading zeros ("0" for zero), NUL-terminated into
 * the host buffer out (cap >= digits + 1); *len = digits. Divide and conquer
 * by 10^(9 2^j), each level's divisions batched. */
b2m_status b2m_to_decimal_device(const uint32_t* d_a, uint64_t na, char* out, uint64_t cap, uint64_t* len,
                                 b2m_stream stream);

/* The same three with host buffers, synchronous on the legacy default
 * stream: the shapes the reference's BigInt functions need (a, b, q, r and
 * out are host limb arrays; out of b2m_to_decimal_host is a host char
 * buffer). */
b2m_status b2m_divmod_host(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb, uint32_t* q,
                           uint64_t q_cap, uint64_t* q_len, uint32_t* r, uint64_t r_cap, uint64_t* r_len);
b2m_status b2m_isqrt_host(const uint32_t* a, uint64_t na, uint32_t* out, uint64_t cap, uint64_t* out_len);
b2m_status b2m_to_decimal_host(const uint32_t* a, uint64_t na, char* out, uint64_t cap, uint64_t* len);

/* Wall-clock split of b2m_compute_pi (milliseconds). */
typedef struct b2m_pi_timings {
    double tree_ms;      /* binary splitting to (P, Q, T) */
    double sqrt_ms;      /* 10^prec and floor(sqrt(10005 * 10^(2 prec))) */
    double div_ms;       /* numerator and the floor division by T */
    double decimal_ms;   /* decimal conversion */
    double total_ms;
    uint64_t terms;
} b2m_pi_timings;

/* Replaces compute_pi_chudnovsky (src/chudnovsky.cpp:107-164) with every
 * step on this GPU: "3." followed by `digits` digits of pi, NUL-terminated,
 * into out (cap >= digits + 3); *len = string length. Same guard digits,
 * term count and integer steps as the reference, so the same string.
 * Term indices stay below 2,000,000 (about 28 million digits). times may
 * be NULL. Uses the legacy default stream. */
b2m_status b2m_compute_pi(uint64_t digits, char* out, uint64_t cap, uint64_t* len, b2m_pi_timings* times);

/* ---- serving ---------------------------------------------------------------------
 * No counterpart in the reference. A continuous-batching multiply server:
 * requests of mixed sizes are submitted at any time, admitted in arrival
 * order while the server's HBM budget allows (generated operands, owned
 * outputs and each product's transform workspace count against it), grouped
 * into a dispatch whenever one of the server's stream slots is free, and run
 * as size buckets on that slot's stream, so dispatches overlap on the device.
 * Every product is checked on the device modulo 2^32 - 1 and 2^32 + 1 before
 * it is reported done. */

typedef struct b2m_server b2m_server;

typedef struct b2m_server_config {
    uint64_t hbm_budget_bytes;  /* device memory the server may hold (0 = half the library budget) */
    uint32_t streams;           /* concurrent dispatches (0 = 4) */
    uint32_t max_batch;         /* requests per dispatch (0 = 256) */
    uint32_t max_pending;       /* queued requests before B2M_ERR_QUEUE_FULL (0 = 2^20) */
    uint32_t reserved;
} b2m_server_config;

typedef struct b2m_request {
    const uint32_t* a;          /* device operand, or NULL: generated from seed_a */
    uint64_t na;
    const uint32_t* b;          /* device operand, or NULL: generated from seed_b */
    uint64_t nb;
    uint64_t seed_a, seed_b;    /* generator of b2m_gen_operand */
    uint32_t kind;              /* generated operands: 0 random limbs, 1 all 0xFFFFFFFF */
    uint32_t reserved;
    uint32_t* out;              /* device output (out_cap >= na + nb), or NULL: the server allocates it */
    uint64_t out_cap;
} b2m_request;

typedef struct b2m_result {
    int32_t state;              /* 0 queued, 1 on the GPU, 2 done, 3 failed */
    b2m_status status;
    uint32_t* out;              /* device pointer of the product (valid until b2m_server_release) */
    uint64_t out_len;           /* trimmed length */
    uint64_t t_submit_ns, t_admit_ns, t_done_ns;  /* steady-clock nanoseconds */
    int32_t residues_ok;        /* product matched mod 2^32 - 1 and 2^32 + 1 */
    int32_t reserved;
} b2m_result;

typedef struct b2m_server_stats {
    uint64_t submitted, completed, failed, dispatches;
    uint64_t inflight_dispatches, queued, max_queue;
    uint64_t bytes_in_use, peak_bytes;
    uint64_t max_inflight_dispatches;  /* most dispatches on the GPU at one time */
    uint64_t host_dispatch_ns;         /* scheduler time spent enqueueing dispatches */
    uint64_t slot_busy_ns;             /* summed over slots: enqueue to observed completion */
} b2m_server_stats;

b2m_status b2m_server_start(const b2m_server_config* cfg, b2m_server** server);
b2m_status b2m_server_submit(b2m_server* server, const b2m_request* req, uint64_t* ticket);
b2m_status b2m_server_poll(b2m_server* server, uint64_t ticket, b2m_result* result);
/* Blocks until the request is done or failed, or the timeout passes
 * (B2M_ERR_DEVICE_TIMEOUT, result still filled). */
b2m_status b2m_server_wait(b2m_server* server, uint64_t ticket, double timeout_s, b2m_result* result);
/* Forgets a finished request and frees the buffers the server owned for it. */
b2m_status b2m_server_release(b2m_server* server, uint64_t ticket);
b2m_status b2m_server_get_stats(b2m_server* server, b2m_server_stats* stats);
/* Completes every queued and running request, then stops the scheduler. */
b2m_status b2m_server_stop(b2m_server* server);

/* Seeded operand on the device: limb i = high 32 bits of splitmix64's output
 * function at seed + (i + 1) * 0x9E3779B97F4A7C15, top limb forced non-zero
 * (kind 0), or all 0xFFFFFFFF limbs (kind 1). No reference counterpart. */
b2m_status b2m_gen_operand(uint64_t seed, uint64_t n, uint32_t kind, uint32_t* d_out, b2m_stream stream);

/* ---- plan inspection and tracing -------------------------------------------- */

/* Kernel kinds of a product's launch sequence. */
enum {
    B2M_K_FWD_FIRST = 1,   /* first forward pass: u32 limbs -> 16-bit digits -> pass 1 */
    B2M_K_FWD_MID = 2,     /* a middle forward pass */
    B2M_K_FWD_LAST = 3,    /* operand A's last forward pass */
    B2M_K_FUSED_LAST = 4,  /* operand B's last forward pass + pointwise + first inverse pass */
    B2M_K_INV_MID = 5,     /* an inverse pass (pass 1 yields the coefficients) */
    B2M_K_CARRY = 6,       /* decoupled-lookback carry into u32 limbs */
    B2M_K_SMALL = 7,       /* whole product in one CTA (transform length <= 2^13) */
    B2M_K_R3_FWD = 8,      /* radix-3 step of a 3 * 2^k-point transform (digits in) */
    B2M_K_R3_INV = 9       /* inverse radix-3 step (coefficients out, natural order) */
};

typedef struct b2m_plan_desc {
    uint32_t ntt_log2;      /* log2 of the transform length */
    uint32_t npass;         /* 0 = single-CTA product, else 2 or 3 passes */
    uint32_t logr[3];       /* radix exponent of each pass */
    uint32_t logc[3];       /* columns per CTA (log2) of each pass */
    uint32_t launches;      /* kernels launched per product */
    uint32_t three;         /* 1: 3 * 2^ntt_log2 points (a radix-3 step around three
                               2^ntt_log2-point transforms with this pass plan) */
} b2m_plan_desc;

/* Describes the transform plan the library uses for an na x nb product (no
 * reference counterpart: the reference always runs radix-2 stages of
 * next_pow2(2na + 2nb) points; this library uses 3 * 2^k points instead when
 * that is fewer and k >= 14). */
b2m_status b2m_plan_describe(uint64_t na, uint64_t nb, b2m_plan_desc* desc);

/* One timed candidate of b2m_autotune. */
typedef struct b2m_tune_entry {
    b2m_plan_desc plan;
    float ms;               /* median device time of one product with that plan */
    uint32_t chosen;        /* 1 for the plan that was kept */
} b2m_tune_entry;

/* No reference counterpart. Times every candidate transform plan (pass
 * splits and tile sizes) for an na x nb product on `stream`, with seeded
 * operands in a temporary allocation, and keeps the fastest: every later
 * product of the same transform length (single, batched, tree, division,
 * serving) uses it. Synchronous. Up to cap timings go to out (may be NULL
 * with cap 0), *n receives how many were written. */
b2m_status b2m_autotune(uint64_t na, uint64_t nb, b2m_stream stream, b2m_tune_entry* out, uint32_t cap,
                        uint32_t* n);

/* Fixes the plan of one transform length (desc->ntt_log2) to desc, which
 * must be one of the candidates b2m_autotune times (its out entries are
 * valid input). For reproducible timings and for testing every plan. */
b2m_status b2m_set_plan(const b2m_plan_desc* desc);

typedef struct b2m_kernel_time {
    uint32_t kind;          /* B2M_K_* */
    uint32_t logr;          /* pass radix exponent (0 for carry) */
    float ms;               /* device time of that launch, CUDA events on the stream */
} b2m_kernel_time;

/* b2m_mul_device with a CUDA event recorded around every kernel launch on
 * `stream`; synchronises and returns the per-launch device times in launch
 * order (at most cap entries, *n receives the count). For tracing and the
 * benchmark's roofline figures; the product is identical to b2m_mul_device. */
b2m_status b2m_mul_device_traced(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                                 uint32_t* d_out, uint64_t out_cap, uint64_t* d_out_len,
                                 b2m_stream stream, b2m_kernel_time* times, uint32_t cap, uint32_t* n);

#ifdef __cplusplus
}
#endif

#endif /* B2M_H */
