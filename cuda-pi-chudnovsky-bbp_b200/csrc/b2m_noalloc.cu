// b2m_noalloc.cu -- the product entry point that allocates no device memory.
//
// Some callers cannot allocate device memory when they multiply: their device
// memory is already owned by another allocator (a framework's caching pool or
// an embedder that reserves all HBM up front), or their loop cannot afford the
// device-wide synchronisation and latency that cudaMalloc brings. For them the
// product's scratch (the two transform buffers and the carry lookback slots)
// lives in one file-scope device array of fixed size instead of the
// stream-ordered pool that b2m_mul_device draws from.
//
// Limits and sharing:
//  * transform length at most 2^NOALLOC_MAX_LOGN = 2^20, i.e. na + nb <= 2^19
//    limbs; larger products are rejected with B2M_ERR_TOO_LARGE;
//  * the array (about 16 MiB) exists on every GPU that loads this library and
//    stays allocated until the process exits;
//  * every call uses the same array, so calls whose device work overlaps (on
//    different streams, or from different host threads) race; callers
//    serialise them. The carry scratch that must start at zero is cleared on
//    the stream by each call before use; the transform buffers are fully
//    overwritten by each call and keep the last call's contents afterwards.
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (host code cannot use the array's name as a device
//    address); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "b2m.h"
#include "b2m_context.h"
#include "b2m_internal.h"

namespace b2m {

constexpr int NOALLOC_MAX_LOGN = 20;
constexpr uint64_t NOALLOC_SCRATCH_BYTES =
    2ull * (8ull << NOALLOC_MAX_LOGN) + ((1ull << NOALLOC_MAX_LOGN) / CARRY_CHUNK) * sizeof(LookbackSlot) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on `device` (which is current).
static b2m_status noalloc_scratch(int device, void** out) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) {
        set_error("device index beyond the no-allocation table");
        return B2M_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_noalloc_ptr[device] = p;
    }
    *out = g_noalloc_ptr[device];
    return B2M_OK;
}

}  // namespace b2m

using namespace b2m;

extern "C" b2m_status b2m_mul_device_noalloc(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                                             uint32_t* d_out, uint64_t out_cap, uint64_t* d_out_len,
                                             b2m_stream stream) {
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
    if (logn > NOALLOC_MAX_LOGN) {
        set_error("b2m_mul_device_noalloc handles transform lengths up to 2^20 (na + nb <= 2^19 limbs)");
        return B2M_ERR_TOO_LARGE;
    }
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    void* ws = nullptr;
    if ((st = noalloc_scratch(c->device, &ws)) != B2M_OK) return st;
    const Plan p = product_plan(c, na, nb);  // at most 2^20 points: within the static scratch
    e = launch_product(d_a, na, d_b, nb, d_out, d_out_len, ws, p, c->tw, c->d_err, s);
    return cuda_status(e, "kernel launch");
}
