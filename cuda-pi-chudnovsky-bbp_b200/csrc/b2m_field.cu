// b2m_field.cu -- element-wise evaluation of the device field arithmetic.
//
// The transforms' butterflies, twiddles and pointwise product are built from
// the device functions of gl.cuh (32-bit-word borrow chains and folds). This
// entry point runs exactly those device functions over arrays so that they
// can be checked one by one against the reference's field
// (include/goldilocks.h:90-189; its own self-test checks it in
// tests/self_test.cu:46-62), on edge values and on random operands, instead
// of only through whole products.
#include <cuda_runtime.h>

#include "b2m.h"
#include "b2m_context.h"
#include "b2m_internal.h"
#include "ntt_engine.cuh"

namespace b2m {

// 8-point transforms of consecutive groups of 8 (n a multiple of 8).
template <bool INV>
__global__ void k_field_dft8(const u64* __restrict__ a, u64* __restrict__ out, u64 groups) {
    for (u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += (u64)gridDim.x * blockDim.x) {
        u64 x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = a[8 * g + i];
        if (INV) dft_inv<8>(x);
        else dft_fwd<8>(x);
#pragma unroll
        for (int i = 0; i < 8; ++i) out[8 * g + i] = x[i];
    }
}

__global__ void k_field_eval(int op, const u64* __restrict__ a, const u64* __restrict__ b, u64* __restrict__ out,
                             u64 n) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 x = a[i], y = b[i];
        u64 r = 0;
        switch (op) {
            case B2M_FIELD_ADD: r = gl_add(x, y); break;
            case B2M_FIELD_SUB: r = gl_sub(x, y); break;
            case B2M_FIELD_MUL: r = gl_mul(x, y); break;
            case B2M_FIELD_SHL: r = gl_shl(x, (int)(y % 192)); break;
            case B2M_FIELD_POW: r = gl_pow(x, y); break;
            case B2M_FIELD_INV: r = gl_inv(x); break;
            case B2M_FIELD_SHL_RT: r = gl_shl_rt(x, (u32)(y % 192)); break;
            case B2M_FIELD_SHL_160: r = gl_shl_160(x, (int)(y % 32)); break;
            case B2M_FIELD_SHL_RT2: {
                // elements 2k and 2k+1 shifted together by b[2k]
                const u64 k0 = i & ~1ull;
                const ulonglong2 q = gl_shl_rt2(a[k0], k0 + 1 < n ? a[k0 + 1] : 0, (u32)(b[k0] % 192));
                r = (i & 1) ? q.y : q.x;
                break;
            }
            default: r = 0; break;
        }
        out[i] = r;
    }
}

}  // namespace b2m

using namespace b2m;

extern "C" b2m_status b2m_field_eval_host(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, uint64_t n) {
    if (n == 0) return B2M_OK;
    const bool dft = op == B2M_FIELD_DFT8 || op == B2M_FIELD_IDFT8;
    if (!a || !out || (!dft && !b) || op < 0 || op > B2M_FIELD_SHL_RT2 || (dft && (n % 8) != 0)) {
        set_error("b2m_field_eval_host: bad op, pointer or length");
        return B2M_ERR_INVALID_ARGUMENT;
    }
    Context* c = ctx();
    if (!c) {
        set_error("b2m_init was not called");
        return B2M_ERR_NOT_INITIALIZED;
    }
    u64* d = nullptr;
    cudaError_t e = cudaMalloc(&d, 3 * n * sizeof(u64));
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(field eval)");
    u64 *da = d, *db = d + n, *dout = d + 2 * n;
    e = cudaMemcpy(da, a, n * sizeof(u64), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !dft) e = cudaMemcpy(db, b, n * sizeof(u64), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const u64 work = dft ? n / 8 : n;
        const unsigned blocks = (unsigned)(work / 256 + 1 < 4096 ? work / 256 + 1 : 4096);
        if (op == B2M_FIELD_DFT8) k_field_dft8<false><<<blocks, 256>>>(da, dout, n / 8);
        else if (op == B2M_FIELD_IDFT8) k_field_dft8<true><<<blocks, 256>>>(da, dout, n / 8);
        else k_field_eval<<<blocks, 256>>>(op, da, db, dout, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, n * sizeof(u64), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return cuda_status(e, "b2m_field_eval_host");
}
