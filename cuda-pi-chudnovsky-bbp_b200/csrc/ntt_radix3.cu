// ntt_radix3.cu -- transforms of N = 3M points (M = 2^k): one radix-3 step
// around three M-point transforms.
//
// Power-of-two lengths waste up to 2x on padding (1.44x on average for
// log-uniform product sizes); a 3 * 2^k length holds the product whenever
// 2(na + nb) <= 3 * 2^k < next power of two. Goldilocks has the roots for it:
// p - 1 = 2^32 * 3 * 5 * 17 * 257 * 65537, and the cube root of unity is
// w = 2^64 (2 has order 192), so the radix-3 butterflies are shifts. The
// primitive (3 * 2^32)-th root Omega is chosen with Omega^3 = RHO and
// Omega^(2^32) = 2^64, so the M-point sub-transforms use the RHO chain of the
// power-of-two path unchanged and W = Omega^(2^(32-k)) is a primitive N-th
// root with W^M = w:
//   Omega^x = RHO^(x * 3^-1 mod 2^32) * 2^(64 (x mod 3)).
//
// Forward (decimation in frequency): y_r[j] = W^(r j) (x_j + w^r x_{j+M} +
// w^(2r) x_{j+2M}), r = 0, 1, 2, and X[3m + r] = DFT_M(y_r)[m]. The pointwise
// product runs per sub-transform; the inverse sub-transforms give z_r and
//   x_{j+tM} = sum_r w^(-t r) W^(-j r) z_r[j]
// with the 1/3 folded into the pointwise N^-1. No reference counterpart: the
// reference's transforms are radix-2 only (src/ntt_cuda.cu:99-114).
#include <cuda_runtime.h>

#include "b2m_internal.h"
#include "ntt_kernels.cuh"

namespace b2m {

constexpr u32 INV3_MOD_2_32 = 0xAAAAAAABu;  // 3 * 0xAAAAAAAB == 1 (mod 2^32)

// Omega^x for x given as (x mod 2^32, x mod 3).
__device__ __forceinline__ u64 omega_pow(u32 xm, u32 x3, const RootTables& tw) {
    const u32 e = xm * INV3_MOD_2_32;
    const u64 r = e ? uroot(e, tw.u1, tw.u2) : 1ull;
    return x3 ? gl_shl(r, 64 * (int)x3) : r;
}

// The exponent of W^j = Omega^(j 2^(32-k)) as (mod 2^32, mod 3).
__device__ __forceinline__ void w_exp(u64 j, int logm, u32* xm, u32* x3) {
    *xm = (u32)(j << (32 - logm));                // j < 2^k: exact
    const u32 t = ((32 - logm) & 1) ? 2u : 1u;    // 2^(32-k) mod 3
    *x3 = (u32)((j % 3) * t % 3);
}

__global__ void __launch_bounds__(256) k_r3_fwd(const u32* __restrict__ limbs, u64 ndig, u64* __restrict__ out,
                                                int logm, RootTables tw, const ProdJob* __restrict__ jobs,
                                                int operand) {
    if (jobs) {
        const ProdJob& J = jobs[blockIdx.y];
        limbs = operand ? J.b : J.a;
        ndig = 2 * (operand ? J.nb : J.na);
        out = operand ? J.bufB : J.bufA;
    }
    const u64 m = 1ull << logm;
    if (2 * ndig <= 3 * m) {
        // The digits fill at most half of the 3m points (N >= 2(na + nb)
        // digits for every product), so x2 = x[j + 2m] is zero: three outputs
        // from x0 and x1 alone.
        for (u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (u64)gridDim.x * blockDim.x) {
            const u64 x0 = digit_of(limbs, ndig, j), x1 = digit_of(limbs, ndig, j + m);
            u32 xm, x3;
            w_exp(j, logm, &xm, &x3);
            const u64 w1 = omega_pow(xm, x3, tw);
            out[j] = gl_add(x0, x1);
            out[m + j] = gl_mul(gl_add(x0, gl_shl(x1, 64)), w1);                  // (x0 + w x1) W^j
            out[2 * m + j] = gl_mul(gl_add(x0, gl_shl(x1, 128)), gl_mul(w1, w1));  // (x0 + w^2 x1) W^2j
        }
        return;
    }
    for (u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (u64)gridDim.x * blockDim.x) {
        const u64 x0 = digit_of(limbs, ndig, j), x1 = digit_of(limbs, ndig, j + m),
                  x2 = digit_of(limbs, ndig, j + 2 * m);
        const u64 y0 = gl_add(x0, gl_add(x1, x2));
        const u64 a1 = gl_add(gl_add(x0, gl_shl(x1, 64)), gl_shl(x2, 128));  // x0 + w x1 + w^2 x2
        const u64 a2 = gl_add(gl_add(x0, gl_shl(x1, 128)), gl_shl(x2, 64));  // x0 + w^2 x1 + w x2
        u32 xm, x3;
        w_exp(j, logm, &xm, &x3);
        const u64 w1 = omega_pow(xm, x3, tw);
        out[j] = y0;
        out[m + j] = gl_mul(a1, w1);
        out[2 * m + j] = gl_mul(a2, gl_mul(w1, w1));
    }
}

__global__ void __launch_bounds__(256) k_r3_inv(u64* __restrict__ buf, int logm, RootTables tw,
                                                const ProdJob* __restrict__ jobs) {
    if (jobs) buf = jobs[blockIdx.y].bufB;
    const u64 m = 1ull << logm;
    for (u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (u64)gridDim.x * blockDim.x) {
        u32 xm, x3;
        w_exp(j, logm, &xm, &x3);
        const u64 v1 = omega_pow(0u - xm, (3u - x3) % 3u, tw);  // W^-j
        const u64 c1 = gl_mul(buf[m + j], v1);
        const u64 c2 = gl_mul(buf[2 * m + j], gl_mul(v1, v1));
        const u64 z0 = buf[j];
        buf[j] = gl_add(z0, gl_add(c1, c2));
        buf[m + j] = gl_add(gl_add(z0, gl_shl(c1, 128)), gl_shl(c2, 64));      // w^-1 = w^2
        buf[2 * m + j] = gl_add(gl_add(z0, gl_shl(c1, 64)), gl_shl(c2, 128));  // w^-2 = w
    }
}

static unsigned r3_grid(int logm) {
    const u64 blocks = ((1ull << logm) + 255) / 256;
    return (unsigned)(blocks < 4096 ? blocks : 4096);
}

cudaError_t launch_r3_fwd(cudaStream_t s, const u32* limbs, u64 ndig, u64* out, int logm, const RootTables& tw,
                          const ProdJob* jobs, unsigned njobs, int operand) {
    k_r3_fwd<<<dim3(r3_grid(logm), njobs), 256, 0, s>>>(limbs, ndig, out, logm, tw, jobs, operand);
    return cudaGetLastError();
}

cudaError_t launch_r3_inv(cudaStream_t s, u64* buf, int logm, const RootTables& tw, const ProdJob* jobs,
                          unsigned njobs) {
    k_r3_inv<<<dim3(r3_grid(logm), njobs), 256, 0, s>>>(buf, logm, tw, jobs);
    return cudaGetLastError();
}

}  // namespace b2m
