// ntt_carry.cu -- the decoupled-lookback carry kernel and its launcher.
//
// Reference counterpart: carry_propagate (include/ntt.h:70-91), which runs
// sequentially on the host after a full device-to-host copy of N u64
// coefficients; here it runs on the device and writes u32 limbs directly.
#include <cuda_runtime.h>

#include "b2m_internal.h"
#include "carry.cuh"

namespace b2m {

// ---------------------------------------------------------------------------
// Carry: coefficients (natural order, N of them) -> nout u32 limbs.
// One CTA per 4096 coefficients, chunks claimed in launch order by ticket so
// that every chunk a CTA waits for belongs to a CTA that is already running
// and publishes its aggregate without waiting. Waits are bounded: after
// ~2^22 polls the kernel flags *err and carries on with a wrong carry (the
// host turns the flag into B2M_ERR_DEVICE_TIMEOUT).
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 ld_acquire(const u32* p) {
    u32 v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(u32* p, u32 v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr int LOOKBACK_SPIN_LIMIT = 1 << 22;

// SC: how the coefficients are scaled by N^-1 before the carry -- 0 not at all
// (the last inverse pass already did, through its scaled twiddle table),
// 1 by 2^nshift with nshift >= 160 (N a power of two), 2 by the multiply with
// ninv. A template parameter, so that the common unscaled kernel keeps all of
// its 32 registers (eight CTAs per SM) for the carry itself.
template <int SC>
__global__ void __launch_bounds__(CARRY_THREADS, 8) k_carry(const u64* __restrict__ coef, u32* __restrict__ out,
                                                         u64 nout, LookbackSlot* slots, u32* ticket,
                                                         unsigned long long* out_len, u32* err,
                                                         const ProdJob* __restrict__ jobs, u64 ninv, int nshift) {
    if (jobs) {
        const ProdJob& J = jobs[blockIdx.y];
        coef = J.bufB;
        out = J.out;
        nout = J.na + J.nb;
        slots = J.slots;
        ticket = J.ticket;
        out_len = J.out_len;
    }
    __shared__ u32 s_chunk;
    __shared__ u64 s_cin;
    __shared__ CState s_ws[CARRY_THREADS / 32 + 1];
    if (threadIdx.x == 0) s_chunk = atomicAdd(ticket, 1u);
    __syncthreads();
    const u32 chunk = s_chunk;

    u64 cf[CARRY_G];
    const u64 cbase = (u64)chunk * CARRY_CHUNK + (u64)threadIdx.x * CARRY_G;
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(coef + cbase);
#pragma unroll
    for (int i = 0; i < CARRY_G / 2; ++i) {
        ulonglong2 p = src[i];
        cf[2 * i] = p.x;
        cf[2 * i + 1] = p.y;
    }
    // The inverse transform leaves N * c (mod p); the scale by N^-1 is done
    // here rather than in the ALU-bound fused pass: for N = 2^k it is the
    // shift by 2^(192 - k) (2 has order 192), otherwise one multiply.
    if constexpr (SC == 1) {
#pragma unroll
        for (int i = 0; i < CARRY_G; ++i) cf[i] = gl_shl_160(cf[i], nshift - 160);
    } else if constexpr (SC == 2) {
#pragma unroll
        for (int i = 0; i < CARRY_G; ++i) cf[i] = gl_mul(cf[i], ninv);
    }
    u32 lm[CARRY_G / 2];
    const CState st = group_carry<CARRY_G>(cf, lm);
    bool has_ex;
    CState agg;
    const CState ex = block_scan_carry(st, &has_ex, &agg, s_ws);

    if (threadIdx.x == 0) {
        u64 cin = 0;
        if (chunk == 0) {
            slots[0].incl = cs_eval(agg, 0);
            __threadfence();
            st_release(&slots[0].flag, 2u);
        } else {
            slots[chunk].agg_h = agg.h;
            slots[chunk].agg_t = agg.t;
            __threadfence();
            st_release(&slots[chunk].flag, 1u);
            // Walk back, composing aggregates until an inclusive value or a
            // carry-independent (constant) composition is found.
            CState acc{0, CS_NEVER};
            bool acc_id = true;
            long p = (long)chunk - 1;
            while (true) {
                u32 f;
                int spins = 0;
                while ((f = ld_acquire(&slots[p].flag)) == 0u) {
                    if (++spins > LOOKBACK_SPIN_LIMIT) break;
                    __nanosleep(64);
                }
                if (f == 0u) {  // gave up: report, use 0 and finish cleanly
                    atomicOr(err, 1u);
                    cin = 0;
                    break;
                }
                if (f == 2u) {
                    const u64 val = *(volatile u64*)&slots[p].incl;
                    cin = acc_id ? val : cs_eval(acc, val);
                    break;
                }
                const CState a{*(volatile u64*)&slots[p].agg_h, *(volatile u64*)&slots[p].agg_t};
                acc = acc_id ? a : cs_then(a, acc);
                acc_id = false;
                if (acc.t == CS_NEVER) {  // constant: earlier chunks cannot matter
                    cin = acc.h;
                    break;
                }
                --p;  // p > 0 here: chunk 0 always publishes inclusive
            }
            slots[chunk].incl = cs_eval(agg, cin);
            __threadfence();
            st_release(&slots[chunk].flag, 2u);
        }
        s_cin = cin;
    }
    __syncthreads();
    const u64 cin_chunk = s_cin;
    const u64 cin = has_ex ? cs_eval(ex, cin_chunk) : cin_chunk;
    group_add_carry<CARRY_G / 2>(lm, cin);

    const u64 lbase = cbase / 2;
    unsigned long long top = 0;
#pragma unroll
    for (int i = 0; i < CARRY_G / 2; ++i)
        if (lm[i] && lbase + i < nout) top = lbase + i + 1;
    if (lbase + CARRY_G / 2 <= nout && ((reinterpret_cast<uintptr_t>(out + lbase) & 15) == 0)) {
        // whole group in range and 16-byte aligned: vector stores
        uint4* dst = reinterpret_cast<uint4*>(out + lbase);
#pragma unroll
        for (int i = 0; i < CARRY_G / 8; ++i) dst[i] = make_uint4(lm[4 * i], lm[4 * i + 1], lm[4 * i + 2], lm[4 * i + 3]);
    } else {
#pragma unroll
        for (int i = 0; i < CARRY_G / 2; ++i)
            if (lbase + i < nout) out[lbase + i] = lm[i];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, top, off);
        top = o > top ? o : top;
    }
    if ((threadIdx.x & 31) == 0 && top) atomicMax(out_len, top);
}


cudaError_t launch_carry(unsigned nchunks, cudaStream_t s, const u64* coef, u32* out, u64 nout,
                         LookbackSlot* slots, u32* ticket, unsigned long long* out_len, u32* err,
                         const ProdJob* jobs, unsigned njobs, u64 points) {
    // scale by points^-1: a shift when points is a power of two (2^(192 - k),
    // k <= 32, is a shift by 160 + (32 - k)), else one multiply
    const dim3 grid(nchunks, njobs);
    if (points <= 1) {
        k_carry<0><<<grid, CARRY_THREADS, 0, s>>>(coef, out, nout, slots, ticket, out_len, err, jobs, 1, 0);
    } else if ((points & (points - 1)) == 0 && points <= (1ull << 32)) {
        int k = 0;
        while ((1ull << k) < points) ++k;
        k_carry<1><<<grid, CARRY_THREADS, 0, s>>>(coef, out, nout, slots, ticket, out_len, err, jobs, 1, 192 - k);
    } else {
        k_carry<2><<<grid, CARRY_THREADS, 0, s>>>(coef, out, nout, slots, ticket, out_len, err, jobs, gl_inv(points),
                                                  -1);
    }
    return cudaGetLastError();
}

}  // namespace b2m
