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
// One CTA per chunk of 4096 coefficients, chunks claimed in launch order by
// ticket so that every chunk a CTA waits for belongs to a CTA that is already
// running and publishes its aggregate without waiting. Warp 0 resolves the
// chunk's carry-in, 32 predecessors per round trip. Waits are bounded:
// after ~2^22 polls the kernel flags *err and carries on with a wrong carry
// (the host turns the flag into B2M_ERR_DEVICE_TIMEOUT).
//
// Each thread normalises 16 contiguous coefficients, but the chunk is read
// coalesced (lane l of a warp reads pair i*32 + l of the warp's 512
// coefficients) and handed to its owner through shared memory: a thread's
// own 128 contiguous bytes read directly would touch 32 cache lines per warp
// load instruction, eight times the L1 wavefronts of the coalesced read.
// ---------------------------------------------------------------------------
__device__ __forceinline__ u64 ld_acquire(const u64* p) {
    u64 v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
// Release store: the thread's earlier writes (the slot's threshold) are
// visible to any thread that reads this word with ld_acquire.
__device__ __forceinline__ void st_release(u64* p, u64 v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

constexpr int LOOKBACK_SPIN_LIMIT = 1 << 22;
constexpr int CARRY_WARP_PAIRS = 32 * CARRY_G / 2;  // coefficient pairs per warp
constexpr int CARRY_MIN_CTAS = CARRY_G >= 16 ? 6 : 8;  // CTAs per SM the staging area allows

// The warp's 32 * CARRY_G coefficients from HBM into cf[] of their owner
// lane (lane l owns coefficients CARRY_G*l .. CARRY_G*l + CARRY_G - 1 of the
// warp's slice). Pair q of the slice belongs to lane o = q / PPL as its pair
// j = q % PPL (PPL = CARRY_G / 2 pairs per lane) and sits in slot
// o*PPL + (j ^ ((o / (8/PPL)) % PPL)) of the warp's staging area: both the
// coalesced stores and the owners' reads touch eight distinct 16-byte bank
// groups per quarter warp.
__device__ __forceinline__ void load_chunk(const u64* __restrict__ coef, u64 wbase, ulonglong2* stage, u64* cf) {
    constexpr int PPL = CARRY_G / 2, OPR = 8 / PPL;  // pairs per lane, owners per 128-byte row
    static_assert(PPL == 4 || PPL == 8, "staging layout for 8 or 16 coefficients per thread");
    const int lane = threadIdx.x & 31;
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(coef + wbase);
    ulonglong2 v[PPL];
#pragma unroll
    for (int i = 0; i < PPL; ++i) v[i] = src[i * 32 + lane];
#pragma unroll
    for (int i = 0; i < PPL; ++i) {
        const int o = i * (32 / PPL) + lane / PPL, j = lane % PPL;  // owner and pair of q = 32i + lane
        stage[o * PPL + (j ^ ((o / OPR) % PPL))] = v[i];
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < PPL; ++j) {
        const ulonglong2 p = stage[lane * PPL + (j ^ ((lane / OPR) % PPL))];
        cf[2 * j] = p.x;
        cf[2 * j + 1] = p.y;
    }
}

constexpr u64 SLOT_CONST = 1, SLOT_INCL = 2, SLOT_AGG = 3;

__device__ __forceinline__ CState cs_shfl(CState f, int src) {
    return {__shfl_sync(0xFFFFFFFFu, f.h, src), __shfl_sync(0xFFFFFFFFu, f.t, src)};
}

// Warp 0 (all lanes): publish chunk `chunk`'s aggregate, then resolve its
// carry-in. Each round reads the slots of the 32 nearest unresolved
// predecessors at once (lane i: chunk base - i); the nearest slot holding a
// constant aggregate or an inclusive value ends the walk, the aggregates in
// front of it are composed onto it. A round with 32 thresholded aggregates
// composes them all and moves 32 chunks further back. Returns the carry-in
// on every lane; the inclusive value is published by the caller.
__device__ __forceinline__ u64 warp_lookback(LookbackSlot* slots, u32 chunk, CState agg, u32* err) {
    const int lane = threadIdx.x & 31;
    if (chunk == 0) {
        if (lane == 0) st_release(&slots[0].word, (cs_eval(agg, 0) << 2) | SLOT_INCL);
        return 0;
    }
    if (lane == 0) {
        if (agg.t != CS_NEVER) slots[chunk].agg_t = agg.t;
        st_release(&slots[chunk].word, (agg.h << 2) | (agg.t == CS_NEVER ? SLOT_CONST : SLOT_AGG));
    }
    CState acc{0, CS_NEVER};  // composition of the predecessors passed so far (nearest applied last)
    bool acc_id = true;
    long base = (long)chunk - 1;
    int spins = 0;
    while (true) {
        const long p = base - lane;
        u64 w = SLOT_INCL;  // before chunk 0: carry 0
        unsigned need;
        int f;
        while (true) {
            if (p >= 0) w = ld_acquire(&slots[p].word);
            const unsigned stop = __ballot_sync(0xFFFFFFFFu, (w & 3) == SLOT_CONST || (w & 3) == SLOT_INCL);
            const unsigned pub = __ballot_sync(0xFFFFFFFFu, (w & 3) != 0);
            f = stop ? __ffs(stop) - 1 : 31;  // lanes 0..f must be published
            need = f == 31 ? 0xFFFFFFFFu : ((2u << f) - 1);
            if ((pub & need) == need) break;
            if (++spins > LOOKBACK_SPIN_LIMIT) {  // gave up: report, use 0 and finish cleanly
                if (lane == 0) atomicOr(err, 1u);
                return 0;
            }
            __nanosleep(64);
        }
        CState mine{w >> 2, CS_NEVER};
        if ((w & 3) == SLOT_AGG) mine.t = *(volatile u64*)&slots[p].agg_t;
        const unsigned stop = __ballot_sync(0xFFFFFFFFu, (w & 3) != SLOT_AGG);
        if (stop & need) {
            // lane f is constant or inclusive: evaluate lanes f-1 .. 0 on its value
            u64 x = __shfl_sync(0xFFFFFFFFu, mine.h, f);
            for (int k = f - 1; k >= 0; --k) x = cs_eval(cs_shfl(mine, k), x);
            return acc_id ? x : cs_eval(acc, x);
        }
        // 32 thresholded aggregates: compose them (lane 31 applies first)
        CState blk = cs_shfl(mine, 31);
        for (int k = 30; k >= 0; --k) blk = cs_then(blk, cs_shfl(mine, k));
        acc = acc_id ? blk : cs_then(blk, acc);
        acc_id = false;
        if (acc.t == CS_NEVER) return acc.h;  // constant: earlier chunks cannot matter
        base -= 32;
    }
}

// SC: how the coefficients are scaled by N^-1 before the carry -- 0 not at all
// (the last inverse pass already did, through its scaled twiddle table),
// 1 by 2^nshift with nshift >= 160 (N a power of two), 2 by the multiply with
// ninv.
template <int SC>
__global__ void __launch_bounds__(CARRY_THREADS, CARRY_MIN_CTAS)
    k_carry(const u64* __restrict__ coef, u32* __restrict__ out, u64 nout, u32 nchunks, LookbackSlot* slots,
            u32* ticket, unsigned long long* out_len, u32* err, const ProdJob* __restrict__ jobs, u64 ninv,
            int nshift) {
    if (jobs) {
        const ProdJob& J = jobs[blockIdx.y];
        coef = J.bufB;
        out = J.out;
        nout = J.na + J.nb;
        slots = J.slots;
        ticket = J.ticket;
        out_len = J.out_len;
    }
    __shared__ ulonglong2 s_stage[CARRY_THREADS / 32][CARRY_WARP_PAIRS];
    __shared__ u32 s_chunk;
    __shared__ u64 s_cin;
    __shared__ unsigned long long s_top[CARRY_THREADS / 32];
    __shared__ u64 s_lasth[CARRY_THREADS / 32];
    __shared__ CState s_ws[CARRY_THREADS / 32 + 1];
    if (threadIdx.x == 0) s_chunk = atomicAdd(ticket, 1u);
    __syncthreads();
    const u32 chunk = s_chunk;
    if (chunk >= nchunks) return;
    const int warp = threadIdx.x >> 5;

    u64 cf[CARRY_G];
    load_chunk(coef, (u64)chunk * CARRY_CHUNK + (u64)warp * (32 * CARRY_G), s_stage[warp], cf);
    // The inverse transform leaves N * c (mod p) unless its last pass
    // already scaled: for N = 2^k the scale is the shift by 2^(192 - k)
    // (2 has order 192), otherwise one multiply.
    if constexpr (SC == 1) {
#pragma unroll
        for (int i = 0; i < CARRY_G; ++i) cf[i] = gl_shl_160(cf[i], nshift - 160);
    } else if constexpr (SC == 2) {
#pragma unroll
        for (int i = 0; i < CARRY_G; ++i) cf[i] = gl_mul(cf[i], ninv);
    }
    u32 lm[CARRY_G / 2];
    const CState st = group_carry<CARRY_G>(cf, lm);
    // park the limbs in the thread's own (already read) staging slots while
    // warp 0 walks back, so that the walk has the registers to itself; slot
    // i ^ (lane % 8) of the lane's eight keeps a quarter warp conflict-free
    const int lane = threadIdx.x & 31;
    {
        uint4* mine = reinterpret_cast<uint4*>(s_stage[warp] + lane * (CARRY_G / 2));
#pragma unroll
        for (int i = 0; i < CARRY_G / 8; ++i)
            mine[i ^ (lane & 7)] = make_uint4(lm[4 * i], lm[4 * i + 1], lm[4 * i + 2], lm[4 * i + 3]);
    }
    const u64 h_before = __shfl_up_sync(0xFFFFFFFFu, st.h, 1);
    if (lane == 31) s_lasth[warp] = st.h;
    u64 cin;
    if (!__syncthreads_or(st.t != CS_NEVER)) {
        // Every group's carry-out is independent of its carry-in (the usual
        // case): group k > 0 takes group k-1's carry-out, no scan needed, and
        // only thread 0 waits for the chunk's carry-in. The chunk's aggregate
        // is constant, which is all a successor needs.
        const CState agg{s_lasth[CARRY_THREADS / 32 - 1], CS_NEVER};
        cin = lane > 0 ? h_before : (warp > 0 ? s_lasth[warp - 1] : 0);
        if (warp == 0) {
            const u64 c = warp_lookback(slots, chunk, agg, err);
            if (lane == 0) cin = c;
        }
    } else {
        bool has_ex;
        CState agg;
        const CState ex = block_scan_carry(st, &has_ex, &agg, s_ws);
        if (warp == 0) {
            const u64 c = warp_lookback(slots, chunk, agg, err);
            if (threadIdx.x == 0) s_cin = c;
        }
        __syncthreads();
        const u64 cin_chunk = s_cin;
        // successors waiting on a thresholded aggregate need the inclusive value
        if (threadIdx.x == 0) st_release(&slots[chunk].word, (cs_eval(agg, cin_chunk) << 2) | SLOT_INCL);
        cin = has_ex ? cs_eval(ex, cin_chunk) : cin_chunk;
    }
    {
        const uint4* mine = reinterpret_cast<const uint4*>(s_stage[warp] + lane * (CARRY_G / 2));
#pragma unroll
        for (int i = 0; i < CARRY_G / 8; ++i) {
            const uint4 q = mine[i ^ (lane & 7)];
            lm[4 * i] = q.x, lm[4 * i + 1] = q.y, lm[4 * i + 2] = q.z, lm[4 * i + 3] = q.w;
        }
    }
    group_add_carry<CARRY_G / 2>(lm, cin);

    const u64 lbase = ((u64)chunk * CARRY_CHUNK + (u64)threadIdx.x * CARRY_G) / 2;
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
    // one length update per CTA
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, top, off);
        top = o > top ? o : top;
    }
    if ((threadIdx.x & 31) == 0) s_top[warp] = top;
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int w = 0; w < CARRY_THREADS / 32; ++w) top = s_top[w] > top ? s_top[w] : top;
        if (top) atomicMax(out_len, top);
    }
}

cudaError_t launch_carry(unsigned nchunks, cudaStream_t s, const u64* coef, u32* out, u64 nout,
                         LookbackSlot* slots, u32* ticket, unsigned long long* out_len, u32* err,
                         const ProdJob* jobs, unsigned njobs, u64 points) {
    if (nchunks == 0 || njobs == 0) return cudaSuccess;
    // the staging area takes 8 * CARRY_CHUNK bytes per CTA: ask for the
    // largest shared memory carveout so that CARRY_MIN_CTAS CTAs fit on an SM
    static const cudaError_t carveout = [] {
        cudaError_t e = cudaFuncSetAttribute(k_carry<0>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_carry<1>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_carry<2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        return e;
    }();
    if (carveout != cudaSuccess) return carveout;
    // scale by points^-1: a shift when points is a power of two (2^(192 - k),
    // k <= 32, is a shift by 160 + (32 - k)), else one multiply
    const dim3 grid(nchunks, njobs);
    if (points <= 1) {
        k_carry<0><<<grid, CARRY_THREADS, 0, s>>>(coef, out, nout, nchunks, slots, ticket, out_len, err, jobs, 1, 0);
    } else if ((points & (points - 1)) == 0 && points <= (1ull << 32)) {
        int k = 0;
        while ((1ull << k) < points) ++k;
        k_carry<1><<<grid, CARRY_THREADS, 0, s>>>(coef, out, nout, nchunks, slots, ticket, out_len, err, jobs, 1,
                                                  192 - k);
    } else {
        k_carry<2><<<grid, CARRY_THREADS, 0, s>>>(coef, out, nout, nchunks, slots, ticket, out_len, err, jobs,
                                                  gl_inv(points), -1);
    }
    return cudaGetLastError();
}

}  // namespace b2m
