// ntt_fam_small.cu -- instantiations and launchers: single-CTA products, N <= 2^13.
// Written by gen_families.py; kernel bodies are in ntt_kernels.cuh. With a
// job table the grid's second dimension (the first, for single-CTA
// products) runs over the jobs.
#include "ntt_kernels.cuh"

namespace b2m {

cudaError_t launch_mul_small(int logn, const PassGeo& g, cudaStream_t s, const u32* a, u64 na, const u32* b, u64 nb, u32* out, u64 nout, unsigned long long* out_len, u64 ninv, const RootTables& tw, const ProdJob* jobs, unsigned njobs) {
    switch (logn) {
        case 2: k_mul_small<2><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 3: k_mul_small<3><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 4: k_mul_small<4><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 5: k_mul_small<5><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 6: k_mul_small<6><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 7: k_mul_small<7><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 8: k_mul_small<8><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 9: k_mul_small<9><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 10: k_mul_small<10><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 11: k_mul_small<11><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 12: k_mul_small<12><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        case 13: k_mul_small<13><<<dim3(g.grid * njobs), g.block, g.smem, s>>>(a, na, b, nb, out, nout, out_len, ninv, tw, jobs); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

cudaError_t configure_small() {
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<9>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<11>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mul_small<13>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    return e;
}

}  // namespace b2m
