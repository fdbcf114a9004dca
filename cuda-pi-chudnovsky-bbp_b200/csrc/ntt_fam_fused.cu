// ntt_fam_fused.cu -- instantiations and launchers: fused last pass of operand B (forward, pointwise, inverse).
// Kernel bodies are in ntt_kernels.cuh; one file per family keeps the
// unrolled instantiations compiling in parallel. With a job table the grid's
// second dimension (the first, for single-CTA products) runs over the jobs.
#include "ntt_kernels.cuh"

namespace b2m {

cudaError_t launch_fused_last(int logr, const PassGeo& g, cudaStream_t s, u64* bbuf, const u64* aspec, u64 ninv, const RootTables& tw, const ProdJob* jobs, unsigned njobs) {
    switch (logr) {
        case 7: k_fused_last<7><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw, jobs); break;
        case 8: k_fused_last<8><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw, jobs); break;
        case 9: k_fused_last<9><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw, jobs); break;
        case 10: k_fused_last<10><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw, jobs); break;
        case 11: k_fused_last<11><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw, jobs); break;
        case 12: k_fused_last<12><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw, jobs); break;
        case 13: k_fused_last<13><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw, jobs); break;
        case 14: k_fused_last<14><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw, jobs); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

cudaError_t configure_fused() {
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fused_last<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fused_last<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fused_last<9>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fused_last<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fused_last<11>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fused_last<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fused_last<13>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fused_last<14>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    return e;
}

}  // namespace b2m
