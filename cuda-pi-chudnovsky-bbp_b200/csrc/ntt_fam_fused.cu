// ntt_fam_fused.cu -- instantiations and launchers: fused last pass of operand B (forward, pointwise, inverse).
// Kernel bodies are in ntt_kernels.cuh; one file per family keeps the
// heavily unrolled instantiations compiling in parallel.
#include "ntt_kernels.cuh"

namespace b2m {

cudaError_t launch_fused_last(int logr, const PassGeo& g, cudaStream_t s, u64* bbuf, const u64* aspec, u64 ninv, const RootTables& tw) {
    switch (logr) {
        case 7: k_fused_last<7><<<g.grid, g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw); break;
        case 8: k_fused_last<8><<<g.grid, g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw); break;
        case 9: k_fused_last<9><<<g.grid, g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw); break;
        case 10: k_fused_last<10><<<g.grid, g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw); break;
        case 11: k_fused_last<11><<<g.grid, g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw); break;
        case 12: k_fused_last<12><<<g.grid, g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw); break;
        case 13: k_fused_last<13><<<g.grid, g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw); break;
        case 14: k_fused_last<14><<<g.grid, g.block, g.smem, s>>>(bbuf, aspec, g.logc, ninv, tw); break;
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
