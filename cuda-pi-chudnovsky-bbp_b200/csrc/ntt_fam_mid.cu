// ntt_fam_mid.cu -- instantiations and launchers: middle forward passes and all non-last inverse passes.
// Kernel bodies are in ntt_kernels.cuh; one file per family keeps the
// heavily unrolled instantiations compiling in parallel.
#include "ntt_kernels.cuh"

namespace b2m {

cudaError_t launch_fwd_mid(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw) {
    switch (logr) {
        case 7: k_fwd_mid<7><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 8: k_fwd_mid<8><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 9: k_fwd_mid<9><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 10: k_fwd_mid<10><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 11: k_fwd_mid<11><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 12: k_fwd_mid<12><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

cudaError_t launch_inv_mid(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw) {
    switch (logr) {
        case 7: k_inv_mid<7><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 8: k_inv_mid<8><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 9: k_inv_mid<9><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 10: k_inv_mid<10><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 11: k_inv_mid<11><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        case 12: k_inv_mid<12><<<g.grid, g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

cudaError_t configure_mid() {
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_mid<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_mid<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_mid<9>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_mid<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_mid<11>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_mid<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_inv_mid<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_inv_mid<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_inv_mid<9>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_inv_mid<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_inv_mid<11>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_inv_mid<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    return e;
}

}  // namespace b2m
