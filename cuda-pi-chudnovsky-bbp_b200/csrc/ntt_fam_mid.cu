// ntt_fam_mid.cu -- instantiations and launchers: middle forward passes and all non-last inverse passes.
// Kernel bodies are in ntt_kernels.cuh; one file per family keeps the
// unrolled instantiations compiling in parallel. With a job table the grid's
// second dimension (the first, for single-CTA products) runs over the jobs.
#include "ntt_kernels.cuh"

namespace b2m {

cudaError_t launch_fwd_mid(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw, const ProdJob* jobs, unsigned njobs, int operand) {
    switch (logr) {
        case 7: k_fwd_mid<7><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 8: k_fwd_mid<8><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 9: k_fwd_mid<9><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 10: k_fwd_mid<10><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 11: k_fwd_mid<11><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 12: k_fwd_mid<12><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

cudaError_t launch_inv_mid(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw, const ProdJob* jobs, unsigned njobs) {
    switch (logr) {
        case 7: k_inv_mid<7><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs); break;
        case 8: k_inv_mid<8><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs); break;
        case 9: k_inv_mid<9><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs); break;
        case 10: k_inv_mid<10><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs); break;
        case 11: k_inv_mid<11><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs); break;
        case 12: k_inv_mid<12><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(buf, g.logs, g.logc, g.logm, tw, jobs); break;
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
