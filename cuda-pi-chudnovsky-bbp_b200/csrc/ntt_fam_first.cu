// ntt_fam_first.cu -- instantiations and launchers: first forward pass (u32 limbs in).
// Kernel bodies are in ntt_kernels.cuh; one file per family keeps the
// unrolled instantiations compiling in parallel. With a job table the grid's
// second dimension (the first, for single-CTA products) runs over the jobs.
#include "ntt_kernels.cuh"

namespace b2m {

cudaError_t launch_fwd_first(int logr, const PassGeo& g, cudaStream_t s, const u32* limbs, u64 ndig, u64* out, const RootTables& tw, const ProdJob* jobs, unsigned njobs, int operand) {
    switch (logr) {
        case 7: k_fwd_first<7><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 8: k_fwd_first<8><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 9: k_fwd_first<9><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 10: k_fwd_first<10><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 11: k_fwd_first<11><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        case 12: k_fwd_first<12><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logc, g.logm, tw, jobs, operand); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

cudaError_t configure_first() {
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<9>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<11>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    return e;
}

}  // namespace b2m
