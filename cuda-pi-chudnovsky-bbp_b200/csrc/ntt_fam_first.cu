// ntt_fam_first.cu -- instantiations and launchers: first forward pass (u32 limbs in).
// Written by gen_families.py; kernel bodies are in ntt_kernels.cuh. With a
// job table the grid's second dimension (the first, for single-CTA
// products) runs over the jobs.
#include "ntt_kernels.cuh"

namespace b2m {

cudaError_t launch_fwd_first(int logr, const PassGeo& g, cudaStream_t s, const u32* limbs, u64 ndig, u64* out, const RootTables& tw, const ProdJob* jobs, unsigned njobs, int operand) {
    switch (logr * 32 + g.logc) {
        case 198: k_fwd_first<6, 6><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 229: k_fwd_first<7, 5><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 260: k_fwd_first<8, 4><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 291: k_fwd_first<9, 3><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 322: k_fwd_first<10, 2><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 353: k_fwd_first<11, 1><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 384: k_fwd_first<12, 0><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 199: k_fwd_first<6, 7><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 230: k_fwd_first<7, 6><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 261: k_fwd_first<8, 5><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 292: k_fwd_first<9, 4><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 323: k_fwd_first<10, 3><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 354: k_fwd_first<11, 2><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 385: k_fwd_first<12, 1><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 200: k_fwd_first<6, 8><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 231: k_fwd_first<7, 7><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 262: k_fwd_first<8, 6><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 293: k_fwd_first<9, 5><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 324: k_fwd_first<10, 4><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 355: k_fwd_first<11, 3><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        case 386: k_fwd_first<12, 2><<<dim3(g.grid, njobs), g.block, g.smem, s>>>(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

cudaError_t configure_first() {
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<6, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<7, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<9, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<10, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<11, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<12, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<6, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<7, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<8, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<9, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<10, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<11, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<12, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<6, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<7, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<8, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<9, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<10, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<11, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_first<12, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    return e;
}

}  // namespace b2m
