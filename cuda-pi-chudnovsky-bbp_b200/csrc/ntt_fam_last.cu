// ntt_fam_last.cu -- instantiations and launchers: last forward pass of operand A.
// Written by gen_families.py; kernel bodies are in ntt_kernels.cuh. With a
// job table the grid's second dimension (the first, for single-CTA
// products) runs over the jobs.
#include "ntt_kernels.cuh"

namespace b2m {

cudaError_t launch_fwd_last(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw, const ProdJob* jobs, unsigned njobs) {
    switch (logr * 32 + g.logc) {
        case 198: k_fwd_last<6, 6><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 229: k_fwd_last<7, 5><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 260: k_fwd_last<8, 4><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 291: k_fwd_last<9, 3><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 322: k_fwd_last<10, 2><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 353: k_fwd_last<11, 1><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 384: k_fwd_last<12, 0><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 199: k_fwd_last<6, 7><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 230: k_fwd_last<7, 6><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 261: k_fwd_last<8, 5><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 292: k_fwd_last<9, 4><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 323: k_fwd_last<10, 3><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 354: k_fwd_last<11, 2><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 385: k_fwd_last<12, 1><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 416: k_fwd_last<13, 0><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 200: k_fwd_last<6, 8><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 231: k_fwd_last<7, 7><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 262: k_fwd_last<8, 6><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 293: k_fwd_last<9, 5><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 324: k_fwd_last<10, 4><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 355: k_fwd_last<11, 3><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 386: k_fwd_last<12, 2><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 417: k_fwd_last<13, 1><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        case 448: k_fwd_last<14, 0><<<dim3(g.grid, njobs, g.zdim), g.block, g.smem, s>>>(buf, tw, jobs, g.zstride); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

cudaError_t configure_last() {
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<6, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<7, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<9, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<10, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<11, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<12, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<6, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<7, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<8, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<9, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<10, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<11, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<12, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<13, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<6, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<7, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<8, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<9, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<10, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<11, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<12, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<13, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_last<14, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    return e;
}

}  // namespace b2m
