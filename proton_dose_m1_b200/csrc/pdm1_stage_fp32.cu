// pdm1_stage_fp32.cu -- the stage kernels with a single-precision stencil.
//
// WENO-Z, the interface projection, the HLL flux and the divergence run in
// float from a float shared-memory tile; the stage update, the cell
// projection near |J|/phi -> 1, the CFL bound and the dose accumulation stay
// in double (pdm1_stage.cuh).  Compiled with --use_fast_math: approximate
// division and square root in the float stencil, FMA contraction throughout.
#include "pdm1_stage.cuh"

namespace pdm1 {

int stage_fp32_set_attributes() {
    const int bytes = (int)stage_smem_bytes<float>();
    cudaError_t e = cudaSuccess;
    e = cudaFuncSetAttribute(stage_kernel<float, MODE_A>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stage_kernel<float, MODE_B>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stage_kernel<float, MODE_C>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stage_kernel<float, MODE_EULER>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stage_kernel<float, MODE_RHS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return (int)e;
}

void launch_stage_fp32(int mode, int grid, const StageArgs &a, cudaStream_t stream) {
    const size_t bytes = stage_smem_bytes<float>();
    switch (mode) {
    case MODE_A: stage_kernel<float, MODE_A><<<grid, NT, bytes, stream>>>(a); break;
    case MODE_B: stage_kernel<float, MODE_B><<<grid, NT, bytes, stream>>>(a); break;
    case MODE_C: stage_kernel<float, MODE_C><<<grid, NT, bytes, stream>>>(a); break;
    case MODE_EULER: stage_kernel<float, MODE_EULER><<<grid, NT, bytes, stream>>>(a); break;
    default: stage_kernel<float, MODE_RHS><<<grid, NT, bytes, stream>>>(a); break;
    }
}

}  // namespace pdm1
