// pdm1_stage_fp32.cu -- the stage kernels with a single-precision stencil.
//
// WENO-Z, the interface projection, the HLL flux and the divergence run in
// float from a float shared-memory tile; the stage update, the cell
// projection near |J|/phi -> 1, the CFL bound and the dose accumulation stay
// in double (pdm1_stage.cuh).  Compiled with --use_fast_math: approximate
// division and square root in the float stencil, FMA contraction throughout.
// One instantiation per tile shape of kTiles.
#include "pdm1_stage.cuh"

namespace pdm1 {

namespace {

template <class Tl>
cudaError_t set_attributes() {
    const int bytes = (int)Tl::template smem_bytes<float>();
    const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<float, MODE_A, Tl>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<float, MODE_B, Tl>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<float, MODE_C, Tl>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<float, MODE_C, Tl, true>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<float, MODE_EULER, Tl>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<float, MODE_RHS, Tl>, attr, bytes);
    return e;
}

template <class Tl>
void launch(int mode, int grid, const StageArgs &a, cudaStream_t stream) {
    const size_t bytes = Tl::template smem_bytes<float>();
    constexpr int nt = Tl::NT;
    switch (mode) {
    case MODE_A: stage_kernel<float, MODE_A, Tl><<<grid, nt, bytes, stream>>>(a); break;
    case MODE_B: stage_kernel<float, MODE_B, Tl><<<grid, nt, bytes, stream>>>(a); break;
    case MODE_C: stage_kernel<float, MODE_C, Tl><<<grid, nt, bytes, stream>>>(a); break;
    case MODE_C_LEARN: stage_kernel<float, MODE_C, Tl, true><<<grid, nt, bytes, stream>>>(a); break;
    case MODE_EULER: stage_kernel<float, MODE_EULER, Tl><<<grid, nt, bytes, stream>>>(a); break;
    default: stage_kernel<float, MODE_RHS, Tl><<<grid, nt, bytes, stream>>>(a); break;
    }
}

}  // namespace

int stage_fp32_set_attributes() {
    cudaError_t e = set_attributes<Tile0>();
    if (e == cudaSuccess) e = set_attributes<Tile1>();
    if (e == cudaSuccess) e = set_attributes<Tile2>();
    return (int)e;
}

void launch_stage_fp32(int mode, int tile_id, int grid, const StageArgs &a, cudaStream_t stream) {
    switch (tile_id) {
    case 1: launch<Tile1>(mode, grid, a, stream); break;
    case 2: launch<Tile2>(mode, grid, a, stream); break;
    default: launch<Tile0>(mode, grid, a, stream); break;
    }
}

}  // namespace pdm1
