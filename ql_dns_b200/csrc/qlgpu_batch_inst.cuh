// qlgpu_batch_inst.cuh -- launch wrapper and sizes of batch_kernel<MODEL, INTEG>,
// included by one translation unit per model x integrator.
#pragma once
#include "qlgpu_batch.cuh"
#include "qlgpu_host.h"

namespace qlgpu {

template <int MODEL, int INTEG, int MAXNZ>
cudaError_t batch_launch(const BatchLaunch& L, int grid, int block, size_t smem, cudaStream_t st) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;  // all CTAs co-resident, or the launch fails
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, batch_kernel<MODEL, INTEG, MAXNZ>, L);
}
template <int MODEL, int INTEG, int MAXNZ>
const void* batch_ptr() {
    return reinterpret_cast<const void*>(&batch_kernel<MODEL, INTEG, MAXNZ>);
}
template <int MODEL>
size_t batch_smem(int NZ, int warps) {
    switch (NZ) {
        case 16: return StageKind<16, MODEL, true, BatchStaging<16>::ON>::SM::bytes(warps);
        case 32: return StageKind<32, MODEL, true, BatchStaging<32>::ON>::SM::bytes(warps);
        case 64: return StageKind<64, MODEL, true, BatchStaging<64>::ON>::SM::bytes(warps);
        case 128: return StageKind<128, MODEL, true, BatchStaging<128>::ON>::SM::bytes(warps);
        case 256: return StageKind<256, MODEL, true, BatchStaging<256>::ON>::SM::bytes(warps);
        default: return 0;
    }
}
template <int MODEL>
int batch_tmem(int NZ, int warps) {
    switch (NZ) {
        case 16: return StageKind<16, MODEL, true, BatchStaging<16>::ON>::SM::tmem_cols(warps);
        case 32: return StageKind<32, MODEL, true, BatchStaging<32>::ON>::SM::tmem_cols(warps);
        case 64: return StageKind<64, MODEL, true, BatchStaging<64>::ON>::SM::tmem_cols(warps);
        case 128: return StageKind<128, MODEL, true, BatchStaging<128>::ON>::SM::tmem_cols(warps);
        case 256: return StageKind<256, MODEL, true, BatchStaging<256>::ON>::SM::tmem_cols(warps);
        default: return 0;
    }
}
template <int MODEL, int INTEG>
bool make_batch_kernel(bool wide, BatchKernel* out) {
    out->launch = wide ? &batch_launch<MODEL, INTEG, 256> : &batch_launch<MODEL, INTEG, 64>;
    out->kernel = wide ? &batch_ptr<MODEL, INTEG, 256> : &batch_ptr<MODEL, INTEG, 64>;
    out->smem = &batch_smem<MODEL>;
    out->tmem = &batch_tmem<MODEL>;
    out->max_nz = wide ? 256 : 64;
    out->max_warps = (wide ? BatchOcc<256>::MAX_THREADS : BatchOcc<64>::MAX_THREADS) / 32;
    return true;
}

}  // namespace qlgpu
