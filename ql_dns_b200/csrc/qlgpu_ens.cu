// The chunk-queue engine of the batched ensemble (qlgpu_ens.cuh): launch
// wrappers of its persistent kernel for RK3CN_Elin and RK3CN.
#include <cstring>

#include "qlgpu_ens.cuh"
#include "qlgpu_ens_host.h"

namespace qlgpu {
namespace ens {

template <int INTEG, bool REC>
static cudaError_t launch_t(const EnsLaunch& L, int grid, size_t smem, cudaStream_t st) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;  // all CTAs co-resident, or the launch fails
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, ens_kernel<INTEG, REC>, L);
}

cudaError_t launch(int integ, bool rec, const EnsLaunch& L, int grid, size_t smem, cudaStream_t st) {
    if (rec)
        return integ == INTEG_EXP ? launch_t<INTEG_EXP, true>(L, grid, smem, st)
                                  : launch_t<INTEG_CN, true>(L, grid, smem, st);
    return integ == INTEG_EXP ? launch_t<INTEG_EXP, false>(L, grid, smem, st)
                              : launch_t<INTEG_CN, false>(L, grid, smem, st);
}

const void* kernel(int integ, bool rec) {
    if (rec)
        return integ == INTEG_EXP ? reinterpret_cast<const void*>(&ens_kernel<INTEG_EXP, true>)
                                  : reinterpret_cast<const void*>(&ens_kernel<INTEG_CN, true>);
    return integ == INTEG_EXP ? reinterpret_cast<const void*>(&ens_kernel<INTEG_EXP, false>)
                              : reinterpret_cast<const void*>(&ens_kernel<INTEG_CN, false>);
}

size_t smem_bytes(int NZ) { return chunk_smem(NZ); }
int threads() { return THREADS; }
int modes_per_pass(int NZ) { return pass_modes(NZ); }

}  // namespace ens
}  // namespace qlgpu
