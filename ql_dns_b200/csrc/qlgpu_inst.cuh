// qlgpu_inst.cuh -- the stage-variant table for one NZ: launch wrappers and
// sizes of stage_kernel<NZ, model, integrator, TMEM|smem>.  Included by one
// translation unit per NZ (qlgpu_nz<NZ>.cu) so the variants compile in parallel.
#pragma once
#include <type_traits>

#include "qlgpu_host.h"
#include "qlgpu_kernel.cuh"

namespace qlgpu {

template <int NZ, int MODEL, int INTEG, bool TM>
void launch_stage(const StageArgs& A, const DevParams& P, int grid, int block, size_t smem, cudaStream_t st) {
    stage_kernel<NZ, MODEL, INTEG, TM><<<grid, block, smem, st>>>(A, P);
}
template <int NZ, int MODEL, int INTEG, bool TM>
const void* stage_ptr() {
    return reinterpret_cast<const void*>(&stage_kernel<NZ, MODEL, INTEG, TM>);
}
template <int NZ, int MODEL, bool TM>
size_t stage_smem(int warps) {
    return StageKind<NZ, MODEL, TM>::SM::bytes(warps);
}
template <int NZ, int MODEL, bool TM>
int stage_tmem(int warps) {
    return StageKind<NZ, MODEL, TM>::SM::tmem_cols(warps);
}
template <int NZ>
void launch_diag(const cplx* lin, const cplx* mf, const double* kx0, const double* ky, const int* kxi, const int* kyi,
                 const DevParams& P, double t, double* out, cudaStream_t st) {
    diag_kernel<NZ><<<1, 128, 0, st>>>(lin, mf, kx0, ky, kxi, kyi, P, t, out);
}

template <int NZ, int MODEL, int INTEG, bool TM>
Variant make_variant() {
    Variant v;
    v.launch = &launch_stage<NZ, MODEL, INTEG, TM>;
    v.kernel = &stage_ptr<NZ, MODEL, INTEG, TM>;
    v.smem = &stage_smem<NZ, MODEL, TM>;
    v.tmem = &stage_tmem<NZ, MODEL, TM>;
    v.diag = &launch_diag<NZ>;
    v.T = Geom<NZ>::T;
    v.PL = StageKind<NZ, MODEL, TM>::SM::PL;
    v.max_warps = StageOcc<NZ>::MAX_THREADS / 32;
    return v;
}

template <int NZ>
bool make_variant_for(int model, int integ, bool tm, Variant* out) {
    if (model == MODEL_BQLIN && integ == INTEG_EXP)
        *out = tm ? make_variant<NZ, MODEL_BQLIN, INTEG_EXP, true>() : make_variant<NZ, MODEL_BQLIN, INTEG_EXP, false>();
    else if (model == MODEL_BQLIN && integ == INTEG_CN)
        *out = tm ? make_variant<NZ, MODEL_BQLIN, INTEG_CN, true>() : make_variant<NZ, MODEL_BQLIN, INTEG_CN, false>();
    else if (model == MODEL_FULLQLIN && integ == INTEG_EXP)
        *out = tm ? make_variant<NZ, MODEL_FULLQLIN, INTEG_EXP, true>()
                  : make_variant<NZ, MODEL_FULLQLIN, INTEG_EXP, false>();
    else if (model == MODEL_FULLQLIN && integ == INTEG_CN)
        *out = tm ? make_variant<NZ, MODEL_FULLQLIN, INTEG_CN, true>()
                  : make_variant<NZ, MODEL_FULLQLIN, INTEG_CN, false>();
    else
        return false;
    return true;
}

}  // namespace qlgpu

#define QLGPU_DEFINE_NZ(NZV)                                                 \
    namespace qlgpu {                                                        \
    bool make_variant_nz##NZV(int model, int integ, bool tm, Variant* out) { \
        return make_variant_for<NZV>(model, integ, tm, out);                 \
    }                                                                        \
    }
