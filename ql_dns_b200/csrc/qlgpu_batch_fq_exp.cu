// Persistent batch kernel for MHD_FullQlin with RK3CN_Elin (NZ = 16 ... 256 in one kernel).
#include "qlgpu_batch_inst.cuh"

namespace qlgpu {
bool batch_kernel_fq_exp(bool wide, BatchKernel* out) { return make_batch_kernel<MODEL_FULLQLIN, INTEG_EXP>(wide, out); }
}  // namespace qlgpu
