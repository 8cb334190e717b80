// Persistent batch kernel for MHD_BQlin with RK3CN_Elin (NZ = 16 ... 256 in one kernel).
#include "qlgpu_batch_inst.cuh"

namespace qlgpu {
bool batch_kernel_bq_exp(bool wide, BatchKernel* out) { return make_batch_kernel<MODEL_BQLIN, INTEG_EXP>(wide, out); }
}  // namespace qlgpu
