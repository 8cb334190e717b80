// qlgpu_ens_host.h -- host view of the chunk-queue engine (qlgpu_ens.cuh):
// the launch wrapper and the sizes the batch host code needs.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "qlgpu_types.h"

namespace qlgpu {
namespace ens {

// rec: the build that records every stage's inputs (qlgpu_batch_set_record on some case)
cudaError_t launch(int integ, bool rec, const EnsLaunch& L, int grid, size_t smem, cudaStream_t st);
int threads();               // threads per CTA of the persistent kernel
const void* kernel(int integ, bool rec);
size_t smem_bytes(int NZ);   // dynamic shared memory of one NZ class (16, 32, 64, 128)
int modes_per_pass(int NZ);  // modes a CTA steps at once

}  // namespace ens
}  // namespace qlgpu
