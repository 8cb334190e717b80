// Stage kernels for NZ = 32 (all models, integrators and private-store backings).
#include "qlgpu_inst.cuh"

QLGPU_DEFINE_NZ(32)
