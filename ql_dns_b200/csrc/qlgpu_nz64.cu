// Stage kernels for NZ = 64 (all models, integrators and private-store backings).
#include "qlgpu_inst.cuh"

QLGPU_DEFINE_NZ(64)
