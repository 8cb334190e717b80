// Stage kernels for NZ = 128 (all models, integrators and private-store backings).
#include "qlgpu_inst.cuh"

QLGPU_DEFINE_NZ(128)
