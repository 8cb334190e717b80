// Stage kernels for NZ = 256 (all models, integrators and private-store backings).
#include "qlgpu_inst.cuh"

QLGPU_DEFINE_NZ(256)
