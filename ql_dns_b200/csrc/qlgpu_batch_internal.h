// qlgpu_batch_internal.h -- entry points of the persistent batch used inside the
// library (the adjoint runs its forward sweep and window recompute for a batch
// of seeds through it).  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "../../include/qlgpu.h"
#include "qlgpu_types.h"

// Device buffers of case c at the batch's current buffer parity.
struct BatchCaseDev {
    qlgpu::cplx* lin;      // [nxy][4][nz] current fields
    qlgpu::cplx* mf;       // [nmf][nz]
    double* kx0;           // [nxy]
    qlgpu::DevClock* clk;  // the case's clock
    size_t nlin, nmfe;
    int nxy;
};

int qlgpu_batch_case_dev(qlgpu_batch_t* b, int c, BatchCaseDev* out);

// Record the stage inputs of case c during the following launches (null rec_lin: off):
// step n, stage s -> rec_lin + (3 n + s) nlin, rec_mf + (3 n + s) nmfe, rec_kx + n nxy, rec_t + n,
// rec_cn + 3 n + s (the Crank-Nicolson old-operator fields; may be null).
int qlgpu_batch_set_record(qlgpu_batch_t* b, int c, qlgpu::cplx* rec_lin, qlgpu::cplx* rec_mf, double* rec_kx,
                           double* rec_t, qlgpu::CnRec* rec_cn = nullptr);

cudaStream_t qlgpu_batch_cuda_stream(qlgpu_batch_t* b);
