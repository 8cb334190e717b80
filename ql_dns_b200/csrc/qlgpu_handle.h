// qlgpu_handle.h -- the single-case handle (struct qlgpu_handle) shared by the
// translation units of the library that drive it (qlgpu.cu, qlgpu_adjoint.cu).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/qlgpu.h"
#include "qlgpu_guard.h"
#include "qlgpu_host.h"
#include "qlgpu_types.h"

using namespace qlgpu;

struct qlgpu_handle {
    qlgpu_params p;
    DevParams dp;
    Variant var;
    int device = 0;
    cudaStream_t stream = nullptr;
    int nxy = 0, nz = 0, NZ = 0, nmf = 0;
    cplx* d_lin[2] = {nullptr, nullptr};
    int cur = 0;
    cplx* d_F1 = nullptr;
    cplx* d_F2 = nullptr;
    cplx* d_mf = nullptr;
    cplx* d_Fmf1 = nullptr;
    cplx* d_Fmf2 = nullptr;
    double* d_kx0 = nullptr;
    double* d_ky = nullptr;
    int* d_kxi = nullptr;
    int* d_kyi = nullptr;
    cplx* d_tw = nullptr;
    double* d_partials = nullptr;
    double* d_gpartials = nullptr;
    DevClock* d_clk = nullptr;
    double* d_diag = nullptr;
    int diag_cap = 0;
    double* d_out15 = nullptr;
    double* d_linop = nullptr;
    double* d_ilap2 = nullptr;
    int tmem_cols = 0;
    int per_sm = 0;
    unsigned long long* d_trace = nullptr;
    double* d_mfr = nullptr;  // [8][NZ] mean-field profile cache
    double* d_ekz = nullptr;  // [3 stages][2][nz]  // QLGPU_TRACE=1: %globaltimer stamps of each stage
    int grid = 0, warps = 4, block = 128;
    size_t smem = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    qlgpu::GuardList guards;  // debug build: canary zones after the device buffers
    int* d_dbg = nullptr;     // debug-build index checks of the adjoint kernels (the clock is restored there)
    std::vector<double> kx_tab, ky_tab;
    std::vector<int> kxi_tab, kyi_tab;
    std::vector<double> il2_tab, ekz_tab;
    StageConst sc[3];
    std::string err;
    // forcing (include/qlgpu.h: qlgpu_set_noise, qlgpu_set_cfl)
    double noise_f = 0.0, noise_klo = 0.0, noise_khi = 0.0;
    unsigned long long noise_seed = 0;
    int noise_only_vel = 0, noise_only_mag = 0;  // MHD_FullQlin drive_only_* switches
    double cfl = 0.0, dt_max = 0.0;
    double dt_sum = 0.0;                 // Integrator::mean_time_step accumulators
    unsigned long long steps_taken = 0;  // since set_state; the noise counter's step word
    double* d_forcing = nullptr;         // [0..3] last rhs mean-field maxima, [4..7] current, [8] step start time
    double* d_kx0_prev = nullptr;        // kx0 at the start of the step (noise)
    bool ekz_dynamic = false;            // stage exp(kz) factors computed in the kernel (variable dt)
};


// One step of the handle's state on its stream (three stage launches); hook,
// when set, runs on the host before each stage launch with the stage index.
void qlgpu_enqueue_step(qlgpu_t* h, cudaEvent_t* ev, const std::function<void(int)>& hook);

// Debug build: the index checks' status bits and the guard zones of the handle after a
// call's launches (QLGPU_ERR_STATUS when one fired).  QLGPU_OK at once in a release build.
int qlgpu_debug_verify(qlgpu_t* h);
