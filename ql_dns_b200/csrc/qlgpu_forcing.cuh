// qlgpu_forcing.cuh -- driving noise and the CFL time step of the QL models
// (sm_100a).
//
// noise_kernel: Model::DrivingNoise after a step of a single handle, one
// thread per (mode, kz) and the four fields (noise_value of qlgpu_noise.cuh).
// Modes that the step's remap zeroed (kx0 changed) are skipped: the reference
// adds their noise before the remap zeroes them (main.cpp:111-123).
//
// mf_absmax2_kernel: max over the NZ grid of |profile|^2 of each mean field, the
// real-space maxima Calculate_CFL reads (MHD_BQlin.cpp:540-552,
// MHD_FullQlin.cpp:769-780), by a direct sum over the stored kz.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "qlgpu_fft.cuh"
#include "qlgpu_noise.cuh"

namespace qlgpu {

struct NoiseArgs {
    cplx* lin;               // [nxy][4][nz]
    const double* kx0_prev;  // kx0 at the start of the step
    const double* kx0_now;   // after the step's remap
    const double* ky;
    const int* kxi;
    const int* kyi;
    int nxy, nz;
    double q, t, kzL;
    unsigned long long step;
    NoiseSpec ns;
};

__global__ void noise_kernel(NoiseArgs a) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.nxy * a.nz) return;
    const int i = idx / a.nz, k = idx % a.nz;
    const double kx0 = a.kx0_prev[i];
    if (a.kx0_now[i] != kx0) return;  // remapped: zeroed after its noise in the reference
    const double ky = a.ky[i];
    const int kxi = a.kxi[i], kyi = a.kyi[i];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        cplx n;
        if (!noise_value(a.ns, a.step, i, k, v, a.nz, kx0, ky, kxi, kyi, a.q, a.t, a.kzL, &n)) continue;
        cplx* p = a.lin + ((size_t)i * 4 + v) * a.nz + k;
        cplx u = *p;
        u.x = __dadd_rn(u.x, n.x);
        u.y = __dadd_rn(u.y, n.y);
        *p = u;
    }
}

// out[m] = max_z |sum_s fac mf[m][s] e^{+2 pi i kz_s z / NZ}|^2, one block.
__global__ void mf_absmax2_kernel(const cplx* mf, int nmf, int nz, int NZ, double fac, double* out) {
    __shared__ double red[256];
    const int H = (nz - 1) / 2;
    for (int m = 0; m < nmf; ++m) {
        double mx = 0.0;
        for (int z = threadIdx.x; z < NZ; z += blockDim.x) {
            double re = 0.0, im = 0.0;
            for (int s = 0; s < nz; ++s) {
                const int kzi = s <= H ? s : s - nz;
                const int ph = ((kzi * z) % NZ + NZ) % NZ;
                double sn, cs;
                sincospi(2.0 * (double)ph / (double)NZ, &sn, &cs);
                const cplx f = mf[(size_t)m * nz + s];
                re += fac * (f.x * cs - f.y * sn);
                im += fac * (f.x * sn + f.y * cs);
            }
            mx = fmax(mx, re * re + im * im);
        }
        red[threadIdx.x] = mx;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
            __syncthreads();
        }
        if (threadIdx.x == 0) out[m] = red[0];
        __syncthreads();
    }
}

}  // namespace qlgpu
