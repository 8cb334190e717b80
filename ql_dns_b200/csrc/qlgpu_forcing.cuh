// qlgpu_forcing.cuh -- driving noise and the CFL time step of the QL models
// (sm_100a).
//
// noise_kernel: Model::DrivingNoise of MHD_BQlin (QL_DNS/Models/MHD_BQlin.cpp:
// 558-618) after a step, one thread per (mode, kz): ky = 0 modes are not driven
// (dont_drive_ky0_modes_ = 1, :18); a mode is driven where lo^2 < |k(t)|^2 < hi^2
// (t = the step's start time) with amplitudes sqrt(m lap2 / lapF) on (u, b) and
// sqrt(-m lap2) on (zeta, eta), m = dt (Nx Ny NZ)^2 / (16 32 32)^2 (:33-36), of
// complex normals of standard deviation f_noise/sqrt(2) per part (:23).  The
// reference's clock-seeded mt19937 cannot be reproduced; every (step, mode, kz,
// field) draws from its own Philox4x32-10 counter instead (Salmon et al., SC'11),
// Box-Muller on two 53-bit uniforms, the same numbers as the oracle.  Modes that
// the step's remap zeroed (kx0 changed) are skipped: the reference adds their
// noise before the remap zeroes them (main.cpp:111-123).
//
// mf_absmax2_kernel: max over the NZ grid of |profile|^2 of each mean field, the
// real-space maxima Calculate_CFL reads (MHD_BQlin.cpp:540-552,
// MHD_FullQlin.cpp:769-780), by a direct sum over the stored kz.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "qlgpu_fft.cuh"

namespace qlgpu {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += W0; k1 += W1; }
        const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
        const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    }
}

__device__ __forceinline__ void philox_normal_pair(unsigned long long seed, unsigned long long step, uint32_t a,
                                                   uint32_t b, double* z1, double* z2) {
    uint32_t c[4] = {a, b, (uint32_t)step, (uint32_t)(step >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const unsigned long long x = ((unsigned long long)c[0] << 32) | c[1];
    const unsigned long long y = ((unsigned long long)c[2] << 32) | c[3];
    const double u1 = ((double)(x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(y >> 11) * (1.0 / 9007199254740992.0);
    const double r = sqrt(-2.0 * log(u1));
    const double ang = __dmul_rn(2.0 * 3.14159265358979323846, u2);
    *z1 = r * cos(ang);
    *z2 = r * sin(ang);
}

struct NoiseArgs {
    cplx* lin;               // [nxy][4][nz]
    const double* kx0_prev;  // kx0 at the start of the step
    const double* kx0_now;   // after the step's remap
    const double* ky;
    const int* kyi;
    int nxy, nz;
    double q, t, kzL, lo2, hi2, multfac, sd;
    unsigned long long seed, step;
};

__global__ void noise_kernel(NoiseArgs a) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.nxy * a.nz) return;
    const int i = idx / a.nz, k = idx % a.nz;
    if (a.kyi[i] == 0) return;
    const double kx0 = a.kx0_prev[i];
    if (a.kx0_now[i] != kx0) return;  // remapped: zeroed after its noise in the reference
    const double ky = a.ky[i];
    const int H = (a.nz - 1) / 2;
    const int kzi = k <= H ? k : k - a.nz;  // Kdata.cpp:74-78
    const double c = __dmul_rn((double)kzi, a.kzL);
    const double kz2 = -__dmul_rn(c, c);
    const double lap2 = __dadd_rn(-__dmul_rn(ky, ky), kz2);  // Kdata.cpp:100-119
    const double kx = __dadd_rn(kx0, __dmul_rn(__dmul_rn(a.q, a.t), ky));
    const double lapF = __dadd_rn(-__dmul_rn(kx, kx), lap2);  // MHD_BQlin.cpp:498-503
    if (!(lapF > -a.hi2 && lapF < -a.lo2)) return;
    const double mu = sqrt(__ddiv_rn(__dmul_rn(a.multfac, lap2), lapF));
    const double mz = sqrt(-__dmul_rn(a.multfac, lap2));
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        double z1, z2;
        philox_normal_pair(a.seed, a.step, (uint32_t)i, (uint32_t)(4 * k + v), &z1, &z2);
        const double m = (v == 0 || v == 2) ? mu : mz;
        cplx* p = a.lin + ((size_t)i * 4 + v) * a.nz + k;
        cplx u = *p;
        u.x = __dadd_rn(u.x, __dmul_rn(m, __dmul_rn(z1, a.sd)));
        u.y = __dadd_rn(u.y, __dmul_rn(m, __dmul_rn(z2, a.sd)));
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
