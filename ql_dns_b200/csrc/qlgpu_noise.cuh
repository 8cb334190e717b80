// qlgpu_noise.cuh -- the driving noise of the QL models (Model::DrivingNoise),
// one value per (mode, kz, field) from a counter-based generator.
//
// MHD_BQlin (QL_DNS/Models/MHD_BQlin.cpp:558-618) and MHD_FullQlin
// (MHD_FullQlin.cpp:786-1045) add, after a step that started at t, complex
// normals of standard deviation f_noise/sqrt(2) per part (:45) to every mode
// with lo^2 < |k(t)|^2 < hi^2: amplitude sqrt(m lap2 / lapF) on u and b,
// sqrt(-m lap2) on zeta and eta, m = dt (Nx Ny NZ)^2 / (16 32 32)^2.  Modes
// with ky = 0 are skipped by MHD_BQlin (dont_drive_ky0_modes_ = 1,
// MHD_BQlin.cpp:18).  MHD_FullQlin drives them (dont_drive_ky0_modes_ = 0,
// MHD_FullQlin.cpp:19) so that the field stays real: the kx < 0 mode of each
// pair (Kdata.cpp:124-146) draws noise at kz indices 1..nz-1 (:969-1023) and
// its kx > 0 partner receives the conjugate at the mirrored index,
// pos[k] += conj(noise_neg[nz - k]) (:1028-1040); kz = 0 stays undriven.
// drive_only_velocity / drive_only_magnetic (:21-22) switch off the magnetic
// (b, eta) or velocity (u, zeta) fields.
//
// The reference's clock-seeded mt19937 cannot be reproduced; every (step, mode,
// kz, field) draws from its own Philox4x32-10 counter (Salmon et al., SC'11),
// Box-Muller on two 53-bit uniforms, the same numbers as the oracle.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "qlgpu_fft.cuh"
#include "qlgpu_types.h"

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

// The noise added to field v (0 u, 1 zeta, 2 b, 3 eta) of mode i at stored kz
// index k by the step with counter `step` that started at t; kx0 is the mode's
// unsheared kx before the step's remap.  Returns false where nothing is added.
// The kx < 0 partner of a ky = 0 mode has unsheared kx -kx0 (ky = 0 modes never
// shear nor remap), so its |k|^2 is this mode's at the mirrored kz.
__device__ __forceinline__ bool noise_value(const NoiseSpec& ns, unsigned long long step, int i, int k, int v,
                                            int nz, double kx0, double ky, int kxi, int kyi, double q, double t,
                                            double kzL, cplx* out) {
    if (v < 2 ? !ns.drive_u : !ns.drive_b) return false;
    int src = i, kk = k;
    bool mirror = false;
    if (kyi == 0) {
        if (!ns.pair_ky0 || kxi == 0 || k == 0) return false;
        if (kxi > 0) {  // Kdata.cpp:39-46: kx index -a sits at position 2 Nx/2 - a - 1
            src = (2 * ns.nxh - kxi - 1) * ns.nyh;
            kk = nz - k;
            mirror = true;
        }
    }
    const int H = (nz - 1) / 2;
    const int kzi = kk <= H ? kk : kk - nz;  // Kdata.cpp:74-78
    const double c = __dmul_rn((double)kzi, kzL);
    const double kz2 = -__dmul_rn(c, c);
    const double lap2 = __dadd_rn(-__dmul_rn(ky, ky), kz2);  // Kdata.cpp:100-119
    const double kx = __dadd_rn(mirror ? -kx0 : kx0, __dmul_rn(__dmul_rn(q, t), ky));
    const double lapF = __dadd_rn(-__dmul_rn(kx, kx), lap2);  // MHD_FullQlin.cpp:722-731
    if (!(lapF > -ns.hi2 && lapF < -ns.lo2)) return false;
    const double m = (v == 0 || v == 2) ? sqrt(__ddiv_rn(__dmul_rn(ns.multfac, lap2), lapF))
                                        : sqrt(-__dmul_rn(ns.multfac, lap2));
    double z1, z2;
    philox_normal_pair(ns.seed, step, (uint32_t)src, (uint32_t)(4 * kk + v), &z1, &z2);
    const double re = __dmul_rn(m, __dmul_rn(z1, ns.sd));
    const double im = __dmul_rn(m, __dmul_rn(z2, ns.sd));
    out->x = re;
    out->y = mirror ? -im : im;
    return true;
}

// Adds the noise of one mode to its fields u[4][nz] (lanes `lane` of `nlanes`
// take the elements in turn).  Out of line: the callers' pipelines keep their
// registers.
static __device__ __noinline__ void noise_mode(const NoiseSpec* nsp, unsigned long long step, cplx* u, int nz,
                                               int lane, int nlanes, int i, double kx0, double ky, int kxi, int kyi,
                                               double q, double t, double kzL) {
    const NoiseSpec ns = *nsp;
    for (int e = lane; e < 4 * nz; e += nlanes) {
        const int v = e / nz, k = e - v * nz;
        cplx n;
        if (!noise_value(ns, step, i, k, v, nz, kx0, ky, kxi, kyi, q, t, kzL, &n)) continue;
        // the fields were just stored by other lanes: read through L2
        const double2 w = __ldcg(reinterpret_cast<const double2*>(u + e));
        *reinterpret_cast<double2*>(u + e) = make_double2(__dadd_rn(w.x, n.x), __dadd_rn(w.y, n.y));
    }
}

}  // namespace qlgpu
