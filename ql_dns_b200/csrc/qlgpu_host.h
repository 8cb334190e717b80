// qlgpu_host.h -- host-side set-up shared by the single-case handle (qlgpu.cu)
// and the batch (qlgpu_batch_host.cu): parameter checks, the run constants of
// a case, the wavenumber / twiddle / 1/lap2 / integrating-factor tables, and
// the tables of compiled kernels.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/qlgpu.h"
#include "qlgpu_types.h"

namespace qlgpu {

struct cplx;

constexpr double kPI = 3.14159265358979323846;  // General_Definitions.h PI

// RK3 coefficients (RK3CN_Elin.cpp:19-20, RK3CN.cpp:19-20)
constexpr double a0_ = 8.0 / 15.0, a1_ = 5.0 / 12.0, a2_ = 3.0 / 4.0, b1_ = -17.0 / 60.0, b2_ = -5.0 / 12.0;
constexpr double p1_ = 8.0 / 15.0, p2_ = 2.0 / 3.0;

typedef void (*stage_launch_fn)(const StageArgs&, const DevParams&, int grid, int block, size_t smem, cudaStream_t);
typedef void (*diag_launch_fn)(const cplx*, const cplx*, const double*, const double*, const int*, const int*,
                               const DevParams&, double, double*, cudaStream_t);
typedef size_t (*smem_fn)(int warps);
typedef int (*tmem_fn)(int warps);
typedef const void* (*kptr_fn)();

// One compiled stage kernel (NZ x model x integrator x private-store backing).
struct Variant {
    stage_launch_fn launch;
    kptr_fn kernel;
    smem_fn smem;
    tmem_fn tmem;
    diag_launch_fn diag;
    int T;          // threads per transform group
    int PL;         // partial vector length (doubles)
    int max_warps;  // widest CTA the kernel is compiled for
};

// Defined in qlgpu_nz<NZ>.cu, one translation unit per NZ.
bool make_variant_nz16(int model, int integ, bool tm, Variant* out);
bool make_variant_nz32(int model, int integ, bool tm, Variant* out);
bool make_variant_nz64(int model, int integ, bool tm, Variant* out);
bool make_variant_nz128(int model, int integ, bool tm, Variant* out);
bool make_variant_nz256(int model, int integ, bool tm, Variant* out);

inline bool pick_variant(int NZ, int model, int integ, bool tm, Variant* out) {
    switch (NZ) {
        case 16: return make_variant_nz16(model, integ, tm, out);
        case 32: return make_variant_nz32(model, integ, tm, out);
        case 64: return make_variant_nz64(model, integ, tm, out);
        case 128: return make_variant_nz128(model, integ, tm, out);
        case 256: return make_variant_nz256(model, integ, tm, out);
        default: return false;
    }
}

// The persistent batch kernel of one model x integrator (qlgpu_batch_<model>_<integ>.cu),
// in two builds: NZ <= 64 only (128 registers, two 8-warp CTAs per SM) and all NZ.
struct BatchKernel {
    cudaError_t (*launch)(const BatchLaunch& L, int grid, int block, size_t smem, cudaStream_t st);
    const void* (*kernel)();
    size_t (*smem)(int NZ, int warps);  // dynamic shared memory of one NZ class
    int (*tmem)(int NZ, int warps);     // TMEM columns of one NZ class
    int max_nz;                         // largest NZ class the build steps
    int max_warps;                      // widest CTA the build is compiled for
};
bool batch_kernel_bq_exp(bool wide, BatchKernel* out);
bool batch_kernel_bq_cn(bool wide, BatchKernel* out);
bool batch_kernel_fq_exp(bool wide, BatchKernel* out);
bool batch_kernel_fq_cn(bool wide, BatchKernel* out);

inline bool pick_batch_kernel(int model, int integ, bool wide, BatchKernel* out) {
    if (model == MODEL_BQLIN)
        return integ == INTEG_EXP ? batch_kernel_bq_exp(wide, out) : batch_kernel_bq_cn(wide, out);
    return integ == INTEG_EXP ? batch_kernel_fq_exp(wide, out) : batch_kernel_fq_cn(wide, out);
}

// The dynamic shared memory limit is an attribute of the kernel function, shared
// by every handle, batch and no-allocation call of the process on a device: it
// is only ever raised, so a launch prepared by one of them is never invalidated
// by another that needs less.
inline cudaError_t ensure_smem_attr(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> set;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = set[std::make_pair(dev, kernel)];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// Threads per transform group for a supported NZ (qlgpu_fft.cuh Geom), 0 if unsupported.
inline int group_threads(int NZ) {
    switch (NZ) {
        case 16: return 4;
        case 32: return 4;
        case 64: return 8;
        case 128: return 8;
        case 256: return 16;
        default: return 0;
    }
}

inline int stored_nz(int NZ) { return 1 + 2 * int(NZ / 3.0); }                   // Model.h:34
inline int mode_count(const qlgpu_params& p) { return (p.nx - 1) * (p.ny / 2); }  // Model.h:36
inline int mean_field_count(const qlgpu_params& p) { return p.model == QLGPU_MODEL_MHD_BQLIN ? 2 : 4; }

// Parameter checks of qlgpu_create; returns QLGPU_OK or an error code with *msg set.
inline int check_params(const qlgpu_params& p, std::string* msg) {
    if (p.model != QLGPU_MODEL_MHD_BQLIN && p.model != QLGPU_MODEL_MHD_FULLQLIN) {
        *msg = "unknown model (no matching model found, main.cpp:71-74)";
        return QLGPU_ERR_ARG;
    }
    if (p.integrator != QLGPU_INTEG_RK3CN_ELIN && p.integrator != QLGPU_INTEG_RK3CN) {
        *msg = "unknown integrator";
        return QLGPU_ERR_ARG;
    }
    if (p.nx < 2 || (p.nx % 2) || p.ny < 2 || (p.ny % 2)) {
        *msg = "nx and ny must be even and >= 2";
        return QLGPU_ERR_ARG;
    }
    if (!(p.dt > 0)) {
        *msg = "dt must be > 0 (variable CFL time step not supported)";
        return QLGPU_ERR_UNSUPPORTED;
    }
    if (!(p.L[0] > 0 && p.L[1] > 0 && p.L[2] > 0)) {
        *msg = "box lengths must be > 0";
        return QLGPU_ERR_ARG;
    }
    if (p.model == QLGPU_MODEL_MHD_BQLIN && p.nu == 0.0) {
        *msg = "MHD_BQlin divides by nu (MHD_BQlin.cpp:251); nu must be nonzero";
        return QLGPU_ERR_ARG;
    }
    if (group_threads(p.NZ) == 0) {
        *msg = "unsupported NZ: must be a power of two in [16, 256]";
        return QLGPU_ERR_UNSUPPORTED;
    }
    return QLGPU_OK;
}

// Run constants of a case (MHD_BQlin.cpp:18-60, MHD_FullQlin.cpp:14-60).
inline DevParams make_devparams(const qlgpu_params& p) {
    DevParams d;
    std::memset(&d, 0, sizeof(d));
    d.nxy = mode_count(p);
    d.nz = stored_nz(p.NZ);
    d.NZ = p.NZ;
    d.nmf = mean_field_count(p);
    d.q = p.q;
    d.Omega = p.model == QLGPU_MODEL_MHD_BQLIN ? 2.0 / 3.0 * p.q : p.omega;
    d.nu = p.nu;
    d.eta = p.eta;
    d.etanu = p.model == QLGPU_MODEL_MHD_BQLIN ? p.eta / p.nu : p.eta;
    d.cb = p.model == QLGPU_MODEL_MHD_BQLIN ? (p.eta / p.nu) * p.nu : p.eta;
    // -|(-kx^2-ky^2)+kz2|^(order/2) is linear in kz2 only for order/2 == 1 (MHD_FullQlin.cpp:372)
    d.factored = (p.model == QLGPU_MODEL_MHD_BQLIN || p.viscosity_order / 2 == 1) ? 1 : 0;
    d.B0z = p.B0z;
    d.visc_half = p.viscosity_order / 2;
    d.ql = p.quasilinear ? 1 : 0;
    d.remap = p.remap ? 1 : 0;
    d.kzL = 2 * kPI / p.L[2];
    d.fac = 1.0 / p.NZ;
    const int Nx = p.nx, Ny = (p.ny / 2) * 2;
    d.rs_fac = 1.0 / (Ny * Nx) / (Ny * Nx);
    long totalN2 = (long)Nx * Ny * p.NZ;
    totalN2 = totalN2 * totalN2;
    d.divfac = p.L[2] / (double)totalN2;
    d.divMF = p.L[2] / ((double)p.NZ * p.NZ);
    const double kxLfac = 2 * kPI / p.L[0];
    const int nxm1 = Nx - 1;
    d.remap_thresh = nxm1 / 2.0 * kxLfac;
    d.remap_shift = nxm1 * kxLfac;
    d.dt = p.dt;
    d.tv_interval = 0.0;
    d.kzmax = 2 * kPI / p.L[2] * (p.NZ / 3);
    return d;
}

// Kdata tables (QL_DNS/Auxiliary/Kdata.cpp:24-46)
inline void ktables(const qlgpu_params& p, std::vector<double>& kx, std::vector<double>& ky, std::vector<int>& kxi,
                    std::vector<int>& kyi) {
    const double kxL = 2 * kPI / p.L[0], kyL = 2 * kPI / p.L[1];
    const int ny = ((p.ny / 2) * 2) / 2, nx = p.nx / 2;
    const int nxy = (p.nx - 1) * (p.ny / 2);
    kx.assign(nxy, 0.0);
    ky.assign(nxy, 0.0);
    kxi.assign(nxy, 0);
    kyi.assign(nxy, 0);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            kx[j + ny * i] = i * kxL;
            ky[j + ny * i] = j * kyL;
            kxi[j + ny * i] = i;
            kyi[j + ny * i] = j;
        }
    for (int i = nx + 1; i < 2 * nx; ++i)
        for (int j = 0; j < ny; ++j) {
            kx[j + ny * (i - 1)] = (-2 * nx + i) * kxL;
            ky[j + ny * (i - 1)] = j * kyL;
            kxi[j + ny * (i - 1)] = -2 * nx + i;
            kyi[j + ny * (i - 1)] = j;
        }
}

// Twiddles of the transform layout: tw[n2*T + t] = exp(+2 pi i n2 t / NZ), as (re, im) pairs.
inline std::vector<double> twiddles(int NZ, int T) {
    std::vector<double> tw(2 * (size_t)NZ);
    const int P = NZ / T;
    for (int n2 = 0; n2 < P; ++n2)
        for (int t = 0; t < T; ++t) {
            const int m = (n2 * t) % NZ;
            const double ang = 2.0 * kPI * (double)m / (double)NZ;
            tw[2 * (n2 * T + t)] = std::cos(ang);
            tw[2 * (n2 * T + t) + 1] = std::sin(ang);
        }
    return tw;
}

// 1/lap2 per (ky index, stored kz), Kdata.cpp:100-119
inline std::vector<double> ilap2_table(const qlgpu_params& p, int nz) {
    std::vector<double> il2((size_t)(p.ny / 2) * nz, 0.0);
    const double kyL = 2 * kPI / p.L[1], kzL = 2 * kPI / p.L[2];
    const int nzl = (nz - 1) / 2;
    for (int j = 0; j < p.ny / 2; ++j) {
        const double kyr = j * kyL;
        for (int s = 0; s < nz; ++s) {
            const int kzi = s <= nzl ? s : (-2 * nzl + s - 1);
            const double c = kzi * kzL;
            const double kz2 = 0.0 * 0.0 - c * c;
            double l2 = -kyr * kyr + kz2;
            double v = 1 / l2;
            if (kyr == 0 && s == 0) v = 1;
            il2[(size_t)j * nz + s] = v;
        }
    }
    return il2;
}

// exp(linC nu kz2), exp(linC cb kz2) per stage, [3][2][nz] (RK3CN_Elin.cpp:89,122,155)
inline std::vector<double> ekz_table(const qlgpu_params& p, const DevParams& d) {
    const int nz = d.nz;
    const double dt = p.dt;
    const double linC[3] = {dt * (a0_), dt * (a1_ + b1_), dt * (a2_ + b2_)};
    const double kzL = 2 * kPI / p.L[2];
    const int nzl = (nz - 1) / 2;
    std::vector<double> e((size_t)6 * nz, 1.0);
    for (int st = 0; st < 3; ++st)
        for (int s = 0; s < nz; ++s) {
            const int kzi = s <= nzl ? s : s - nz;
            const double c = kzi * kzL;
            const double kz2 = -(c * c);
            e[(size_t)(st * 2) * nz + s] = std::exp(linC[st] * d.nu * kz2);
            e[(size_t)(st * 2 + 1) * nz + s] = std::exp(linC[st] * d.cb * kz2);
        }
    return e;
}

// Noise constants of a case stepping with dt (MHD_FullQlin.cpp:45-66,804;
// MHD_BQlin.cpp:23-36,563): ky = 0 pairs are driven by MHD_FullQlin only.
inline NoiseSpec noise_spec(const qlgpu_params& p, int NZ, double dt, double f_noise, double k_low, double k_high,
                            unsigned long long seed, int only_velocity, int only_magnetic) {
    NoiseSpec n;
    std::memset(&n, 0, sizeof(n));
    const int Ny = (p.ny / 2) * 2;
    const double tot = (double)p.nx * (double)Ny * (double)NZ;
    const double mult_noise_fac = (1.0 / (16 * 32 * 32)) * (1.0 / (16 * 32 * 32));
    n.lo2 = k_low * k_low;
    n.hi2 = k_high * k_high;
    n.multfac = dt * (tot * tot) * mult_noise_fac;
    n.sd = f_noise / std::sqrt(2.0);
    n.seed = seed;
    n.pair_ky0 = p.model == QLGPU_MODEL_MHD_FULLQLIN;
    n.drive_u = !only_magnetic;
    n.drive_b = !only_velocity;
    n.nxh = p.nx / 2;
    n.nyh = Ny / 2;
    return n;
}

// Stage constants of RK3CN_Elin::Step / RK3CN::Step for stage s of a step
// (RK3CN_Elin.cpp:89-91,122-125,155-158; RK3CN.cpp:92-94).
inline StageConst stage_const(const qlgpu_params& p, int s) {
    const double dt = p.dt;
    const bool cn = p.integrator == QLGPU_INTEG_RK3CN;
    const double lcf = cn ? dt / 2 : dt;
    StageConst c;
    std::memset(&c, 0, sizeof(c));
    if (s == 0) {
        c.t_off = 0.0;
        c.dt_lin = dt * p1_;
        c.linC = lcf * a0_;
        c.n1 = a0_ * dt;
        c.n2 = 0.0;
        c.has_prev = 0;
    } else if (s == 1) {
        c.t_off = dt * p1_;
        c.dt_lin = dt * (p2_ - p1_);
        c.linC = lcf * (a1_ + b1_);
        c.n1 = a1_ * dt;
        c.n2 = b1_ * dt;
        c.has_prev = 1;
    } else {
        c.t_off = dt * p2_;
        c.dt_lin = dt * (1.0 - p2_);
        c.linC = lcf * (a2_ + b2_);
        c.n1 = a2_ * dt;
        c.n2 = b2_ * dt;
        c.has_prev = 1;
    }
    c.last = (s == 2);
    return c;
}

}  // namespace qlgpu
