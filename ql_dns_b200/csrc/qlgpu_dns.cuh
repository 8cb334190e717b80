// qlgpu_dns.cuh -- FP64 kernels of the full 3-D shearing-box MHD DNS (sm_100a).
//
// One right-hand side is four launches over data that stays in L2:
//   A  dns_inv_zx<NZ,MX>  grid (ky, field):   per ky plane, the z inverse of every
//                         column (padded from nz) and the x inverse of every z row
//                         (bins kx0 mod Mx) -> X[f][ky][x][z]
//   B  dns_phys<MY>       grid (x, z chunk):  y inverse of u and b (two real fields per
//                         complex transform, Hermitian in ky), the nine products
//                         T_ij = u_i u_j - b_i b_j and E = u x b in shared memory, and
//                         their y forward transforms -> P[p][ky][x][z]
//   C  dns_fwd_xz<MX,NZ>  grid (ky, product): x forward of every z row, gather of the
//                         plane's columns, z forward and truncation -> T[p][mode][kz]
//   D  dns_update         one thread per (mode, kz): the rhs (projection, shear,
//                         rotation, B0z, the i k.T and i k x E terms), the RK3 update
//                         (RK3CN_Elin exponential or RK3CN Crank-Nicolson), the 2/3
//                         mask in x at the next stage time, the divergence correction
//                         and, at the last stage, the remap zeroing.
// Transforms use the register/shared-memory FFT of qlgpu_fft.cuh (one group of
// T threads per row).  Sign and scale: backward exp(+), forward exp(-), both
// unnormalised; 1/(Mx My NZ) is applied when the state is loaded.
#pragma once
#include <cuda_runtime.h>

#include "qlgpu_debug.cuh"
#include "qlgpu_fft.cuh"

namespace qlgpu {
namespace dns {

constexpr int BLOCK = 256;
constexpr int NPROD = 9;

struct DnsArgs {
    int nxy, nz, ncol, Kyn, nx;  // columns, stored kz, columns per ky, ky count, QL nx
    int Mx, My, NZ;
    int order_half, remap, integ;
    double dkx, q, omega, nu, eta, B0z, scale, kmask, dt;
    double remap_thresh, remap_shift;  // (nx-1)/2 dkx and (nx-1) dkx (MHD_FullQlin.cpp:472-474)
    const double* ky;  // [nxy]
    const double* kz;  // [nz]
    const cplx* twz;
    const cplx* twx;
    const cplx* twy;
    cplx* lin;      // [nxy][6][nz]
    double* kx0;    // [nxy]
    cplx* X;        // [6][Kyn][Mx][NZ]
    cplx* P;        // [9][Kyn][Mx][NZ]
    cplx* T;        // [9][nxy][nz]
    cplx* F[2];     // [nxy][6][nz]
    double* clock;  // [0] = t at the start of the step
    int* status;
};

struct DnsStage {
    double t_off, dt_lin, linC, n1, n2, tn_off;  // stage time t + t_off, next evaluation at t + tn_off
    int cur, prev, has_prev, last, rhs_only;     // F buffers, flags
    double t_abs;                                 // rhs_only: absolute time
};

// Programmatic dependent launch (the step's kernels are launched with it): a
// kernel lets the next one be scheduled as soon as all its CTAs have started, and
// waits for the previous kernel to complete (and its memory to be visible) before
// it touches global memory.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_start() {
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

__device__ __forceinline__ unsigned group_mask(int T) {
    const int lane = threadIdx.x & 31;
    const unsigned m = (T == 32) ? 0xffffffffu : ((1u << T) - 1u);
    return m << (lane / T * T);
}

// kx(t) = kx0 + (q t) ky, rounded as the host restatement does (no contraction)
__device__ __forceinline__ double kx_at(double kx0, double q, double t, double ky) {
    return __dadd_rn(kx0, __dmul_rn(__dmul_rn(q, t), ky));
}

__device__ __forceinline__ int xbin(double kx0, double dkx, int M) {
    long long m = llrint(kx0 / dkx);
    int b = (int)(m % M);
    return b < 0 ? b + M : b;
}

// ---------------------------------------------------------------------------
// A: z inverse + x inverse of one field on one ky plane
// ---------------------------------------------------------------------------
template <int NZ, int MX>
struct InvZX {
    using GZ = Geom<NZ>;
    using GX = Geom<MX>;
    static constexpr int SROW = NZ + 1;  // padded rows (bank spread)
    static constexpr int XZ = (BLOCK / GZ::T) * GZ::XSIZE;
    static constexpr int XX = (BLOCK / GX::T) * GX::XSIZE;
    static constexpr int XCH = XZ > XX ? XZ : XX;
    static size_t smem(int ncol) { return sizeof(cplx) * ((size_t)ncol * SROW + XCH) + sizeof(int) * MX; }
};

template <int NZ, int MX>
__global__ void __launch_bounds__(BLOCK, 2) dns_inv_zx(DnsArgs a) {
    pdl_start();
    using K = InvZX<NZ, MX>;
    using GZ = typename K::GZ;
    using GX = typename K::GX;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx* S = reinterpret_cast<cplx*>(smraw);
    cplx* xch = S + (size_t)a.ncol * K::SROW;
    int* bin2col = reinterpret_cast<int*>(xch + K::XCH);
    const int ky = blockIdx.x, f = blockIdx.y, tid = threadIdx.x;
    for (int b = tid; b < MX; b += BLOCK) bin2col[b] = -1;
    __syncthreads();
    for (int c = tid; c < a.ncol; c += BLOCK) bin2col[QLGPU_CHECK_INDEX(xbin(a.kx0[QLGPU_CHECK_INDEX(ky + a.Kyn * c, a.nxy, a.status)], a.dkx, MX), MX, a.status)] = c;
    __syncthreads();
    {  // z inverse of every column of the plane
        constexpr int T = GZ::T, NG = BLOCK / T;
        const int g = tid / T, t = tid % T;
        const unsigned gm = group_mask(T);
        cplx* xg = xch + g * GZ::XSIZE;
        for (int c = g; c < a.ncol; c += NG) {
            const cplx* src = a.lin + ((size_t)QLGPU_CHECK_INDEX(ky + a.Kyn * c, a.nxy, a.status) * 6 + f) * a.nz;
            cplx x[GZ::P];
#pragma unroll
            for (int k2 = 0; k2 < GZ::P; ++k2) {
                const int s = QLGPU_CHECK_STORED(stored_index<GZ>(t + T * k2), a.nz, a.status);
                x[k2] = s >= 0 ? cscale(src[s], a.scale) : mk(0.0, 0.0);
            }
            inv_fft<GZ>(x, xg, a.twz, t, gm);
#pragma unroll
            for (int j = 0; j < GZ::P; ++j) S[c * K::SROW + zpos<GZ>(t, j)] = x[j];
        }
    }
    __syncthreads();
    {  // x inverse of every z row, stored to X[f][ky][x][z]: the groups of a warp take
       // consecutive z, so each store instruction writes whole 32-byte sectors
        constexpr int T = GX::T, NG = BLOCK / T;
        const int g = tid / T, t = tid % T;
        const unsigned gm = group_mask(T);
        cplx* xg = xch + g * GX::XSIZE;
        cplx* dst = a.X + ((size_t)f * a.Kyn + ky) * MX * NZ;
        for (int z = g; z < NZ; z += NG) {
            cplx x[GX::P];
#pragma unroll
            for (int k2 = 0; k2 < GX::P; ++k2) {
                const int c = bin2col[t + T * k2];
                x[k2] = c >= 0 ? S[c * K::SROW + z] : mk(0.0, 0.0);
            }
            inv_fft<GX>(x, xg, a.twx, t, gm);
#pragma unroll
            for (int j = 0; j < GX::P; ++j) dst[(size_t)zpos<GX>(t, j) * NZ + z] = x[j];
        }
    }
}

// ---------------------------------------------------------------------------
// B: y transforms and the products, per (x, chunk of z lines)
// ---------------------------------------------------------------------------
template <int MY>
struct Phys {
    using GY = Geom<MY>;
    // 192 threads and 8 lines (4 at MY = 256) keep the shared memory near 105 KB, so two
    // CTAs share an SM; the inverse phase (3 transforms per line) is one round of the groups
    static constexpr int THREADS = 192;
    static constexpr int ZC = MY >= 256 ? 4 : 8;
    static constexpr int PY = MY + 1;
    static constexpr int NG = THREADS / GY::T;
    static constexpr int XS = GY::XSIZE > MY ? GY::XSIZE : MY;
    static size_t smem() {
        size_t ph = sizeof(double) * 6 * ZC * PY;
        ph = (ph + 15) / 16 * 16;
        return ph + sizeof(cplx) * (size_t)NG * XS;
    }
};

__device__ __forceinline__ double product(int p, const double* v) {
    // v = ux, uy, uz, bx, by, bz
    switch (p) {
        case 0: return v[0] * v[0] - v[3] * v[3];
        case 1: return v[1] * v[1] - v[4] * v[4];
        case 2: return v[2] * v[2] - v[5] * v[5];
        case 3: return v[0] * v[1] - v[3] * v[4];
        case 4: return v[0] * v[2] - v[3] * v[5];
        case 5: return v[1] * v[2] - v[4] * v[5];
        case 6: return v[1] * v[5] - v[2] * v[4];
        case 7: return v[2] * v[3] - v[0] * v[5];
        case 8: return v[0] * v[4] - v[1] * v[3];
        default: return 0.0;
    }
}

template <int MY>
__global__ void __launch_bounds__(Phys<MY>::THREADS, 2) dns_phys(DnsArgs a) {
    pdl_start();
    using K = Phys<MY>;
    using GY = typename K::GY;
    constexpr int T = GY::T, NG = K::NG, ZC = K::ZC, PY = K::PY;
    extern __shared__ __align__(16) unsigned char smraw[];
    double* Ph = reinterpret_cast<double*>(smraw);
    size_t phb = sizeof(double) * 6 * ZC * PY;
    phb = (phb + 15) / 16 * 16;
    cplx* xch = reinterpret_cast<cplx*>(smraw + phb);
    const int x = blockIdx.x, z0 = blockIdx.y * ZC, tid = threadIdx.x;
    const int g = tid / T, t = tid % T;
    const unsigned gm = group_mask(T);
    cplx* xg = xch + g * K::XS;
    const int Kyn = a.Kyn, MX = a.Mx, NZ = a.NZ;
    // inverse: three complex transforms per line carry (ux,uy), (uz,bx), (by,bz)
    for (int task = g; task < 3 * ZC; task += NG) {
        const int l = task % ZC, pr = task / ZC;
        const int fa = 2 * pr, fb = 2 * pr + 1;
        const size_t zoff = (size_t)x * NZ + z0 + l;
        cplx v[GY::P];
#pragma unroll
        for (int k2 = 0; k2 < GY::P; ++k2) {
            const int k = t + T * k2;
            cplx c = mk(0.0, 0.0);
            if (k < Kyn) {
                cplx A = a.X[((size_t)fa * Kyn + k) * MX * NZ + zoff];
                cplx B = a.X[((size_t)fb * Kyn + k) * MX * NZ + zoff];
                if (k == 0) { A.y = 0.0; B.y = 0.0; }
                c = mk(A.x - B.y, A.y + B.x);
            } else if (k > MY - Kyn) {
                const int kk = MY - k;
                const cplx A = a.X[((size_t)fa * Kyn + kk) * MX * NZ + zoff];
                const cplx B = a.X[((size_t)fb * Kyn + kk) * MX * NZ + zoff];
                c = mk(A.x + B.y, B.x - A.y);
            }
            v[k2] = c;
        }
        inv_fft<GY>(v, xg, a.twy, t, gm);
#pragma unroll
        for (int j = 0; j < GY::P; ++j) {
            const int y = zpos<GY>(t, j);
            Ph[(fa * ZC + l) * PY + y] = v[j].x;
            Ph[(fb * ZC + l) * PY + y] = v[j].y;
        }
    }
    __syncthreads();
    // products and their forward transforms, two per complex transform
    for (int task = g; task < 5 * ZC; task += NG) {
        const int l = task % ZC, pp = task / ZC;
        const int pa = 2 * pp, pb = 2 * pp + 1;
        cplx v[GY::P];
#pragma unroll
        for (int j = 0; j < GY::P; ++j) {
            const int y = zpos<GY>(t, j);
            double f6[6];
#pragma unroll
            for (int f = 0; f < 6; ++f) f6[f] = Ph[(f * ZC + l) * PY + y];
            v[j] = mk(product(pa, f6), pb < NPROD ? product(pb, f6) : 0.0);
        }
        fwd_fft<GY>(v, xg, a.twy, t, gm);
#pragma unroll
        for (int k2 = 0; k2 < GY::P; ++k2) xg[t + T * k2] = v[k2];
        __syncwarp(gm);
        const size_t zoff = (size_t)x * NZ + z0 + l;
        for (int k = t; k < Kyn; k += T) {
            const cplx c = xg[k];
            const cplx cm = xg[(MY - k) & (MY - 1)];
            a.P[((size_t)pa * Kyn + k) * MX * NZ + zoff] = mk(0.5 * (c.x + cm.x), 0.5 * (c.y - cm.y));
            if (pb < NPROD)
                a.P[((size_t)pb * Kyn + k) * MX * NZ + zoff] = mk(0.5 * (c.y + cm.y), -0.5 * (c.x - cm.x));
        }
        __syncwarp(gm);
    }
}

// ---------------------------------------------------------------------------
// C: x forward + z forward of one product on one ky plane
// ---------------------------------------------------------------------------
template <int MX, int NZ>
struct FwdXZ {
    using GZ = Geom<NZ>;
    using GX = Geom<MX>;
    static constexpr int SROW = NZ + 1;
    static constexpr int XZ = (BLOCK / GZ::T) * GZ::XSIZE;
    static constexpr int XX = (BLOCK / GX::T) * GX::XSIZE;
    static constexpr int XCH = XZ > XX ? XZ : XX;
    static size_t smem(int ncol) { return sizeof(cplx) * ((size_t)ncol * SROW + XCH) + sizeof(int) * MX; }
};

template <int MX, int NZ>
__global__ void __launch_bounds__(BLOCK, 2) dns_fwd_xz(DnsArgs a) {
    pdl_start();
    using K = FwdXZ<MX, NZ>;
    using GZ = typename K::GZ;
    using GX = typename K::GX;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx* S = reinterpret_cast<cplx*>(smraw);
    cplx* xch = S + (size_t)a.ncol * K::SROW;
    int* bin2col = reinterpret_cast<int*>(xch + K::XCH);
    const int ky = blockIdx.x, p = blockIdx.y, tid = threadIdx.x;
    for (int b = tid; b < MX; b += BLOCK) bin2col[b] = -1;
    const cplx* src = a.P + ((size_t)p * a.Kyn + ky) * MX * NZ;
    __syncthreads();
    for (int c = tid; c < a.ncol; c += BLOCK) bin2col[QLGPU_CHECK_INDEX(xbin(a.kx0[QLGPU_CHECK_INDEX(ky + a.Kyn * c, a.nxy, a.status)], a.dkx, MX), MX, a.status)] = c;
    __syncthreads();
    {  // x forward of every z row (loads: consecutive z per warp, whole sectors), kept at
       // the plane's column bins
        constexpr int T = GX::T, NG = BLOCK / T;
        const int g = tid / T, t = tid % T;
        const unsigned gm = group_mask(T);
        cplx* xg = xch + g * GX::XSIZE;
        for (int z = g; z < NZ; z += NG) {
            cplx x[GX::P];
#pragma unroll
            for (int j = 0; j < GX::P; ++j) x[j] = src[(size_t)zpos<GX>(t, j) * NZ + z];
            fwd_fft<GX>(x, xg, a.twx, t, gm);
#pragma unroll
            for (int k2 = 0; k2 < GX::P; ++k2) {
                const int c = bin2col[t + T * k2];
                if (c >= 0) S[c * K::SROW + z] = x[k2];
            }
        }
    }
    __syncthreads();
    {  // z forward of every column, truncated to the stored kz
        constexpr int T = GZ::T, NG = BLOCK / T;
        const int g = tid / T, t = tid % T;
        const unsigned gm = group_mask(T);
        cplx* xg = xch + g * GZ::XSIZE;
        for (int c = g; c < a.ncol; c += NG) {
            cplx x[GZ::P];
#pragma unroll
            for (int j = 0; j < GZ::P; ++j) x[j] = S[c * K::SROW + zpos<GZ>(t, j)];
            fwd_fft<GZ>(x, xg, a.twz, t, gm);
            cplx* dst = a.T + ((size_t)p * a.nxy + QLGPU_CHECK_INDEX(ky + a.Kyn * c, a.nxy, a.status)) * a.nz;
#pragma unroll
            for (int k2 = 0; k2 < GZ::P; ++k2) {
                const int s = QLGPU_CHECK_STORED(stored_index<GZ>(t + T * k2), a.nz, a.status);
                if (s >= 0) dst[s] = x[k2];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// D: right-hand side, RK3 update, mask, divergence correction, remap zeroing
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ipow(double x, int n) {
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

// -|k|^(2 order_half) at kx = kx0 + q t ky (+ q dt_lin ky), MHD_FullQlin.cpp:371-376
__device__ __forceinline__ double lap_order(const DnsArgs& a, double kx0, double ky, double kz, double t,
                                            double dt_lin) {
    double kxt = kx_at(kx0, a.q, t, ky);
    kxt = kx_at(kxt, a.q, dt_lin, ky);
    const double kz2 = -__dmul_rn(kz, kz);
    return -ipow(fabs(__dadd_rn(__dsub_rn(-__dmul_rn(kxt, kxt), __dmul_rn(ky, ky)), kz2)), a.order_half);
}

__device__ __forceinline__ cplx cmuli(cplx a) { return mk(-a.y, a.x); }  // i a

__global__ void __launch_bounds__(BLOCK) dns_update(DnsArgs a, DnsStage st) {
    pdl_start();
    const int idx = blockIdx.x * BLOCK + threadIdx.x;
    if (idx >= a.nxy * a.nz) return;
    const int mode = idx / a.nz, s = idx % a.nz;
    const double t0 = st.rhs_only ? st.t_abs : a.clock[0];
    const double ts = st.rhs_only ? st.t_abs : t0 + st.t_off;
    const double kx0 = a.kx0[mode], ky = a.ky[mode], kz = a.kz[s];
    const double Kx = kx_at(kx0, a.q, ts, ky);
    cplx u[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) u[c] = a.lin[((size_t)mode * 6 + c) * a.nz + s];
    cplx Tm[NPROD];
#pragma unroll
    for (int p = 0; p < NPROD; ++p) Tm[p] = a.T[((size_t)p * a.nxy + mode) * a.nz + s];
    const double om = a.omega, q = a.q, B0z = a.B0z;
    // A = -i k.T + (2 Om u_y, (q - 2 Om) u_x, 0) + i kz B0z b
    cplx kT[3];
    kT[0] = mk(Kx * Tm[0].x + ky * Tm[3].x + kz * Tm[4].x, Kx * Tm[0].y + ky * Tm[3].y + kz * Tm[4].y);
    kT[1] = mk(Kx * Tm[3].x + ky * Tm[1].x + kz * Tm[5].x, Kx * Tm[3].y + ky * Tm[1].y + kz * Tm[5].y);
    kT[2] = mk(Kx * Tm[4].x + ky * Tm[5].x + kz * Tm[2].x, Kx * Tm[4].y + ky * Tm[5].y + kz * Tm[2].y);
    cplx A[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const cplx mi = mk(kT[c].y, -kT[c].x);           // -i kT
        const cplx bz = cmuli(cscale(u[3 + c], kz * B0z));  // i kz B0z b
        A[c] = cadd(mi, bz);
    }
    A[0] = cadd(A[0], cscale(u[1], 2 * om));
    A[1] = cadd(A[1], cscale(u[0], q - 2 * om));
    const double K2 = Kx * Kx + ky * ky + kz * kz;
    const double iK2 = K2 > 0 ? 1.0 / K2 : 0.0;
    cplx sdot = cadd(cadd(cscale(A[0], Kx), cscale(A[1], ky)), cadd(cscale(A[2], kz), cscale(u[0], q * ky)));
    sdot = cscale(sdot, iK2);
    cplx F[6];
    F[0] = csub(A[0], cscale(sdot, Kx));
    F[1] = csub(A[1], cscale(sdot, ky));
    F[2] = csub(A[2], cscale(sdot, kz));
    // i k x E + (0, -q b_x, 0) + i kz B0z u
    const cplx Ex = Tm[6], Ey = Tm[7], Ez = Tm[8];
    F[3] = cadd(cmuli(csub(cscale(Ez, ky), cscale(Ey, kz))), cmuli(cscale(u[0], kz * B0z)));
    F[4] = cadd(csub(cmuli(csub(cscale(Ex, kz), cscale(Ez, Kx))), cscale(u[3], q)), cmuli(cscale(u[1], kz * B0z)));
    F[5] = cadd(cmuli(csub(cscale(Ey, Kx), cscale(Ex, ky))), cmuli(cscale(u[2], kz * B0z)));
    const bool keep_s = fabs(Kx) <= a.kmask;
    if (!keep_s) {
#pragma unroll
        for (int c = 0; c < 6; ++c) F[c] = mk(0.0, 0.0);
    }
    cplx* Fc = a.F[st.cur];
#pragma unroll
    for (int c = 0; c < 6; ++c) Fc[((size_t)mode * 6 + c) * a.nz + s] = F[c];
    if (st.rhs_only) return;
    // update (RK3CN_Elin.cpp:102-104 / RK3CN.cpp:105-107), operator at t_s + dt_lin
    // the kx = ky = 0 column (the means) has ordinary diffusion at every order, as the
    // mean-field operator of MHD_FullQlin (linOpMF = coef kz2, MHD_FullQlin.cpp:449-455)
    const bool mean_col = (mode == 0);
    const double kz2m = -__dmul_rn(kz, kz);
    const double Lu = mean_col ? a.nu * kz2m : a.nu * lap_order(a, kx0, ky, kz, ts, st.dt_lin);
    const double Lb = mean_col ? a.eta * kz2m : a.eta * lap_order(a, kx0, ky, kz, ts, st.dt_lin);
    const cplx* Fp = a.F[st.prev];
    cplx nw[6];
    if (a.integ == 0) {
        const double eu = exp(st.linC * Lu), eb = exp(st.linC * Lb);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            cplx acc = cscale(F[c], st.n1);
            if (st.has_prev) acc = cadd(acc, cscale(Fp[((size_t)mode * 6 + c) * a.nz + s], st.n2));
            nw[c] = cscale(cadd(acc, u[c]), c < 3 ? eu : eb);
        }
    } else {
        const double Lou = mean_col ? Lu : a.nu * lap_order(a, kx0, ky, kz, ts, 0.0);
        const double Lob = mean_col ? Lb : a.eta * lap_order(a, kx0, ky, kz, ts, 0.0);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double L = c < 3 ? Lu : Lb, Lo = c < 3 ? Lou : Lob;
            cplx acc = cscale(F[c], st.n1);
            if (st.has_prev) acc = cadd(acc, cscale(Fp[((size_t)mode * 6 + c) * a.nz + s], st.n2));
            acc = cadd(acc, cscale(u[c], 1 + st.linC * Lo));
            nw[c] = cscale(acc, 1.0 / (1.0 - st.linC * L));
        }
    }
    // 2/3 mask in x and divergence correction at the next evaluation time
    const double tn = t0 + st.tn_off;
    const double Kxn = kx_at(kx0, q, tn, ky);
    bool zero = fabs(Kxn) > a.kmask;
    if (st.last && a.remap) zero = zero || (Kxn > a.remap_thresh);
    if (zero) {
#pragma unroll
        for (int c = 0; c < 6; ++c) nw[c] = mk(0.0, 0.0);
    } else {
        const double kp2 = ky * ky + kz * kz;
        const double ikp = kp2 > 0 ? 1.0 / kp2 : 0.0;
#pragma unroll
        for (int b = 0; b < 6; b += 3) {
            const cplx D = cadd(cadd(cscale(nw[b], Kxn), cscale(nw[b + 1], ky)), cscale(nw[b + 2], kz));
            if (kp2 > 0) {
                nw[b + 1] = csub(nw[b + 1], cscale(cscale(D, ky), ikp));
                nw[b + 2] = csub(nw[b + 2], cscale(cscale(D, kz), ikp));
            } else if (Kxn != 0.0) {
                nw[b] = mk(0.0, 0.0);
            } else {
                nw[b + 2] = mk(0.0, 0.0);
            }
        }
    }
    bool bad = false;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        bad = bad || !isfinite(nw[c].x) || !isfinite(nw[c].y);
        a.lin[((size_t)mode * 6 + c) * a.nz + s] = nw[c];
    }
    if (bad) atomicOr(a.status, 1);
}

// After the last stage: shift kx0 of the columns that left the box (their
// fields were zeroed by dns_update), MHD_FullQlin.cpp:464-481.
__global__ void dns_remap_kx(DnsArgs a) {
    pdl_start();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nxy || !a.remap) return;
    const double tn = a.clock[0] + a.dt;
    const double kxt = kx_at(a.kx0[i], a.q, tn, a.ky[i]);
    if (kxt > a.remap_thresh) a.kx0[i] = __dsub_rn(a.kx0[i], a.remap_shift);
}

__global__ void dns_advance_clock(DnsArgs a) {
    pdl_start();
    if (threadIdx.x == 0 && blockIdx.x == 0) a.clock[0] = a.clock[0] + a.dt;
}

// ---------------------------------------------------------------------------
// Diagnostics: one warp per column, then one block in fixed order
// ---------------------------------------------------------------------------
__global__ void dns_diag_modes(DnsArgs a, double* part) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= a.nxy) return;
    const double t = a.clock[0];
    const double Kx = kx_at(a.kx0[w], a.q, t, a.ky[w]), ky = a.ky[w];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int s = lane; s < a.nz; s += 32) {
        const cplx* c = a.lin + (size_t)w * 6 * a.nz + s;
        const cplx ux = c[0], uy = c[a.nz], uz = c[2 * a.nz];
        const cplx bx = c[3 * a.nz], by = c[4 * a.nz], bz = c[5 * a.nz];
        const double kz = a.kz[s];
        if (w == 0) {  // means: energy, stress, dissipation of (Ux, Uy) and (Bx, By)
            const double eu = ux.x * ux.x + ux.y * ux.y + uy.x * uy.x + uy.y * uy.y;
            const double eb = bx.x * bx.x + bx.y * bx.y + by.x * by.x + by.y * by.y;
            acc[0] += eu;
            acc[1] += eb;
            acc[2] += ux.x * uy.x + ux.y * uy.y;
            acc[3] += bx.x * by.x + bx.y * by.y;
            acc[4] += kz * kz * eu;
            acc[5] += kz * kz * eb;
        } else {
            const double eu = ux.x * ux.x + ux.y * ux.y + uy.x * uy.x + uy.y * uy.y + uz.x * uz.x + uz.y * uz.y;
            const double eb = bx.x * bx.x + bx.y * bx.y + by.x * by.x + by.y * by.y + bz.x * bz.x + bz.y * bz.y;
            const double K2 = Kx * Kx + ky * ky + kz * kz;
            acc[0] += eu;
            acc[1] += eb;
            acc[2] += ux.x * uy.x + ux.y * uy.y;
            acc[3] += bx.x * by.x + bx.y * by.y;
            acc[4] += K2 * eu;
            acc[5] += K2 * eb;
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if (lane == 0) {
        const double wgt = (w != 0 && ky != 0.0) ? 2.0 : 1.0;  // conjugate column counted
#pragma unroll
        for (int k = 0; k < 6; ++k) part[(size_t)w * 6 + k] = acc[k] * wgt;
    }
}

__global__ void __launch_bounds__(256) dns_diag_final(DnsArgs a, const double* part, double divf, double kzmax,
                                                      double* out) {
    __shared__ double sh[256][6];
    const int tid = threadIdx.x;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int m = 1 + tid; m < a.nxy; m += 256)
        for (int k = 0; k < 6; ++k) acc[k] += part[(size_t)m * 6 + k];
    for (int k = 0; k < 6; ++k) sh[tid][k] = acc[k];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (tid < o)
            for (int k = 0; k < 6; ++k) sh[tid][k] += sh[tid + o][k];
        __syncthreads();
    }
    if (tid == 0) {
        const double Eu = sh[0][0] * divf, Eb = sh[0][1] * divf;
        const double AMu = sh[0][2] * divf, AMb = sh[0][3] * divf;
        const double Du = a.nu * sh[0][4] * divf, Db = a.eta * sh[0][5] * divf;
        const double eMU = part[0] * divf, eMB = part[1] * divf, aMU = part[2] * divf, aMB = part[3] * divf;
        const double dMU = a.nu * part[4] * divf, dMB = a.eta * part[5] * divf;
        out[0] = a.clock[0];
        out[1] = eMU / 2; out[2] = eMB / 2; out[3] = Eu / 2; out[4] = Eb / 2;
        out[5] = aMU; out[6] = aMB; out[7] = AMu; out[8] = AMb;
        out[9] = dMU; out[10] = dMB; out[11] = Du; out[12] = Db;
        out[13] = pow(a.nu * a.nu * a.nu / (dMU + Du), 0.25) * kzmax;
        out[14] = pow(a.eta * a.eta * a.eta / (dMB + Db), 0.25) * kzmax;
    }
}

}  // namespace dns
}  // namespace qlgpu
