// qlgpu_stage.cuh -- one fused RK3 stage of the quasi-linear shearing-box step
// on sm_100a.
//
// One launch = one stage of RK3CN_Elin::Step (QL_DNS/Integrators/
// RK3CN_Elin.cpp:86-177) or RK3CN::Step (QL_DNS/Integrators/RK3CN.cpp:86-180)
// for every (kx,ky) mode, fused with the model right-hand side
// (MHD_BQlin::rhs, QL_DNS/Models/MHD_BQlin.cpp:117-284; MHD_FullQlin::rhs,
// QL_DNS/Models/MHD_FullQlin.cpp:171-427), the diagonal diffusion factor, the
// EMF / stress sum over modes that replaces the MPI_Allreduce
// (QL_DNS/Auxiliary/MPIdata.cpp:148-157), the mean-field update, and on the
// last stage the shearing-wave remap (MHD_BQlin.cpp:314-331) and the
// energy / stress / dissipation diagnostics (MHD_BQlin.cpp:337-488).
//
// Work split: a group of T threads owns one mode at a time (qlgpu_fft.cuh).
// Per-CTA partial sums go through a fixed-order two-level reduction; the CTA
// that arrives last at the top performs the mean-field stage.  Everything is
// FP64.
#pragma once
#include "qlgpu_fft.cuh"
#include "qlgpu_types.h"

namespace qlgpu {

// ---------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ cplx ldc(const cplx* p) {
    double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return mk(v.x, v.y);
}
__device__ __forceinline__ cplx ldc_cg(const cplx* p) {
    double2 v = __ldcg(reinterpret_cast<const double2*>(p));
    return mk(v.x, v.y);
}
__device__ __forceinline__ void stc(cplx* p, cplx v) {
    *reinterpret_cast<double2*>(p) = make_double2(v.x, v.y);
}
// i*s*a for real s
__device__ __forceinline__ cplx imul(cplx a, double s) { return mk(-a.y * s, a.x * s); }

// kx(t) = kx0 + (q t) ky, evaluated with the reference's rounding order
// (MHD_BQlin.cpp:498: K->kx[i] + q_*t*kyctmp_)
__device__ __forceinline__ double kx_at(double kx0, double q, double t, double ky) {
    return __dadd_rn(kx0, __dmul_rn(__dmul_rn(q, t), ky));
}

// kz integer -> double wavenumber (Kdata.cpp:76-78: i*kzLfac)
__device__ __forceinline__ double kzval(int kzi, double kzL) { return __dmul_rn((double)kzi, kzL); }
// kz2 = (kz*kz).real() = -(c*c)  (Kdata.cpp:80)
__device__ __forceinline__ double kz2val(double c) { return -__dmul_rn(c, c); }
// lap2 = -ky*ky + kz2 with the ky=kz=0 fix (Kdata.cpp:105-113)
__device__ __forceinline__ double lap2val(double ky, double kz2, bool ky0kz0) {
    return ky0kz0 ? 0.0 : __dadd_rn(-__dmul_rn(ky, ky), kz2);
}
__device__ __forceinline__ double ilap2val(double lap2, bool ky0kz0) {
    return ky0kz0 ? 1.0 : __drcp_rn(lap2);
}

// Laplacian factor of the fluctuation linear operator at the stage end
// (MHD_BQlin.cpp:248-249: (-kx^2 - ky^2) + kz2; MHD_FullQlin.cpp:371-372:
// -|(-kx^2 - ky^2) + kz2|^(order/2)).  kxe = kx(t_s) + q dt_lin ky.
template <int MODEL>
__device__ __forceinline__ double lap_end(const DevParams& P, double kxe, double ky, double kz2) {
    double lap = __dadd_rn(__dsub_rn(-__dmul_rn(kxe, kxe), __dmul_rn(ky, ky)), kz2);
    if (MODEL == MODEL_BQLIN) return lap;
    double a = fabs(lap), r = 1.0;
    for (int i = 0; i < P.visc_half; ++i) r = __dmul_rn(r, a);
    return -r;
}
// linearOPs_Init form (MHD_BQlin.cpp:291, MHD_FullQlin.cpp:435): -kx^2 + lap2
template <int MODEL>
__device__ __forceinline__ double lap_init(const DevParams& P, double kx, double lap2) {
    double lapF = __dadd_rn(-__dmul_rn(kx, kx), lap2);
    if (MODEL == MODEL_BQLIN) return lapF;
    double a = fabs(lapF), r = 1.0;
    for (int i = 0; i < P.visc_half; ++i) r = __dmul_rn(r, a);
    return -r;
}
// L for field f (0 u, 1 zeta, 2 b, 3 eta) from the laplacian factor:
// BQlin L_u = nu lap, L_b = (eta/nu) L_u (MHD_BQlin.cpp:249-252);
// FullQlin L_u = nu lap, L_b = eta lap (MHD_FullQlin.cpp:373-376).
template <int MODEL>
__device__ __forceinline__ double linop_f(const DevParams& P, double lap, int f) {
    const double Lu = __dmul_rn(P.nu, lap);
    if (f < 2) return Lu;
    return MODEL == MODEL_BQLIN ? __dmul_rn(P.etanu, Lu) : __dmul_rn(P.eta, lap);
}

// RK update of one coefficient.  Elin: exp(linC L)(n1 F + n2 Fp + u)
// (RK3CN_Elin.cpp:102-104).  CN: n1 d F + n2 d Fp + (1 + linC Lold) d u,
// d = 1/(1 - linC L) (RK3CN.cpp:105-107).
template <int INTEG>
__device__ __forceinline__ cplx rk_update(const StageConst& S, double L, double Lold, cplx F, cplx Fp, cplx u,
                                          bool has_prev) {
    if (INTEG == INTEG_EXP) {
        double e = exp(__dmul_rn(S.linC, L));
        cplx acc = has_prev ? cadd(cadd(cscale(F, S.n1), cscale(Fp, S.n2)), u) : cadd(cscale(F, S.n1), u);
        return cscale(acc, e);
    } else {
        double d = __drcp_rn(__dsub_rn(1.0, __dmul_rn(S.linC, L)));
        double c1 = __dmul_rn(S.n1, d);
        double c3 = __dmul_rn(__dadd_rn(1.0, __dmul_rn(S.linC, Lold)), d);
        cplx r = cscale(F, c1);
        if (has_prev) r = cadd(r, cscale(Fp, __dmul_rn(S.n2, d)));
        return cadd(r, cscale(u, c3));
    }
}

// CN: where the previous stage's operator was evaluated (RK3CN.cpp:119-122)
struct CnOld {
    double t_old, dtlin_old;
    int old_init;
};

// ---------------------------------------------------------------------------
// Shared-memory carve-up
// ---------------------------------------------------------------------------
template <class G, int MODEL>
struct Smem {
    static constexpr int SW = 32 / G::T;          // groups per warp
    static constexpr int NMFR = MODEL == MODEL_BQLIN ? 3 : 8;  // real-space mean-field profiles
    static constexpr int NPRIV = MODEL == MODEL_BQLIN ? 4 : 6; // private per-thread buffers (P cplx)
    static constexpr int NEMF = MODEL == MODEL_BQLIN ? 2 : 4;  // stress profiles summed over modes
    static constexpr int PL = NEMF * G::NZ + 8;   // partial vector length (doubles)
    static size_t bytes(int warps) {
        size_t b = 0;
        b += sizeof(cplx) * G::NZ;                       // twiddles
        b += sizeof(double) * NMFR * G::NZ;              // mean-field profiles
        b += sizeof(double) * 2 * NEMF * (G::H + 1);     // top-CTA spectra scratch
        b += sizeof(cplx) * (size_t)warps * SW * G::XSIZE;     // exchange
        b += sizeof(cplx) * (size_t)warps * NPRIV * G::P * 32; // private buffers
        return b;
    }
};

// ---------------------------------------------------------------------------
// Per-mode work for MHD_BQlin (MHD_BQlin.cpp:135-257) fused with the update.
// Real-space fields R_f = inv(f / NZ); the products follow MHD_BQlin.cpp:153-201
// with the scalar wavenumbers pulled out of the transforms.
// ---------------------------------------------------------------------------
template <class G, int INTEG>
__device__ __forceinline__ void bqlin_mode(const StageArgs& A, const DevParams& P, int mode, int t, unsigned gmask,
                                           cplx* xch, cplx* priv, int lane, const cplx* tw, const double* mfr,
                                           double* emfx, double* emfy, double tclock, const CnOld& cn) {
    constexpr int Pn = G::P;
    const StageConst& S = A.sc;
    const double fac = P.fac;
    const double ky = __ldg(A.ky + mode);
    const double kx0 = A.kx0[mode];
    const int kyi = __ldg(A.kyi + mode), kxi = __ldg(A.kxi + mode);
    const double ts = S.abs_time ? S.t_off : __dadd_rn(tclock, S.t_off);
    const double a = kx_at(kx0, P.q, ts, ky);         // kx(t_s)
    const double b = ky;
    const double ab = __dmul_rn(a, b);
    const double Om2 = __dmul_rn(2.0, P.Omega);
    const double mult = (ky == 0.0) ? 1.0 : 2.0;
    const cplx* u_in = A.lin_in + (size_t)mode * 4 * P.nz;
    cplx* u_out = A.lin_out + (size_t)mode * 4 * P.nz;
    const cplx* Fp = A.Fprev ? A.Fprev + (size_t)mode * 4 * P.nz : nullptr;
    cplx* Fo = A.Fout ? A.Fout + (size_t)mode * 4 * P.nz : nullptr;
    const double* By = mfr;
    const double* dBy = mfr + G::NZ;
    const double* ddBy = mfr + 2 * G::NZ;
    cplx* K1 = priv;                    // R_bz
    cplx* K2 = priv + 1 * Pn * 32;      // R_uz
    cplx* A1 = priv + 2 * Pn * 32;      // accumulator for G_eta then G_zeta
    cplx* A2 = priv + 3 * Pn * 32;      // spectral fwd(i ky By R_b) for F_u
#define PRIV(buf, j) buf[(j) * 32 + lane]
    cplx x[Pn];

    // Stage-end linear operators and update, per spectral register k2
    const double kxe = __dadd_rn(a, __dmul_rn(__dmul_rn(P.q, S.dt_lin), ky));  // MHD_BQlin.cpp:248
    double kxo = 0.0;  // CN: kx of the previous stage end (or t0 for the init form)
    if (INTEG == INTEG_CN) {
        if (cn.old_init) kxo = kx_at(kx0, P.q, tclock, ky);
        else kxo = __dadd_rn(kx_at(kx0, P.q, cn.t_old, ky), __dmul_rn(__dmul_rn(P.q, cn.dtlin_old), ky));
    }

    // Load a derived spectral field into x (scaled by 1/NZ), zero in the padding gap.
    // which: 0 u,1 zeta,2 b,3 eta, 4 uz, 5 bz, 6 i kz uz, 7 uy, 8 by
    auto load = [&](int which) {
#pragma unroll
        for (int k2 = 0; k2 < Pn; ++k2) {
            const int k = t + G::T * k2;
            const int s = stored_index<G>(k);
            cplx v = mk(0.0, 0.0);
            if (s >= 0) {
                if (which < 4) {
                    v = ldc(u_in + which * P.nz + s);
                } else {
                    const bool mag = (which == 5 || which == 8);
                    cplx f0 = ldc(u_in + (mag ? 2 : 0) * P.nz + s);
                    cplx f1 = ldc(u_in + (mag ? 3 : 1) * P.nz + s);
                    const double c = kzval(kz_int<G>(k), P.kzL);
                    const bool z0 = (kyi == 0 && s == 0);
                    const double il2 = ilap2val(lap2val(ky, kz2val(c), z0), z0);
                    if (which == 7 || which == 8) {
                        // uy = ((-ky kx) f0 + kz f1) ilap2 = (ab f0 + i c f1) ilap2   (MHD_BQlin.cpp:143)
                        v = cscale(cadd(cscale(f0, ab), imul(f1, c)), il2);
                    } else {
                        // uz = (-kx kz f0 - ky f1) ilap2 = (a c f0 - i b f1) ilap2   (MHD_BQlin.cpp:144)
                        v = cscale(csub(cscale(f0, __dmul_rn(a, c)), imul(f1, b)), il2);
                        if (which == 6) v = imul(v, c);
                    }
                }
            }
            x[k2] = cscale(v, fac);
        }
    };

    // Finish one field: x holds fwd(G) in spectral layout; F = x + lin(k); update and store.
    // f: field index; lin: lambda giving the linear rhs contribution at (k2, s, c)
    auto finish = [&](int f, auto&& lin) {
#pragma unroll
        for (int k2 = 0; k2 < Pn; ++k2) {
            const int k = t + G::T * k2;
            const int s = stored_index<G>(k);
            if (s < 0) continue;
            const double c = kzval(kz_int<G>(k), P.kzL);
            const double kz2 = kz2val(c);
            cplx F = lin(k2, s, c, x[k2]);
            cplx uin = ldc(u_in + f * P.nz + s);
            cplx fp = (Fp && S.has_prev) ? ldc(Fp + f * P.nz + s) : mk(0.0, 0.0);
            double L = linop_f<MODEL_BQLIN>(P, lap_end<MODEL_BQLIN>(P, kxe, ky, kz2), f);
            double Lo = 0.0;
            if (INTEG == INTEG_CN) {
                const bool z0 = (kyi == 0 && s == 0);
                const double lo = cn.old_init ? lap_init<MODEL_BQLIN>(P, kxo, lap2val(ky, kz2, z0))
                                             : lap_end<MODEL_BQLIN>(P, kxo, ky, kz2);
                Lo = linop_f<MODEL_BQLIN>(P, lo, f);
            }
            if (A.rhs_only) {
                stc(u_out + f * P.nz + s, F);
                if (A.linop_out) A.linop_out[((size_t)mode * 4 + f) * P.nz + s] = L;
            } else {
                if (Fo) stc(Fo + f * P.nz + s, F);
                stc(u_out + f * P.nz + s, rk_update<INTEG>(S, L, Lo, F, fp, uin, S.has_prev));
            }
        }
    };

    // 1. R_bz -> K1
    load(5);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) PRIV(K1, j) = x[j];
    // 2. R_uz -> K2
    load(4);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) PRIV(K2, j) = x[j];
    // 3. R_u: EMF_x += Re(bz conj u); A1 = -i a dzBy R_u; G_b = i b By R_u -> F_b
    load(0);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) {
        const int z = zpos<G>(t, j);
        cplx k1 = PRIV(K1, j);
        emfx[j] += mult * (k1.x * x[j].x + k1.y * x[j].y);
        PRIV(A1, j) = imul(x[j], -a * dBy[z]);
        x[j] = imul(x[j], b * By[z]);
    }
    fwd_fft<G>(x, xch, tw, t, gmask);
    finish(2, [&](int, int, double, cplx g) { return g; });  // F_b = fwd(ky By u)  (MHD_BQlin.cpp:182-185)
    // 4. R_zeta: A1 += i b By R_zeta
    load(1);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) {
        const int z = zpos<G>(t, j);
        PRIV(A1, j) = cadd(PRIV(A1, j), imul(x[j], b * By[z]));
    }
    // 5. R_{i kz uz}: G_eta = A1 - 2 dzBy R_kzuz - ddBy R_uz -> F_eta
    load(6);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) {
        const int z = zpos<G>(t, j);
        cplx g = cadd(PRIV(A1, j), cscale(x[j], -2.0 * dBy[z]));
        x[j] = csub(g, cscale(PRIV(K2, j), ddBy[z]));
    }
    fwd_fft<G>(x, xch, tw, t, gmask);
    {
        const cplx* bin = u_in + 2 * P.nz;
        // F_eta = fwd(..) - q kz b   (MHD_BQlin.cpp:201)
        finish(3, [&](int, int s, double c, cplx g) { return csub(g, imul(ldc(bin + s), P.q * c)); });
    }
    // 6. R_b: EMF_x -= Re(uz conj b); A1 = -i a dzBy R_b + ddBy R_bz; A2 = fwd(i b By R_b)
    load(2);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) {
        const int z = zpos<G>(t, j);
        cplx k2v = PRIV(K2, j);
        emfx[j] -= mult * (k2v.x * x[j].x + k2v.y * x[j].y);
        PRIV(A1, j) = cadd(imul(x[j], -a * dBy[z]), cscale(PRIV(K1, j), ddBy[z]));
        x[j] = imul(x[j], b * By[z]);
    }
    fwd_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int k2 = 0; k2 < Pn; ++k2) PRIV(A2, k2) = x[k2];
    // 7. R_eta: G_zeta = A1 + i b By R_eta -> F_zeta
    load(3);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) {
        const int z = zpos<G>(t, j);
        x[j] = cadd(PRIV(A1, j), imul(x[j], b * By[z]));
    }
    fwd_fft<G>(x, xch, tw, t, gmask);
    {
        const cplx* uin0 = u_in;
        const double qm = P.q - Om2;
        // F_zeta = fwd(..) + (q - 2 Omega) kz u   (MHD_BQlin.cpp:178)
        finish(1, [&](int, int s, double c, cplx g) { return cadd(g, imul(ldc(uin0 + s), qm * c)); });
    }
    // 8. G_u2 = 2ab dzBy R_bz -> F_u = A2 + ilapF (2abq u + 2 Omega kz zeta + fwd(G_u2))
#pragma unroll
    for (int j = 0; j < Pn; ++j) {
        const int z = zpos<G>(t, j);
        x[j] = cscale(PRIV(K1, j), 2.0 * ab * dBy[z]);
    }
    fwd_fft<G>(x, xch, tw, t, gmask);
    {
        const cplx* uin0 = u_in;
        const cplx* zin = u_in + P.nz;
        const double c2 = __dmul_rn(__dmul_rn(2.0, ab), P.q);
        finish(0, [&](int k2, int s, double c, cplx g) {
            // MHD_BQlin.cpp:162, ilapF = 1/(-kx^2 + lap2) with the kx=ky=kz=0 fix (:505-507)
            const bool z0 = (kyi == 0 && s == 0);
            const double lapF = __dadd_rn(-__dmul_rn(a, a), lap2val(ky, kz2val(c), z0));
            const double ilapF = (z0 && kxi == 0) ? 1.0 : __drcp_rn(lapF);
            cplx lin = cadd(cadd(cscale(ldc(uin0 + s), c2), imul(ldc(zin + s), Om2 * c)), g);
            return cadd(PRIV(A2, k2), cscale(lin, ilapF));
        });
    }
    // 9-10. EMF_y = Re(bz conj uy) - Re(uz conj by)
    load(7);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) {
        cplx k1 = PRIV(K1, j);
        emfy[j] += mult * (k1.x * x[j].x + k1.y * x[j].y);
    }
    load(8);
    inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
    for (int j = 0; j < Pn; ++j) {
        cplx k2v = PRIV(K2, j);
        emfy[j] -= mult * (k2v.x * x[j].x + k2v.y * x[j].y);
    }
#undef PRIV
}

}  // namespace qlgpu
