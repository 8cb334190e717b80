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
#include "qlgpu_debug.cuh"
#include "qlgpu_fft.cuh"
#include "qlgpu_priv.cuh"
#include "qlgpu_types.h"

namespace qlgpu {

// ---------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------
// State loads (fields, previous right-hand sides) go through L2 (ld.global.cg):
// the persistent batch kernel rewrites these buffers while it runs, so the
// non-coherent read-only path must not cache them.
__device__ __forceinline__ cplx ldc(const cplx* p) {
    double2 v = __ldcg(reinterpret_cast<const double2*>(p));
    return mk(v.x, v.y);
}
// The fields of the mode being transformed, staged in shared memory by its pair.
__device__ __forceinline__ cplx lds(const cplx* p) { return *p; }
// A read of the mode's input fields: the pair's staged copy in shared memory
// (STG) or an L2-coherent global load where the field is used.
template <bool STG>
__device__ __forceinline__ cplx ldu(const cplx* p) {
    if constexpr (STG) return lds(p);
    else return ldc(p);
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

// Asynchronous prefetch of a contiguous range into L2 (one bulk request, no
// registers or shared memory held; bytes a multiple of 16, address 16-aligned).
__device__ __forceinline__ void l2_prefetch(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// SM cycle counter, ordered with the surrounding memory operations (trace only)
__device__ __forceinline__ unsigned long long ctimer() {
    unsigned long long v;
    asm volatile("mov.u64 %0, %%clock64;" : "=l"(v)::"memory");
    return v;
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long v;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(v)::"memory");
    return v;
}

// Asynchronous global -> shared copies (cp.async), 16 or 8 bytes each
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

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
// Per-stage tables shared by all modes of a CTA: exp(linC * coef * kz2) for the
// factored integrating factor of RK3CN_Elin (exp(linC L) = exp(linC c h)
// exp(linC c kz2) with L = c ((-kx^2 - ky^2) + kz2), MHD_BQlin.cpp:249-252).
// ---------------------------------------------------------------------------
struct StageTables {
    const double* ekz_u;  // [nz]  exp(linC nu kz2)
    const double* ekz_b;  // [nz]  exp(linC (eta/nu) nu kz2)
    const double* ilap2;  // [Ny/2][nz] 1/lap2 with the ky=kz=0 fix (Kdata.cpp:100-119)
};

// Buffers of the private store used by the BQlin pipeline
enum { PB_E = 0, PB_A = 1, PB_S = 2, PB_COUNT = 3 };

// ---------------------------------------------------------------------------
// MHD_BQlin right-hand side (MHD_BQlin.cpp:135-257) fused with the RK update
// for one mode, held by a PAIR of transform groups that run the same code on
// mirrored fields: role 0 ("U") owns the velocity-side transforms, role 1
// ("B") the magnetic-side ones.  Real-space fields are R_f = inv(f/NZ); the
// scalar wavenumbers (i kx, i ky) commute with the z transforms and are applied
// in real space.  Only R_uz and R_bz cross between the two groups (shared
// memory KU, KB); everything else stays in each thread's private store.
//
//   step  U (velocity side)                      B (magnetic side)
//   0 inv R_uz -> KU                             R_bz -> KB
//   1 inv R_u : Ex += Re(KB R_u*)                R_b : Ex -= Re(KU R_b*)
//         A = -i kx dBy R_u                      A = -i kx dBy R_b + ddBy KB
//     fwd i ky By R_u -> F_b (update b)          i ky By R_b -> S
//   2 inv R_zeta : A += i ky By R_zeta           R_eta : G = A + i ky By R_eta
//     fwd (idle)                                 G -> F_zeta (update zeta)
//   3 inv R_{i kz uz} :                          R_by : Ey -= Re(KU R_by*)
//         G = A - 2 dBy R - ddBy KU                     G = 2 kx ky dBy KB
//     fwd G -> F_eta (update eta)                G -> F_u = S + ilapF(...) (update u)
//   4 inv R_uy : Ey += Re(KB R_uy*)              (idle)
// The stress profiles Ex, Ey (MHD_BQlin.cpp:212-241) are summed over modes
// before their forward transform (linear), in each thread's private store.
// All lanes of a warp run the same step at the same time (warp-convergent);
// `valid` is false for the padding pairs of the last pass (no stores, no sums).
// ---------------------------------------------------------------------------
struct PairShared {
    cplx* KU;  // R_uz, [P][T]
    cplx* KB;  // R_bz, [P][T]
};

template <class G, int INTEG, class Priv, bool STG>
__device__ __forceinline__ void bqlin_pair(const StageArgs& A, const DevParams& P, const StageTables& TB, int mode,
                                           bool valid, int role, int t, unsigned gmask, unsigned pmask, cplx* xch,
                                           const PairShared& ps, const Priv& pv, const cplx* tw, const double* mfr,
                                           double tclock, const CnOld& cn, const cplx* stg) {
    constexpr int Pn = G::P;
    const StageConst& S = A.sc;
    const double fac = P.fac;
    if (A.trace && blockIdx.x == 0 && threadIdx.x == 0) A.trace[7] = gtimer();
    const double ky = __ldg(A.ky + mode);
    const double kx0 = __ldcg(A.kx0 + mode);
    const int kyi = __ldg(A.kyi + mode), kxi = __ldg(A.kxi + mode);
    const double ts = S.abs_time ? S.t_off : __dadd_rn(tclock, S.t_off);
    const double a = kx_at(kx0, P.q, ts, ky);  // kx(t_s), MHD_BQlin.cpp:498
    const double b = ky;
    const double ab = __dmul_rn(a, b);
    const double Om2 = __dmul_rn(2.0, P.Omega);
    const double mult = valid ? ((ky == 0.0) ? 1.0 : 2.0) : 0.0;
    const cplx* __restrict__ u_in = stg;  // this mode's lin_in fields (staged copy or global, STG)
    cplx* u_out = A.lin_out + (size_t)mode * 4 * P.nz;
    const cplx* Fp = (A.Fprev && S.has_prev) ? A.Fprev + (size_t)mode * 4 * P.nz : nullptr;
    cplx* Fo = A.Fout ? A.Fout + (size_t)mode * 4 * P.nz : nullptr;
    const double* By = mfr;
    const double* dBy = mfr + G::NZ;
    const double* ddBy = mfr + 2 * G::NZ;
    const double* __restrict__ il2row = TB.ilap2 + (size_t)kyi * P.nz;
    cplx* Kown = role ? ps.KB : ps.KU;
    const cplx* Koth = role ? ps.KU : ps.KB;
    const int fbase = role ? 2 : 0;  // u,zeta for U; b,eta for B

    // Stage-end operator: kx' = kx(t_s) + q dt_lin ky (MHD_BQlin.cpp:248)
    const double kxe = __dadd_rn(a, __dmul_rn(__dmul_rn(P.q, S.dt_lin), ky));
    const double hxy = __dsub_rn(-__dmul_rn(kxe, kxe), __dmul_rn(ky, ky));
    double em_u = 1.0, em_b = 1.0;
    if (INTEG == INTEG_EXP && !A.rhs_only) {
        em_u = exp(S.linC * P.nu * hxy);
        em_b = exp(S.linC * P.cb * hxy);
    }
    double kxo = 0.0;  // CN: kx of the previous stage end (or of t0 for the init form)
    if (INTEG == INTEG_CN) {
        if (cn.old_init) kxo = kx_at(kx0, P.q, tclock, ky);
        else kxo = __dadd_rn(kx_at(kx0, P.q, cn.t_old, ky), __dmul_rn(__dmul_rn(P.q, cn.dtlin_old), ky));
    }
    const bool tr = A.trace && blockIdx.x == 0 && threadIdx.x == 0;
    if (tr) A.trace[8] = gtimer();

    cplx x[Pn];
    __syncwarp(pmask);  // the previous mode's readers of KU / KB are done

#pragma unroll 1
    for (int step = 0; step < 5; ++step) {
        if (tr) A.trace[9 + step] = gtimer();
        const bool trs = tr && step == 1;  // cycle stamps of the phases of step 1: [23..27]
        if (trs) A.trace[23] = ctimer();
        // field updated by this group's forward transform at this step (-1: none)
        int fupd = -1;
        if (step == 1) fupd = role ? -2 : 2;  // B: S buffer
        if (step == 2) fupd = role ? 1 : -1;
        if (step == 3) fupd = role ? 0 : 3;
        // ---- inverse transform of this step's field (scaled by 1/NZ)
        {
            // kind: 0 plain, 1 z-component (a c f0 - i b f1) il2, 2 i kz z-component,
            //       3 y-component (ab f0 + i c f1) il2 (MHD_BQlin.cpp:143-146), 4 none
            int kind, f0;
            switch (step) {
                case 0: kind = 1; f0 = fbase; break;
                case 1: kind = 0; f0 = fbase; break;
                case 2: kind = 0; f0 = fbase + 1; break;
                case 3: kind = role ? 3 : 2; f0 = fbase; break;
                default: kind = role ? 4 : 3; f0 = fbase; break;
            }
            const cplx* __restrict__ p0 = u_in + f0 * P.nz;
            const cplx* __restrict__ p1 = p0 + P.nz;
#pragma unroll
            for (int k2 = 0; k2 < Pn; ++k2) {
                const int k = t + G::T * k2;
                const int s = QLGPU_CHECK_STORED(stored_index<G>(k), P.nz, &A.clk->status);
                cplx v = mk(0.0, 0.0);
                if (s >= 0 && kind != 4) {
                    const cplx g0 = ldu<STG>(p0 + s);
                    if (kind == 0) {
                        v = g0;
                    } else {
                        const cplx g1 = ldu<STG>(p1 + s);
                        const double c = kzval(kz_int<G>(k), P.kzL);
                        const double il2 = __ldg(il2row + s);
                        if (kind == 3) {
                            v = cscale(cadd(cscale(g0, ab), imul(g1, c)), il2);
                        } else {
                            v = cscale(csub(cscale(g0, __dmul_rn(a, c)), imul(g1, b)), il2);
                            if (kind == 2) v = imul(v, c);
                        }
                    }
                }
                x[k2] = cscale(v, fac);
            }
            inv_fft<G>(x, xch, tw, t, gmask);
        }
        if (trs) A.trace[24] = ctimer();
        // ---- real-space products (role-dependent values are selected, not branched:
        // every TMEM access below is executed by the whole warp)
        __syncwarp();
        if (step == 0) {
#pragma unroll
            for (int j = 0; j < Pn; ++j) Kown[j * G::T + t] = x[j];
            __syncwarp();
        } else if (step == 1) {
            // U: Ex += Re(R_bz R_u*), A = -i kx dBy R_u
            // B: Ex -= Re(R_uz R_b*), A = -i kx dBy R_b + ddBy R_bz
            const double sg = role ? -mult : mult;
            const double kdd = role ? 1.0 : 0.0;
#pragma unroll
            for (int c4 = 0; c4 < Pn / 4; ++c4) {
                cplx e[4], av[4];
                pv.ld4(PB_E, c4, e);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int j = 4 * c4 + i;
                    const int z = zpos<G>(t, j);
                    const cplx ko = Koth[j * G::T + t];
                    e[i].x += sg * (ko.x * x[j].x + ko.y * x[j].y);
                    av[i] = cadd(imul(x[j], -a * dBy[z]), cscale(Kown[j * G::T + t], kdd * ddBy[z]));
                    x[j] = imul(x[j], b * By[z]);
                }
                __syncwarp();
                pv.st4(PB_E, c4, e);
                pv.st4(PB_A, c4, av);
            }
            pv.st_fence();
        } else if (step == 2) {
            // U: A += i ky By R_zeta;  B: G_zeta = A + i ky By R_eta
#pragma unroll
            for (int c4 = 0; c4 < Pn / 4; ++c4) {
                cplx av[4];
                pv.ld4(PB_A, c4, av);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int j = 4 * c4 + i;
                    av[i] = cadd(av[i], imul(x[j], b * By[zpos<G>(t, j)]));
                    x[j] = av[i];
                }
                pv.st4(PB_A, c4, av);
            }
            pv.st_fence();
        } else if (step == 3) {
            // U: G_eta = A - 2 dBy R_{i kz uz} - ddBy R_uz       (MHD_BQlin.cpp:189-198)
            // B: Ey -= Re(R_uz R_by*);  G_u2 = 2ab dBy R_bz       (MHD_BQlin.cpp:156-158,232-240)
            const double sgy = role ? -mult : 0.0;
#pragma unroll
            for (int c4 = 0; c4 < Pn / 4; ++c4) {
                cplx e[4], av[4];
                pv.ld4(PB_E, c4, e);
                pv.ld4(PB_A, c4, av);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int j = 4 * c4 + i;
                    const int z = zpos<G>(t, j);
                    const cplx ko = Koth[j * G::T + t];
                    const cplx kw = Kown[j * G::T + t];
                    e[i].y += sgy * (ko.x * x[j].x + ko.y * x[j].y);
                    const cplx gu = csub(cadd(av[i], cscale(x[j], -2.0 * dBy[z])), cscale(kw, ddBy[z]));
                    const cplx gb = cscale(kw, 2.0 * ab * dBy[z]);
                    x[j] = role ? gb : gu;
                }
                __syncwarp();
                pv.st4(PB_E, c4, e);
            }
            pv.st_fence();
        } else {
            // step 4, U: Ey += Re(R_bz R_uy*)  (B contributes zero)
            const double sgy = role ? 0.0 : mult;
#pragma unroll
            for (int c4 = 0; c4 < Pn / 4; ++c4) {
                cplx e[4];
                pv.ld4(PB_E, c4, e);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int j = 4 * c4 + i;
                    const cplx ko = Koth[j * G::T + t];
                    e[i].y += sgy * (ko.x * x[j].x + ko.y * x[j].y);
                }
                pv.st4(PB_E, c4, e);
            }
            pv.st_fence();
            break;
        }
        // ---- forward transform and the update of one field
        if (trs) A.trace[25] = ctimer();
        fwd_fft<G>(x, xch, tw, t, gmask);
        if (trs) A.trace[26] = ctimer();
        __syncwarp();
        if (step == 1) {
            // B keeps fwd(i ky By R_b) for F_u (the U lanes store into their own, unused, buffer)
#pragma unroll
            for (int c4 = 0; c4 < Pn / 4; ++c4) pv.st4(PB_S, c4, x + 4 * c4);
            pv.st_fence();
        }
        if (trs) A.trace[28] = ctimer();
        const int f = fupd;  // field this group updates now (-1/-2: none)
        const int fs = f < 0 ? 0 : f;
        const cplx* __restrict__ fin = u_in + fs * P.nz;
        const cplx* __restrict__ lin0 = u_in + (f == 3 ? 2 : 0) * P.nz;
        const cplx* __restrict__ zin = u_in + P.nz;
        const cplx* __restrict__ fpp = Fp ? Fp + fs * P.nz : nullptr;
        cplx* __restrict__ outp = u_out + fs * P.nz;
        cplx* __restrict__ fop = Fo ? Fo + fs * P.nz : nullptr;
        const double* ekzt = (f < 2) ? TB.ekz_u : TB.ekz_b;
        const double em = (f < 2) ? em_u : em_b;
        // linear terms (MHD_BQlin.cpp:162,178,201): F = fu * S + ilapF^fu (x + i cl c l0 + rl l0 + i co c l1)
        const bool fu = (f == 0);
        const double cl = (f == 3) ? -P.q : ((f == 1) ? (P.q - Om2) : 0.0);  // times i kz
        const double rl = fu ? __dmul_rn(__dmul_rn(2.0, ab), P.q) : 0.0;      // 2 kx ky q u (F_u)
        const double co = fu ? Om2 : 0.0;                                      // 2 Omega i kz zeta (F_u)
#pragma unroll
        for (int c4 = 0; c4 < Pn / 4; ++c4) {
            cplx sv[4];
            if (step == 3) {  // the TMEM load is warp-wide: reconverge first
                __syncwarp();
                pv.ld4(PB_S, c4, sv);
            }
            if (f < 0 || !valid) continue;
            cplx uin[4], fpv[4], l0[4], l1[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int s = QLGPU_CHECK_STORED(stored_index<G>(t + G::T * (4 * c4 + i)), P.nz, &A.clk->status);
                const int sl = s < 0 ? 0 : s;
                uin[i] = ldu<STG>(fin + sl);
                fpv[i] = fpp ? ldc(fpp + sl) : mk(0.0, 0.0);
                l0[i] = ldu<STG>(lin0 + sl);
                l1[i] = ldu<STG>(zin + sl);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int k2 = 4 * c4 + i;
                const int k = t + G::T * k2;
                const int s = QLGPU_CHECK_STORED(stored_index<G>(k), P.nz, &A.clk->status);
                if (s < 0) continue;
                const double c = kzval(kz_int<G>(k), P.kzL);
                const double kz2 = kz2val(c);
                // ilapF = 1/(-kx^2 + lap2) with the kx=ky=kz=0 fix (MHD_BQlin.cpp:505-507)
                const bool z0 = (kyi == 0 && s == 0);
                const double lapF = __dadd_rn(-__dmul_rn(a, a), lap2val(ky, kz2, z0));
                const double ilapF = fu ? ((z0 && kxi == 0) ? 1.0 : __drcp_rn(lapF)) : 1.0;
                const cplx lin = cadd(cadd(x[k2], imul(l0[i], cl * c)), cadd(cscale(l0[i], rl), imul(l1[i], co * c)));
                cplx F = cscale(lin, ilapF);
                if (fu) F = cadd(sv[i], F);
                if (A.rhs_only) {
                    stc(outp + s, F);
                    if (A.linop_out)
                        A.linop_out[((size_t)mode * 4 + f) * P.nz + s] =
                            linop_f<MODEL_BQLIN>(P, lap_end<MODEL_BQLIN>(P, kxe, ky, kz2), f);
                    continue;
                }
                cplx nv;
                if (INTEG == INTEG_EXP) {
                    const double e = em * ekzt[s];
                    const cplx acc = fpp ? cadd(cadd(cscale(F, S.n1), cscale(fpv[i], S.n2)), uin[i])
                                         : cadd(cscale(F, S.n1), uin[i]);
                    nv = cscale(acc, e);
                } else {
                    const double L = linop_f<MODEL_BQLIN>(P, lap_end<MODEL_BQLIN>(P, kxe, ky, kz2), f);
                    const double lo = cn.old_init ? lap_init<MODEL_BQLIN>(P, kxo, lap2val(ky, kz2, z0))
                                                  : lap_end<MODEL_BQLIN>(P, kxo, ky, kz2);
                    nv = rk_update<INTEG_CN>(S, L, linop_f<MODEL_BQLIN>(P, lo, f), F, fpv[i], uin[i],
                                             fpp != nullptr);
                }
                if (fop) stc(fop + s, F);
                stc(outp + s, nv);
            }
        }
        __syncwarp();
        if (trs) A.trace[27] = ctimer();
    }
}

// ---------------------------------------------------------------------------
// One coefficient update of field f at stored index s (the RK3 stage update of
// RK3CN_Elin.cpp:102-104 / RK3CN.cpp:105-107), writing F (stages 1,2) and the
// new value; rhs-only mode writes F and the linear operator instead.
// ---------------------------------------------------------------------------
template <int MODEL, int INTEG>
__device__ __forceinline__ void update_coef(const StageArgs& A, const DevParams& P, const StageConst& S,
                                            const StageTables& TB, const CnOld& cn, int mode, int f, int s, double c,
                                            double kz2, double kxe, double kxo, double ky, int kyi, double em,
                                            cplx F, cplx uin, const cplx* fpp, cplx* outp, cplx* fop) {
    if (A.rhs_only) {
        stc(outp + s, F);
        if (A.linop_out)
            A.linop_out[((size_t)mode * 4 + f) * P.nz + s] = linop_f<MODEL>(P, lap_end<MODEL>(P, kxe, ky, kz2), f);
        return;
    }
    const cplx fpv = fpp ? ldc(fpp + s) : mk(0.0, 0.0);
    cplx nv;
    if (INTEG == INTEG_EXP) {
        double e;
        if (P.factored) e = em * ((f < 2) ? TB.ekz_u : TB.ekz_b)[s];
        else e = exp(__dmul_rn(S.linC, linop_f<MODEL>(P, lap_end<MODEL>(P, kxe, ky, kz2), f)));
        const cplx acc = fpp ? cadd(cadd(cscale(F, S.n1), cscale(fpv, S.n2)), uin) : cadd(cscale(F, S.n1), uin);
        nv = cscale(acc, e);
    } else {
        const double L = linop_f<MODEL>(P, lap_end<MODEL>(P, kxe, ky, kz2), f);
        const bool z0 = (kyi == 0 && s == 0);
        const double lo = cn.old_init ? lap_init<MODEL>(P, kxo, lap2val(ky, kz2, z0)) : lap_end<MODEL>(P, kxo, ky, kz2);
        nv = rk_update<INTEG_CN>(S, L, linop_f<MODEL>(P, lo, f), F, fpv, uin, fpp != nullptr);
    }
    if (fop) stc(fop + s, F);
    stc(outp + s, nv);
}

// ---------------------------------------------------------------------------
// MHD_FullQlin right-hand side (MHD_FullQlin.cpp:209-381) fused with the RK
// update for one mode held by a pair of transform groups.  The six real-space
// components U = (Ux, Uy, Uz), B = (Bx, By, Bz) are shared through shared
// memory (SH[6][P][T]); d/dx and d/dy are the scalars i kx, i ky applied in z
// space, so only 10 inverse transforms are needed (the reference does 22).
// With aU = i(kx MUx + ky MUy), aB = i(kx MBx + ky MBy) (MHD_FullQlin.cpp:271-299):
//   T1 = aU Ux + Uz dzMUx - aB Bx - Bz dzMBx    S1 = aU Bx + Uz dzMBx - aB Ux - Bz dzMUx
//   T2 = aU Uy + Uz dzMUy - aB By - Bz dzMBy    S2 = aU By + Uz dzMBy - aB Uy - Bz dzMUy
//   T3 = aU Uz - aB Bz                          S3 = aU Bz - aB Uz
//   step  U (velocity side)                     B (magnetic side)
//   0-2 inv Ux, Uy, Uz -> SH                    Bx, By, Bz -> SH
//   3 inv dz Ux : stresses; fwd T1 -> S_1       dz Bx : stresses; fwd S1 -> F_b
//   4 inv dz Uy : stresses; fwd T2 -> S_2       dz By : stresses; fwd S2 -> S_2
//   5 fwd T3 -> F_u, F_zeta                     fwd S3 -> F_eta
// Stresses (MHD_FullQlin.cpp:314-362): E.x Bx drive, E.y By drive (U side,
// differentiated in z after the sum), E2.x Ux drive, E2.y Uy drive.
// ---------------------------------------------------------------------------
enum { PF_E = 0, PF_E2 = 1, PF_S1 = 2, PF_S2 = 3, PF_COUNT = 4 };

template <class G, int INTEG, class Priv, bool STG>
__device__ __forceinline__ void fullqlin_pair(const StageArgs& A, const DevParams& P, const StageTables& TB, int mode,
                                              bool valid, int role, int t, unsigned gmask, unsigned pmask, cplx* xch,
                                              cplx* SH, const Priv& pv, const cplx* tw, const double* mfr,
                                              double tclock, const CnOld& cn, const cplx* stg) {
    constexpr int Pn = G::P;
    const StageConst& S = A.sc;
    const double fac = P.fac;
    const double ky = __ldg(A.ky + mode);
    const double kx0 = __ldcg(A.kx0 + mode);
    const int kyi = __ldg(A.kyi + mode), kxi = __ldg(A.kxi + mode);
    const double ts = S.abs_time ? S.t_off : __dadd_rn(tclock, S.t_off);
    const double a = kx_at(kx0, P.q, ts, ky);  // kx(t_s), MHD_FullQlin.cpp:727
    const double b = ky;
    const double ab = __dmul_rn(a, b);
    const double Om2 = __dmul_rn(2.0, P.Omega);
    const double mult = valid ? ((ky == 0.0) ? 1.0 : 2.0) : 0.0;
    const cplx* __restrict__ u_in = stg;  // this mode's lin_in fields (staged copy or global, STG)
    cplx* u_out = A.lin_out + (size_t)mode * 4 * P.nz;
    const cplx* Fp = (A.Fprev && S.has_prev) ? A.Fprev + (size_t)mode * 4 * P.nz : nullptr;
    cplx* Fo = A.Fout ? A.Fout + (size_t)mode * 4 * P.nz : nullptr;
    const double *MBx = mfr, *dMBx = mfr + G::NZ, *MBy = mfr + 2 * G::NZ, *dMBy = mfr + 3 * G::NZ;
    const double *MUx = mfr + 4 * G::NZ, *dMUx = mfr + 5 * G::NZ, *MUy = mfr + 6 * G::NZ, *dMUy = mfr + 7 * G::NZ;
    const double* __restrict__ il2row = TB.ilap2 + (size_t)kyi * P.nz;
    const int fbase = role ? 2 : 0;
    const double kxe = __dadd_rn(a, __dmul_rn(__dmul_rn(P.q, S.dt_lin), ky));  // MHD_FullQlin.cpp:371
    const double hxy = __dsub_rn(-__dmul_rn(kxe, kxe), __dmul_rn(ky, ky));
    double em_u = 1.0, em_b = 1.0;
    if (INTEG == INTEG_EXP && !A.rhs_only && P.factored) {
        em_u = exp(S.linC * P.nu * hxy);
        em_b = exp(S.linC * P.cb * hxy);
    }
    double kxo = 0.0;
    if (INTEG == INTEG_CN) {
        if (cn.old_init) kxo = kx_at(kx0, P.q, tclock, ky);
        else kxo = __dadd_rn(kx_at(kx0, P.q, cn.t_old, ky), __dmul_rn(__dmul_rn(P.q, cn.dtlin_old), ky));
    }
#define SHV(f, j) SH[((f) * Pn + (j)) * G::T + t]
    cplx x[Pn];
    __syncwarp(pmask);  // the previous mode's readers of SH are done

#pragma unroll 1
    for (int step = 0; step < 6; ++step) {
        // ---- inverse transform (steps 0-4): kind 0 plain, 3 y-component, 1 z-component,
        //      5 i kz * plain, 6 i kz * y-component
        if (step < 5) {
            int kind;
            switch (step) {
                case 0: kind = 0; break;
                case 1: kind = 3; break;
                case 2: kind = 1; break;
                case 3: kind = 5; break;
                default: kind = 6; break;
            }
            const cplx* __restrict__ p0 = u_in + fbase * P.nz;
            const cplx* __restrict__ p1 = p0 + P.nz;
#pragma unroll
            for (int k2 = 0; k2 < Pn; ++k2) {
                const int k = t + G::T * k2;
                const int s = QLGPU_CHECK_STORED(stored_index<G>(k), P.nz, &A.clk->status);
                cplx v = mk(0.0, 0.0);
                if (s >= 0) {
                    const cplx g0 = ldu<STG>(p0 + s);
                    const double c = kzval(kz_int<G>(k), P.kzL);
                    if (kind == 0 || kind == 5) {
                        v = g0;
                    } else {
                        const cplx g1 = ldu<STG>(p1 + s);
                        const double il2 = __ldg(il2row + s);
                        if (kind == 1) v = cscale(csub(cscale(g0, __dmul_rn(a, c)), imul(g1, b)), il2);
                        else v = cscale(cadd(cscale(g0, ab), imul(g1, c)), il2);  // (MHD_FullQlin.cpp:220-221)
                    }
                    if (kind >= 5) v = imul(v, c);
                }
                x[k2] = cscale(v, fac);
            }
            inv_fft<G>(x, xch, tw, t, gmask);
        }
        __syncwarp();
        if (step < 3) {
#pragma unroll
            for (int j = 0; j < Pn; ++j) SHV(role * 3 + step, j) = x[j];
            __syncwarp();
            continue;
        }
        // ---- stresses (steps 3, 4) and the forward-transform input
        if (step < 5) {
            const double sgn = role ? mult : -mult;  // minus the u part, plus the b part
            const double semf = role ? 0.0 : mult;   // EMFs computed once, by the U lanes
#pragma unroll
            for (int c4 = 0; c4 < Pn / 4; ++c4) {
                cplx e[4], e2[4];
                pv.ld4(PF_E, c4, e);
                pv.ld4(PF_E2, c4, e2);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int j = 4 * c4 + i;
                    const cplx Ux = SHV(0, j), Uy = SHV(1, j), Uz = SHV(2, j);
                    const cplx Bx = SHV(3, j), By = SHV(4, j), Bz = SHV(5, j);
                    const cplx Fx = role ? Bx : Ux, Fy = role ? By : Uy, Fz = role ? Bz : Uz;
                    // Re(a conj b)
                    auto rc = [](cplx p, cplx q) { return p.x * q.x + p.y * q.y; };
                    if (step == 3) {
                        // EMF (MHD_FullQlin.cpp:322,330): Re(bz ux*) - Re(uz bx*), Re(bz uy*) - Re(uz by*)
                        e[i].x += semf * (rc(Bz, Ux) - rc(Uz, Bx));
                        e[i].y += semf * (rc(Bz, Uy) - rc(Uz, By));
                        // x drive (:342-343): Re(Fx (i kx Fx)*) + Re(Fy (i ky Fx)*) + Re(Fz (dz Fx)*)
                        e2[i].x += sgn * (rc(Fx, imul(Fx, a)) + rc(Fy, imul(Fx, b)) + rc(Fz, x[j]));
                    } else {
                        // y drive (:357-358): Re(Fx (i kx Fy)*) + Re(Fy (i ky Fy)*) + Re(Fz (dz Fy)*)
                        e2[i].y += sgn * (rc(Fx, imul(Fy, a)) + rc(Fy, imul(Fy, b)) + rc(Fz, x[j]));
                    }
                }
                __syncwarp();
                pv.st4(PF_E, c4, e);
                pv.st4(PF_E2, c4, e2);
            }
            pv.st_fence();
        }
        // forward input: U -> T(step-2), B -> S(step-2)
#pragma unroll
        for (int j = 0; j < Pn; ++j) {
            const int z = zpos<G>(t, j);
            const cplx Ux = SHV(0, j), Uy = SHV(1, j), Uz = SHV(2, j);
            const cplx Bx = SHV(3, j), By = SHV(4, j), Bz = SHV(5, j);
            const double aU = a * MUx[z] + b * MUy[z], aB = a * MBx[z] + b * MBy[z];  // times i
            const cplx Fx = role ? Bx : Ux, Gx = role ? Ux : Bx;   // own / other x component
            const cplx Fy = role ? By : Uy, Gy = role ? Uy : By;
            const cplx Fz = role ? Bz : Uz, Gz = role ? Uz : Bz;
            // T_n: aU U - aB B (+ z terms);  S_n: aU B - aB U (+ z terms)
            const cplx own = role ? Bx : Ux;
            (void)own;
            cplx v;
            if (step == 3) {
                const double d1 = role ? dMBx[z] : dMUx[z], d2 = role ? dMUx[z] : dMBx[z];
                v = csub(cadd(imul(Fx, aU), cscale(Uz, d1)), cadd(imul(Gx, aB), cscale(Bz, d2)));
            } else if (step == 4) {
                const double d1 = role ? dMBy[z] : dMUy[z], d2 = role ? dMUy[z] : dMBy[z];
                v = csub(cadd(imul(Fy, aU), cscale(Uz, d1)), cadd(imul(Gy, aB), cscale(Bz, d2)));
            } else {
                v = csub(imul(Fz, aU), imul(Gz, aB));
            }
            x[j] = v;
        }
        fwd_fft<G>(x, xch, tw, t, gmask);
        __syncwarp();
        if (step == 3 || step == 4) {
            // U keeps T1 (step 3) and T2 (step 4); B keeps S2 (step 4)
#pragma unroll
            for (int c4 = 0; c4 < Pn / 4; ++c4) pv.st4(step == 3 ? PF_S1 : PF_S2, c4, x + 4 * c4);
            pv.st_fence();
        }
        // ---- updates: step 3 B -> F_b; step 5 U -> F_u, F_zeta; B -> F_eta
#pragma unroll
        for (int c4 = 0; c4 < Pn / 4; ++c4) {
            cplx s1v[4], s2v[4];
            __syncwarp();
            if (step == 5) {
                pv.ld4(PF_S1, c4, s1v);
                pv.ld4(PF_S2, c4, s2v);
            }
            if (!valid || step == 4 || (step == 3 && role == 0)) continue;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int k2 = 4 * c4 + i;
                const int k = t + G::T * k2;
                const int s = QLGPU_CHECK_STORED(stored_index<G>(k), P.nz, &A.clk->status);
                if (s < 0) continue;
                const double c = kzval(kz_int<G>(k), P.kzL);
                const double kz2 = kz2val(c);
                const cplx u0 = ldu<STG>(u_in + s), ze = ldu<STG>(u_in + P.nz + s), b0 = ldu<STG>(u_in + 2 * P.nz + s),
                           et = ldu<STG>(u_in + 3 * P.nz + s);
                if (step == 3) {
                    // F_b = B0z kz u - s1 (MHD_FullQlin.cpp:303)
                    const cplx F = csub(imul(u0, P.B0z * c), x[k2]);
                    update_coef<MODEL_FULLQLIN, INTEG>(A, P, S, TB, cn, mode, 2, s, c, kz2, kxe, kxo, ky, kyi, em_b,
                                                       F, b0, Fp ? Fp + 2 * P.nz : nullptr, u_out + 2 * P.nz,
                                                       Fo ? Fo + 2 * P.nz : nullptr);
                } else if (role == 0) {
                    // F_u, F_zeta (MHD_FullQlin.cpp:283-285) with t1 = S1, t2 = S2, t3 = x
                    const cplx t1 = s1v[i], t2 = s2v[i], t3 = x[k2];
                    const bool z0 = (kyi == 0 && s == 0);
                    const double lapF = __dadd_rn(-__dmul_rn(a, a), lap2val(ky, kz2, z0));
                    const double ilapF = (z0 && kxi == 0) ? 1.0 : __drcp_rn(lapF);
                    // (-2 kx ky q) u + 2 Om kz zeta + kx^2 t1 + kx ky t2 + kx kz t3, kx = i a etc.
                    cplx inner = cadd(cscale(u0, __dmul_rn(__dmul_rn(2.0, ab), P.q)), imul(ze, Om2 * c));
                    inner = csub(inner, cadd(cadd(cscale(t1, a * a), cscale(t2, ab)), cscale(t3, a * c)));
                    const cplx Fu = csub(cadd(cscale(inner, ilapF), imul(b0, P.B0z * c)), t1);
                    // zeta: (q - 2 Om) kz u + B0z kz eta - (kz t2 - ky t3)
                    const cplx Fz = csub(cadd(imul(u0, (P.q - Om2) * c), imul(et, P.B0z * c)),
                                         csub(imul(t2, c), imul(t3, b)));
                    update_coef<MODEL_FULLQLIN, INTEG>(A, P, S, TB, cn, mode, 0, s, c, kz2, kxe, kxo, ky, kyi, em_u,
                                                       Fu, u0, Fp, u_out, Fo);
                    update_coef<MODEL_FULLQLIN, INTEG>(A, P, S, TB, cn, mode, 1, s, c, kz2, kxe, kxo, ky, kyi, em_u,
                                                       Fz, ze, Fp ? Fp + P.nz : nullptr, u_out + P.nz,
                                                       Fo ? Fo + P.nz : nullptr);
                } else {
                    // F_eta = -q kz b + B0z kz zeta - (kz s2 - ky s3) (MHD_FullQlin.cpp:305)
                    const cplx s2 = s2v[i], s3 = x[k2];
                    const cplx Fe = csub(cadd(imul(b0, -P.q * c), imul(ze, P.B0z * c)), csub(imul(s2, c), imul(s3, b)));
                    update_coef<MODEL_FULLQLIN, INTEG>(A, P, S, TB, cn, mode, 3, s, c, kz2, kxe, kxo, ky, kyi, em_b,
                                                       Fe, et, Fp ? Fp + 3 * P.nz : nullptr, u_out + 3 * P.nz,
                                                       Fo ? Fo + 3 * P.nz : nullptr);
                }
            }
        }
        __syncwarp();
    }
#undef SHV
}

}  // namespace qlgpu
