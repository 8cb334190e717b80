// qlgpu_kernel.cuh -- the stage kernel (sm_100a): mean-field profiles, the
// per-mode loop, the remap / diagnostics epilogue, the fixed-order two-level
// reduction over CTAs and the mean-field update done by the last CTA.
#pragma once
#include <type_traits>

#include "qlgpu_debug.cuh"
#include "qlgpu_noise.cuh"
#include "qlgpu_stage.cuh"

namespace qlgpu {

constexpr int RED_GROUP = 16;  // CTAs per first-level reduction group

// Mean-field real-space profiles for the stage (MHD_BQlin.cpp:122-127:
// By, dz By, dz^2 By; MHD_FullQlin.cpp:180-198: Bx, By, Ux, Uy and dz of each),
// real part kept (the mean fields are real in z).
template <class G, int MODEL>
__device__ __forceinline__ void mean_profiles(const DevParams& P, const cplx* mf, double* mfr, cplx* xch, const cplx* tw,
                                              int gidx, int ngroups, int t, unsigned gmask) {
    constexpr int NMFR = MODEL == MODEL_BQLIN ? 3 : 8;
    for (int arr = gidx; arr < NMFR; arr += ngroups) {
        int src, deriv;
        if (MODEL == MODEL_BQLIN) {
            src = 1;
            deriv = arr;  // 0: By, 1: dz By, 2: dz^2 By
        } else {
            src = arr / 2;  // Bx, By, Ux, Uy
            deriv = arr % 2;
        }
        cplx x[G::P];
#pragma unroll
        for (int k2 = 0; k2 < G::P; ++k2) {
            const int k = t + G::T * k2;
            const int s = stored_index<G>(k);
            cplx v = mk(0.0, 0.0);
            if (s >= 0) {
                v = cscale(ldc_cg(mf + src * P.nz + s), P.fac);
                const double c = kzval(kz_int<G>(k), P.kzL);
                if (deriv == 1) v = imul(v, c);
                if (deriv == 2) v = cscale(v, kz2val(c));
            }
            x[k2] = v;
        }
        inv_fft<G>(x, xch, tw, t, gmask);
#pragma unroll
        for (int j = 0; j < G::P; ++j) mfr[arr * G::NZ + zpos<G>(t, j)] = x[j].x;
    }
}

// Diagnostic contributions of one mode at time t (MHD_BQlin.cpp:365-407):
// acc[0..5] += mult*{energy_u, energy_b, AM_u, AM_b}, mult*nu*diss_u, mult*eta*diss_b
template <class G>
__device__ __forceinline__ void mode_diag(const DevParams& P, const cplx* u, int mode_kxi, int kyi, double kx0,
                                          double ky, double t, int tt, double* acc) {
    const double a = kx_at(kx0, P.q, t, ky);
    const double ab = __dmul_rn(a, ky);
    const double mult = (ky == 0.0) ? 1.0 : 2.0;
    (void)mode_kxi;
#pragma unroll
    for (int k2 = 0; k2 < G::P; ++k2) {
        const int k = tt + G::T * k2;
        const int s = stored_index<G>(k);
        if (s < 0) continue;
        const double c = kzval(kz_int<G>(k), P.kzL);
        const bool z0 = (kyi == 0 && s == 0);
        const double lap2 = lap2val(ky, kz2val(c), z0);
        const double il2 = ilap2val(lap2, z0);
        const double lapF = __dadd_rn(-__dmul_rn(a, a), lap2);
        const double l2 = __dmul_rn(lapF, il2);
        cplx f[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) f[v] = ldc_cg(u + v * P.nz + s);
        const double n0 = f[0].x * f[0].x + f[0].y * f[0].y, n1 = f[1].x * f[1].x + f[1].y * f[1].y;
        const double n2 = f[2].x * f[2].x + f[2].y * f[2].y, n3 = f[3].x * f[3].x + f[3].y * f[3].y;
        const double eu = l2 * n0 - il2 * n1, eb = l2 * n2 - il2 * n3;
        acc[0] += mult * eu;
        acc[1] += mult * eb;
        // uy = (ab u + i c zeta) ilap2 (MHD_BQlin.cpp:388-392)
        cplx uy = cscale(cadd(cscale(f[0], ab), imul(f[1], c)), il2);
        cplx by = cscale(cadd(cscale(f[2], ab), imul(f[3], c)), il2);
        acc[2] += mult * (f[0].x * uy.x + f[0].y * uy.y);
        acc[3] += mult * (f[2].x * by.x + f[2].y * by.y);
        acc[4] += mult * P.nu * (-lapF * eu);
        acc[5] += mult * P.eta * (-lapF * eb);
    }
}

// ---------------------------------------------------------------------------
// Mean-field stage, run by the CTA that arrives last: stress spectra, the
// mean-field right-hand side and RK update, the time / diagnostic bookkeeping.
// tot[] holds the stress profiles summed over all modes (real z) followed by
// the six fluctuation diagnostic sums.
// ---------------------------------------------------------------------------
template <class G, int MODEL, int INTEG, int NEMF>
__device__ __forceinline__ void mean_field_stage(const StageArgs& A, const DevParams& P, const double* tot,
                                                 double* spec, cplx* xch, const cplx* tw_s, int gidx, int ngc, int t,
                                                 unsigned gmask, double tclock, double t_new, bool last,
                                                 bool diag_due) {
    const StageConst& S = A.sc;
    const int tid = threadIdx.x;
    const int nzd = P.nz;
    // Forward transform of each summed profile, half spectrum k = 0..H
    // (MHD_BQlin.cpp:228-240 after the sum over modes; the transform is linear)
    for (int e = gidx; e < NEMF; e += ngc) {
        cplx x[G::P];
#pragma unroll
        for (int j = 0; j < G::P; ++j) x[j] = mk(tot[e * G::NZ + zpos<G>(t, j)], 0.0);
        fwd_fft<G>(x, xch, tw_s, t, gmask);
#pragma unroll
        for (int k2 = 0; k2 < G::P; ++k2) {
            const int k = t + G::T * k2;
            if (k <= G::H) {
                cplx v = cscale(x[k2], P.rs_fac);
                if (MODEL == MODEL_BQLIN || e < 2) v = imul(v, kzval(k, P.kzL));  // times kz (z derivative)
                spec[(e * (G::H + 1) + k) * 2 + 0] = v.x;
                spec[(e * (G::H + 1) + k) * 2 + 1] = v.y;
            }
        }
    }
    __syncthreads();
    for (int s = tid; s < nzd; s += blockDim.x) {
        // unpack: full[s] = half[s] (s <= H) or conj(half[nz - s]) (MHD_BQlin.cpp:264-267)
        cplx drive[NEMF];
#pragma unroll
        for (int e = 0; e < NEMF; ++e) {
            const int hs = s <= G::H ? s : nzd - s;
            cplx v = mk(spec[(e * (G::H + 1) + hs) * 2], spec[(e * (G::H + 1) + hs) * 2 + 1]);
            drive[e] = s <= G::H ? v : conjc(v);
        }
        const int kzi = s <= G::H ? s : s - nzd;
        const double c = kzval(kzi, P.kzL);
        const double kz2 = kz2val(c);
        cplx m[4], F[4];
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) {
            m[mm] = (mm < P.nmf) ? ldc_cg(A.mf + mm * nzd + s) : mk(0.0, 0.0);
            F[mm] = mk(0.0, 0.0);
        }
        if (MODEL == MODEL_BQLIN) {
            // dBy = -q Bx + EMF_y, dBx = EMF_x (MHD_BQlin.cpp:274-280)
            if (P.ql) {
                F[0] = drive[0];
                F[1] = cadd(cscale(m[0], -P.q), drive[1]);
            }
        } else {
            // MHD_FullQlin.cpp:411-423 (B0z kz terms with kz = i c)
            if (P.ql) {
                F[1] = cadd(cadd(cscale(m[0], -P.q), imul(m[3], P.B0z * c)), drive[1]);
                F[0] = cadd(imul(m[2], P.B0z * c), drive[0]);
                F[2] = cadd(cadd(cscale(m[3], 2.0 * P.Omega), imul(m[0], P.B0z * c)), drive[2]);
                F[3] = cadd(cadd(cscale(m[2], P.q - 2.0 * P.Omega), imul(m[1], P.B0z * c)), drive[3]);
            }
        }
        for (int mm = 0; mm < P.nmf; ++mm) {
            if (A.rhs_only) {
                stc(A.Fmf_out + mm * nzd + s, F[mm]);
                continue;
            }
            const double Lm = P.ql ? __dmul_rn((MODEL == MODEL_FULLQLIN && mm >= 2) ? P.nu : P.eta, kz2) : 0.0;
            cplx fp = S.has_prev ? ldc_cg(A.Fmf_prev + mm * nzd + s) : mk(0.0, 0.0);
            cplx nv = rk_update<INTEG>(S, Lm, Lm, F[mm], fp, m[mm], S.has_prev);
            if (A.Fmf_out) stc(A.Fmf_out + mm * nzd + s, F[mm]);
            stc(A.mf + mm * nzd + s, nv);
            const double mag = nv.x * nv.x + nv.y * nv.y;
            if (!(mag == mag) || isinf(mag)) atomicOr(&A.clk->status, QLGPU_STATUS_NONFINITE);
            else if (mag > 1e40) atomicOr(&A.clk->status, QLGPU_STATUS_UNSTABLE);
        }
    }
    __syncthreads();
    if (A.rhs_only || tid != 0) return;
    DevClock* C = A.clk;
    // CN bookkeeping: this stage's operator time becomes "old" (RK3CN.cpp:119-122)
    C->t_old = S.abs_time ? S.t_off : __dadd_rn(tclock, S.t_off);
    C->dtlin_old = S.dt_lin;
    C->old_init = 0;
    if (!last) return;
    C->t = t_new;
    C->timevar = __dadd_rn(C->timevar, P.dt);
    C->since += 1;
    C->nstep += 1;
    if (!diag_due) return;
    // Calc_Energy_AM_Diss (MHD_BQlin.cpp:408-477)
    double eMB = 0, aMB = 0, dMB = 0, eMU = 0, aMU = 0, dMU = 0;
    for (int s = 0; s < nzd; ++s) {
        const int kzi = s <= G::H ? s : s - nzd;
        const double kz2 = kz2val(kzval(kzi, P.kzL));
        cplx b0 = ldc_cg(A.mf + s), b1 = ldc_cg(A.mf + nzd + s);
        eMB += (b0.x * b0.x + b0.y * b0.y) + (b1.x * b1.x + b1.y * b1.y);
        aMB += b0.x * b1.x + b0.y * b1.y;
        dMB += -kz2 * (b0.x * b0.x + b0.y * b0.y) - kz2 * (b1.x * b1.x + b1.y * b1.y);
        if (P.nmf == 4) {
            cplx u0 = ldc_cg(A.mf + 2 * nzd + s), u1 = ldc_cg(A.mf + 3 * nzd + s);
            eMU += (u0.x * u0.x + u0.y * u0.y) + (u1.x * u1.x + u1.y * u1.y);
            aMU += u0.x * u1.x + u0.y * u1.y;
            dMU += -kz2 * (u0.x * u0.x + u0.y * u0.y) - kz2 * (u1.x * u1.x + u1.y * u1.y);
        }
    }
    eMB *= P.divMF; eMU *= P.divMF; aMB *= P.divMF; aMU *= P.divMF;
    dMB *= P.divMF * P.eta; dMU *= P.divMF * P.nu;
    const double* ds = tot + NEMF * G::NZ;
    const double eu = ds[0] * P.divfac, eb = ds[1] * P.divfac;
    const double au = ds[2] * P.divfac, abv = ds[3] * P.divfac;
    const double du = ds[4] * P.divfac, db = ds[5] * P.divfac;
    const int r = C->ndiag;
    if (r < A.diag_cap) {
        double* o = A.diag_ring + (size_t)QLGPU_CHECK_INDEX(r, A.diag_cap, &C->status) * 15;
        o[0] = t_new;
        o[1] = eMU / 2; o[2] = eMB / 2; o[3] = eu / 2; o[4] = eb / 2;
        o[5] = aMU; o[6] = aMB; o[7] = au; o[8] = abv;
        o[9] = dMU; o[10] = dMB; o[11] = du; o[12] = db;
        o[13] = pow(P.nu * P.nu * P.nu / (dMU + du), 0.25) * P.kzmax;
        o[14] = pow(P.eta * P.eta * P.eta / (dMB + db), 0.25) * P.kzmax;
    } else {
        C->status |= QLGPU_STATUS_DIAG_FULL;
    }
    C->ndiag = r + 1;
    C->timevar = __dsub_rn(C->timevar, P.tv_interval);
    C->since = 0;
}

// ---------------------------------------------------------------------------
// Shared-memory carve-up of the stage kernel
// ---------------------------------------------------------------------------
template <class G, int MODEL, class Priv, bool STG>
struct Smem {
    static constexpr int SW = 32 / G::T;                        // groups per warp
    static constexpr int NMFR = MODEL == MODEL_BQLIN ? 3 : 8;   // real-space mean-field profiles
    static constexpr int NEMF = MODEL == MODEL_BQLIN ? 2 : 4;   // stress profiles summed over modes
    static constexpr int PL = NEMF * G::NZ + 8;                 // partial vector length (doubles)
    static constexpr int NZD = G::nz;
    // offsets in bytes
    static constexpr size_t o_tw = 0;
    static constexpr size_t o_mfr = o_tw + sizeof(cplx) * G::NZ;
    static constexpr size_t o_ekz = o_mfr + sizeof(double) * NMFR * G::NZ;
    static constexpr size_t o_spec = o_ekz + sizeof(double) * 2 * ((NZD + 1) & ~1);
    static constexpr size_t o_tot = o_spec + sizeof(double) * 2 * NEMF * (G::H + 1);
    static constexpr size_t o_work = o_tot + sizeof(double) * ((PL + 1) & ~1);
    // per pair of groups: BQlin R_uz, R_bz (2 NZ cplx); FullQlin the six components (6 NZ cplx)
    static constexpr size_t GS_BYTES = sizeof(cplx) * G::NZ * (MODEL == MODEL_BQLIN ? 1 : 3);
    // per pair of groups: the 4 nz fields of the mode being transformed, staged once per mode
    // (STG; otherwise the fields are read from L2 where they are used)
    static constexpr size_t STG_BYTES = STG ? sizeof(cplx) * 4 * G::nz : 0;
    __host__ __device__ static size_t work_bytes(int warps) {
        const size_t xch = sizeof(cplx) * (size_t)warps * SW * G::XSIZE;
        const size_t red = sizeof(double) * ((size_t)warps * NEMF * G::NZ + (size_t)warps * 32 * 6);
        return xch > red ? xch : red;
    }
    __host__ __device__ static size_t bytes(int warps) {
        return o_work + work_bytes(warps) + Priv::smem_bytes_per_warp() * (size_t)warps +
               GS_BYTES * (size_t)warps * SW + STG_BYTES * (size_t)warps * (SW / 2);
    }
    __host__ __device__ static int tmem_cols(int warps) {
        int need = Priv::tmem_cols_per_warp() * ((warps + 3) / 4);
        if (need == 0) return 0;
        int c = 32;
        while (c < need) c <<= 1;
        return c;
    }
};

// Static shared words of a stage: the TMEM base address, the last-arriver flag
// and a flag the persistent batch kernel uses to leave its step loop.
struct StageShared {
    uint32_t tmem;
    int last;
    int ok;
    int pad;
};

// Types of one stage variant.  STG: each pair stages its mode's fields in
// shared memory (the single-case kernel always; the persistent batch kernel for
// transforms of up to 8 points per thread, where the shared memory it frees
// for 16-point transforms buys a warp per SM more than staging saves).
template <int NZ, int MODEL, bool USE_TMEM, bool STG = true>
struct StageKind {
    using G = Geom<NZ>;
    static constexpr int NB = MODEL == MODEL_BQLIN ? (int)PB_COUNT : (int)PF_COUNT;
    using Priv = typename std::conditional<USE_TMEM, PrivTmem<G, NB>, PrivSmem<G, NB>>::type;
    using SM = Smem<G, MODEL, Priv, STG>;
};

// One stage over the modes of one case, executed by one CTA that is number
// `cta` of the `ncta` CTAs working on that case.  The CTA's TMEM columns (if
// any) are allocated by the caller and passed in ss.tmem.  Returns true in the
// one CTA that arrived last and ran the mean-field stage; every other CTA
// returns as soon as its partial sums are published.
template <int NZ, int MODEL, int INTEG, bool USE_TMEM, bool STG = true>
__device__ __forceinline__ bool stage_body(const StageArgs& A, const DevParams& P, const int cta, const int ncta,
                                           unsigned char* smem_raw, StageShared& ss) {
    using K = StageKind<NZ, MODEL, USE_TMEM, STG>;
    using G = typename K::G;
    constexpr int NB = K::NB;
    using Priv = typename K::Priv;
    using SM = typename K::SM;
    constexpr int SW = SM::SW;
    static_assert(SW % 2 == 0, "a warp holds whole pairs of groups");
    constexpr int NEMF = SM::NEMF;
    constexpr int PL = SM::PL;
    const int warps = blockDim.x >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int slot = lane / G::T, t = lane % G::T;
    const unsigned gmask = (G::T == 32 ? 0xffffffffu : (((1u << G::T) - 1u) << (slot * G::T)));
    cplx* tw_s = reinterpret_cast<cplx*>(smem_raw + SM::o_tw);
    double* mfr = reinterpret_cast<double*>(smem_raw + SM::o_mfr);
    double* ekz = reinterpret_cast<double*>(smem_raw + SM::o_ekz);
    double* spec = reinterpret_cast<double*>(smem_raw + SM::o_spec);
    double* tot = reinterpret_cast<double*>(smem_raw + SM::o_tot);
    unsigned char* work = smem_raw + SM::o_work;
    cplx* xch = reinterpret_cast<cplx*>(work) + (size_t)(warp * SW + slot) * G::XSIZE;
    const int gidx = warp * SW + slot;  // group index in the CTA
    const int ngc = warps * SW;         // groups per CTA
    const StageConst& S = A.sc;
    const int nzd = P.nz;

    // optional trace (CTA 0 thread 0 and the top CTA): [0] start, [1] prologue done,
    // [2] mode loop done, [3] partials written, [4] top CTA start, [5] top done,
    // [8] first mode staged, [9..18] start of pipeline steps 0..9
    const bool tr = A.trace && cta == 0 && tid == 0;
    const bool tr2 = A.trace && cta == ncta - 1 && tid == 0;
    if (tr) A.trace[0] = gtimer();
    if (tr2) A.trace[20] = gtimer();
    // ---- private store: TMEM allocation (one warp) or a shared-memory region
    Priv pv;
    if constexpr (USE_TMEM) {
        pv.init(ss.tmem, warp);
    } else {
        pv.init(reinterpret_cast<cplx*>(work + SM::work_bytes(warps)) + (size_t)warp * NB * G::P * 32, lane);
    }
    // pair layout: octet o = lane / T, pair pi = o / 2, role = o % 2 (0: velocity side, 1: magnetic side)
    const int role = slot & 1;
    const int pi = slot >> 1;
    const unsigned pmask = (2 * G::T == 32) ? 0xffffffffu : (((1u << (2 * G::T)) - 1u) << (pi * 2 * G::T));
    PairShared ps;
    cplx* stg_buf;  // this pair's staged mode fields
    {
        unsigned char* gbase = work + SM::work_bytes(warps) + Priv::smem_bytes_per_warp() * (size_t)warps;
        cplx* k_all = reinterpret_cast<cplx*>(gbase);
        cplx* kpair = k_all + (size_t)(warp * (SW / 2) + pi) * 2 * G::NZ * (MODEL == MODEL_BQLIN ? 1 : 3);
        ps.KU = kpair;
        ps.KB = kpair + G::NZ;
        cplx* s_all = reinterpret_cast<cplx*>(gbase + SM::GS_BYTES * (size_t)warps * SW);
        stg_buf = s_all + (size_t)(warp * (SW / 2) + pi) * 4 * G::nz;
    }
    {   // zero the stress accumulators
        cplx z4[4] = {mk(0, 0), mk(0, 0), mk(0, 0), mk(0, 0)};
#pragma unroll
        for (int c4 = 0; c4 < G::P / 4; ++c4) {
            pv.st4(0, c4, z4);  // PB_E / PF_E
            if (MODEL == MODEL_FULLQLIN) pv.st4(PF_E2, c4, z4);
        }
        pv.st_fence();
    }

    for (int i = tid; i < G::NZ; i += blockDim.x) tw_s[i] = A.tw[i];
    const double tclock = __ldcg(&A.clk->t);
    CnOld cn;
    cn.t_old = __ldcg(&A.clk->t_old);
    cn.dtlin_old = __ldcg(&A.clk->dtlin_old);
    cn.old_init = __ldcg(&A.clk->old_init);
    // factored integrating factor tables exp(linC c kz2), per stored kz
    if (INTEG == INTEG_EXP) {
        for (int s = tid; s < nzd; s += blockDim.x) {
            if (A.ekz_tab) {
                ekz[s] = __ldg(A.ekz_tab + s);
                ekz[SM::NZD + (SM::NZD & 1) + s] = __ldg(A.ekz_tab + nzd + s);
            } else {
                const int kzi = s <= G::H ? s : s - nzd;
                const double kz2 = kz2val(kzval(kzi, P.kzL));
                ekz[s] = exp(S.linC * P.nu * kz2);
                ekz[SM::NZD + (SM::NZD & 1) + s] = exp(S.linC * P.cb * kz2);
            }
        }
    }
    const bool mfr_cached = A.mfr_cache && !A.rhs_only && __ldcg(&A.clk->mfr_valid);
    if (mfr_cached)
        for (int i = tid; i < SM::NMFR * G::NZ; i += blockDim.x) mfr[i] = __ldcg(A.mfr_cache + i);
    StageTables TB;
    TB.ekz_u = ekz;
    TB.ekz_b = ekz + SM::NZD + (SM::NZD & 1);
    TB.ilap2 = A.ilap2;
    __syncthreads();
    if (!mfr_cached) {
        mean_profiles<G, MODEL>(P, A.mf, mfr, xch, tw_s, gidx, ngc, t, gmask);
        __syncthreads();
    }
    if (tr) A.trace[1] = gtimer();
    if (tr2) A.trace[21] = gtimer();

    // Last-stage bookkeeping identical in every CTA (main.cpp:111-130)
    const double t_new = __dadd_rn(tclock, P.dt);
    const bool last = S.last && !A.rhs_only;
    bool diag_due = false;
    if (last && P.tv_interval > 0.0) {
        const double tv = __dadd_rn(__ldcg(&A.clk->timevar), P.dt);
        diag_due = __dsub_rn(tv, P.tv_interval) > -1e-8;
    }
    const double qt = __dmul_rn(P.q, t_new);
    double dacc[6] = {0, 0, 0, 0, 0, 0};

    // ---- optional record of the stage input (the adjoint's window recompute): CTA 0 of the
    // case copies the mean fields and, in a step's first stage, kx0 and the clock; stable
    // here because the previous stage (and its remap) completed before any CTA started this one
    if (A.rec_mf && cta == 0) {
        const int nmfe = P.nmf * P.nz;
        for (int i = threadIdx.x; i < nmfe; i += blockDim.x) A.rec_mf[i] = ldc(A.mf + i);
        if (A.rec_kx)
            for (int i = threadIdx.x; i < P.nxy; i += blockDim.x) A.rec_kx[i] = __ldcg(A.kx0 + i);
        if (A.rec_t && threadIdx.x == 0) A.rec_t[0] = __ldcg(&A.clk->t);
        if (A.rec_cn && threadIdx.x == 0) {
            A.rec_cn->t_old = __ldcg(&A.clk->t_old);
            A.rec_cn->dtlin_old = __ldcg(&A.clk->dtlin_old);
            A.rec_cn->old_init = __ldcg(&A.clk->old_init);
        }
    }
    // ---- mode loop: one mode per pair of groups, warp-uniform trip count (TMEM access is warp-wide)
    constexpr int PW = SW / 2;  // pairs per warp
    if (tr) A.trace[6] = gtimer();
    const int wglobal = cta * warps + warp;
    const int WG = ncta * warps;
    // The fields (and previous right-hand side) of a mode are contiguous, 64 nz
    // bytes each: one lane per pair requests the pair's next mode into L2 while
    // the current one is transformed, so the stage's loads wait on L2, not DRAM.
    const bool pf_lane = (role == 0 && t == 0);
    const cplx* pf_prev = (A.Fprev && A.sc.has_prev) ? A.Fprev : nullptr;
    const unsigned pf_bytes = 64u * (unsigned)P.nz;
    if (pf_lane && wglobal * PW + pi < P.nxy) {
        l2_prefetch(A.lin_in + (size_t)(wglobal * PW + pi) * 4 * P.nz, pf_bytes);
        if (pf_prev) l2_prefetch(pf_prev + (size_t)(wglobal * PW + pi) * 4 * P.nz, pf_bytes);
    }
    for (int base = wglobal * PW; base < P.nxy; base += WG * PW) {
        const int mode_raw = base + pi;
        const bool valid = mode_raw < P.nxy;
        const int mode = QLGPU_CHECK_INDEX(valid ? mode_raw : P.nxy - 1, P.nxy, &A.clk->status);
        if (pf_lane && mode_raw + WG * PW < P.nxy) {
            l2_prefetch(A.lin_in + (size_t)(mode_raw + WG * PW) * 4 * P.nz, pf_bytes);
            if (pf_prev) l2_prefetch(pf_prev + (size_t)(mode_raw + WG * PW) * 4 * P.nz, pf_bytes);
        }
        const cplx* src = A.lin_in + (size_t)mode * 4 * P.nz;
        const cplx* stg = src;
        if constexpr (STG) {
            stg = stg_buf;
            // stage the mode's 4 nz fields (contiguous, 16-byte aligned) into the pair's buffer:
            // one round trip per mode instead of one per transform and per update chunk
            const int lp = role * G::T + t;  // lane within the pair
            __syncwarp(pmask);               // the previous mode's readers are done
            for (int i = lp; i < 4 * G::nz; i += 2 * G::T) cp_async16(stg_buf + i, src + i);
            cp_async_commit();
            cp_async_wait_all();
            __syncwarp(pmask);
        }
        if (A.rec_lin && valid) {  // record the mode's input fields
            cplx* dst = A.rec_lin + (size_t)mode * 4 * P.nz;
            for (int i = role * G::T + t; i < 4 * G::nz; i += 2 * G::T) dst[i] = ldu<STG>(stg + i);
        }
        if constexpr (MODEL == MODEL_BQLIN)
            bqlin_pair<G, INTEG, Priv, STG>(A, P, TB, mode, valid, role, t, gmask, pmask, xch, ps, pv, tw_s, mfr, tclock,
                                       cn, stg);
        else
            fullqlin_pair<G, INTEG, Priv, STG>(A, P, TB, mode, valid, role, t, gmask, pmask, xch, ps.KU, pv, tw_s, mfr,
                                          tclock, cn, stg);
        if (last && valid && role == 0) {
            // ShearingBox_Remap(q t) after t += dt (main.cpp:122-123, MHD_BQlin.cpp:319-329)
            double kx0 = __ldcg(A.kx0 + mode);
            const double ky = __ldg(A.ky + mode);
            bool zeroed = false;
            if (P.remap) {
                const double kxt = __dadd_rn(kx0, __dmul_rn(qt, ky));
                if (kxt > P.remap_thresh) {
                    zeroed = true;
                    kx0 = __dsub_rn(kx0, P.remap_shift);
                    cplx* uo = A.lin_out + (size_t)mode * 4 * P.nz;
                    __syncwarp(pmask & gmask);
#pragma unroll
                    for (int k2 = 0; k2 < G::P; ++k2) {
                        const int s = stored_index<G>(t + G::T * k2);
                        if (s < 0) continue;
#pragma unroll
                        for (int v = 0; v < 4; ++v) stc(uo + v * P.nz + s, mk(0.0, 0.0));
                    }
                    if (t == 0) A.kx0[mode] = kx0;
                }
            }
            if (A.noise && !zeroed) {
                // Model::DrivingNoise after the step (main.cpp:111-113), before the diagnostics see it
                noise_mode(A.noise, __ldcg(&A.clk->nstep), A.lin_out + (size_t)mode * 4 * P.nz, P.nz, t, G::T,
                           mode, kx0, ky, __ldg(A.kxi + mode), __ldg(A.kyi + mode), P.q, tclock, P.kzL);
                __syncwarp(gmask);
            }
            if (diag_due && !zeroed)
                mode_diag<G>(P, A.lin_out + (size_t)mode * 4 * P.nz, __ldg(A.kxi + mode), __ldg(A.kyi + mode), kx0,
                             ky, t_new, t, dacc);
        }
        __syncwarp();
    }

    // ---- CTA reduction of the stress profiles and diagnostics (fixed order)
    __syncthreads();
    if (tr) A.trace[2] = gtimer();
    if (tr2) A.trace[22] = gtimer();
    double* red = reinterpret_cast<double*>(work);  // [warps][NEMF][NZ] then [blockDim][6]
#pragma unroll
    for (int eb = 0; eb < NEMF / 2; ++eb) {
#pragma unroll
        for (int c4 = 0; c4 < G::P / 4; ++c4) {
            cplx e[4];
            pv.ld4(eb, c4, e);  // PB_E / PF_E, then PF_E2
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                // groups of a warp own the same z set (lane t of each group): sum them in lane order
                double ex = e[i].x, ey = e[i].y;
                double sx = 0.0, sy = 0.0;
#pragma unroll
                for (int g = 0; g < SW; ++g) {
                    sx += __shfl_sync(0xffffffffu, ex, g * G::T + t);
                    sy += __shfl_sync(0xffffffffu, ey, g * G::T + t);
                }
                if (slot == 0) {
                    const int z = zpos<G>(t, 4 * c4 + i);
                    red[(warp * NEMF + 2 * eb + 0) * G::NZ + z] = sx;
                    red[(warp * NEMF + 2 * eb + 1) * G::NZ + z] = sy;
                }
            }
        }
    }
    double* dred = red + (size_t)warps * NEMF * G::NZ;
    if (diag_due) {
        // the diagnostic sums (zero in stages without a record): lanes by a fixed
        // shuffle tree, then warps in order
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            double v = dacc[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if ((tid & 31) == 0) dred[warp * 6 + c] = v;
        }
    }
    if constexpr (USE_TMEM) tmem_fence_before_sync();
    __syncthreads();
    if constexpr (USE_TMEM) tmem_fence_after_sync();
    double* part = A.partials + (size_t)cta * PL;
    for (int idx = tid; idx < NEMF * G::NZ; idx += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < warps; ++w) s += red[w * NEMF * G::NZ + idx];
        part[idx] = s;
    }
    if (tid < 6) {
        double s = 0.0;
        if (diag_due)
            for (int w = 0; w < warps; ++w) s += dred[w * 6 + tid];
        part[NEMF * G::NZ + tid] = s;
    }

    // ---- two-level last-arriver reduction
    __threadfence();
    __syncthreads();
    if (tr) A.trace[3] = gtimer();
    const int ngroups = (ncta + RED_GROUP - 1) / RED_GROUP;
    const int grp = QLGPU_CHECK_INDEX(cta / RED_GROUP, 64, &A.clk->status);  // DevClock::cnt_group
    const int c0 = grp * RED_GROUP;
    const int cn_in = min(RED_GROUP, ncta - c0);
    if (tid == 0) {
        unsigned tk = atomicAdd(&A.clk->cnt_group[grp], 1u);
        ss.last = (tk == (unsigned)(cn_in - 1));
    }
    __syncthreads();
    if (!ss.last) return false;
    __threadfence();
    double* gpart = A.gpartials + (size_t)grp * PL;
    for (int idx = tid; idx < PL; idx += blockDim.x) {
        // CTAs in order; four loads in flight at a time
        double s = 0.0;
        for (int c = 0; c < cn_in; c += 8) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = c + u < cn_in ? __ldcg(A.partials + (size_t)(c0 + c + u) * PL + idx) : 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (c + u < cn_in) s += v[u];
        }
        gpart[idx] = s;
    }
    if (tid == 0) atomicExch(&A.clk->cnt_group[grp], 0u);
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        unsigned tk = atomicAdd(&A.clk->cnt_top, 1u);
        ss.last = (tk == (unsigned)(ngroups - 1));
    }
    __syncthreads();
    if (!ss.last) return false;
    __threadfence();
    for (int idx = tid; idx < PL; idx += blockDim.x) {
        double s = 0.0;
        for (int g = 0; g < ngroups; g += 8) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = g + u < ngroups ? __ldcg(A.gpartials + (size_t)(g + u) * PL + idx) : 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (g + u < ngroups) s += v[u];
        }
        tot[idx] = s;
    }
    if (tid == 0) atomicExch(&A.clk->cnt_top, 0u);
    if (A.trace && tid == 0) A.trace[4] = gtimer();
    __syncthreads();
    mean_field_stage<G, MODEL, INTEG, NEMF>(A, P, tot, spec, xch, tw_s, gidx, ngc, t, gmask, tclock, t_new, last,
                                           diag_due);
    if (A.mfr_cache && !A.rhs_only) {
        // real-space profiles of the updated mean field for the next stage
        __syncthreads();
        mean_profiles<G, MODEL>(P, A.mf, mfr, xch, tw_s, gidx, ngc, t, gmask);
        __syncthreads();
        for (int i = tid; i < SM::NMFR * G::NZ; i += blockDim.x) A.mfr_cache[i] = mfr[i];
        __threadfence();
        __syncthreads();
        if (tid == 0) A.clk->mfr_valid = 1;
    }
    if (A.trace && tid == 0) A.trace[5] = gtimer();
    return true;
}

// One stage launch of a single case: one CTA per SM at most, TMEM allocated
// for the duration of the launch.
// CTA size bound.  A kernel that allocates TMEM runs one CTA per SM, so the
// resident warps of an SM are the warps of one CTA.  Transform groups of P = 8
// points per thread fit 128 registers and run 16-warp CTAs; P = 16 keeps
// 8-warp CTAs with up to 255 registers.
template <int NZ>
struct StageOcc {
    static constexpr int MAX_THREADS = Geom<NZ>::P <= 8 ? 512 : 256;
};

template <int NZ, int MODEL, int INTEG, bool USE_TMEM>
__global__ void __launch_bounds__(StageOcc<NZ>::MAX_THREADS, 1) stage_kernel(StageArgs A, DevParams P) {
    using SM = typename StageKind<NZ, MODEL, USE_TMEM>::SM;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ StageShared ss;
    const int warp = threadIdx.x >> 5;
    const int tcols = SM::tmem_cols(blockDim.x >> 5);
    if constexpr (USE_TMEM) {
        if (warp == 0) tmem_alloc(&ss.tmem, (uint32_t)tcols);
        tmem_fence_before_sync();
        __syncthreads();
        tmem_fence_after_sync();
    }
    stage_body<NZ, MODEL, INTEG, USE_TMEM>(A, P, (int)blockIdx.x, (int)gridDim.x, smem_raw, ss);
    if constexpr (USE_TMEM) {
        tmem_fence_before_sync();
        __syncthreads();
        tmem_fence_after_sync();
        if (warp == 0) tmem_dealloc(ss.tmem, (uint32_t)tcols);
    }
}

// Diagnostics of the current state without stepping (the initial record,
// main.cpp:98-103).  One CTA, fixed-order reduction.
template <int NZ>
__global__ void diag_kernel(const cplx* lin, const cplx* mf, const double* kx0, const double* ky, const int* kxi,
                            const int* kyi, DevParams P, double t, double* out) {
    using G = Geom<NZ>;
    __shared__ double red[1024 * 6 / 8];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int groups = blockDim.x / G::T;
    const int g = threadIdx.x / G::T, tt = threadIdx.x % G::T;
    for (int mode = g; mode < P.nxy; mode += groups)
        mode_diag<G>(P, lin + (size_t)mode * 4 * P.nz, kxi[mode], kyi[mode], kx0[mode], ky[mode], t, tt, acc);
    // reduce: blockDim <= 128 keeps red within 768 doubles
    for (int c = 0; c < 6; ++c) red[threadIdx.x * 6 + c] = acc[c];
    __syncthreads();
    if (threadIdx.x == 0) {
        double ds[6] = {0, 0, 0, 0, 0, 0};
        for (int r = 0; r < (int)blockDim.x; ++r)
            for (int c = 0; c < 6; ++c) ds[c] += red[r * 6 + c];
        const int nzd = P.nz;
        double eMB = 0, aMB = 0, dMB = 0, eMU = 0, aMU = 0, dMU = 0;
        for (int s = 0; s < nzd; ++s) {
            const int kzi = s <= G::H ? s : s - nzd;
            const double kz2 = kz2val(kzval(kzi, P.kzL));
            cplx b0 = mf[s], b1 = mf[nzd + s];
            eMB += (b0.x * b0.x + b0.y * b0.y) + (b1.x * b1.x + b1.y * b1.y);
            aMB += b0.x * b1.x + b0.y * b1.y;
            dMB += -kz2 * (b0.x * b0.x + b0.y * b0.y) - kz2 * (b1.x * b1.x + b1.y * b1.y);
            if (P.nmf == 4) {
                cplx u0 = mf[2 * nzd + s], u1 = mf[3 * nzd + s];
                eMU += (u0.x * u0.x + u0.y * u0.y) + (u1.x * u1.x + u1.y * u1.y);
                aMU += u0.x * u1.x + u0.y * u1.y;
                dMU += -kz2 * (u0.x * u0.x + u0.y * u0.y) - kz2 * (u1.x * u1.x + u1.y * u1.y);
            }
        }
        eMB *= P.divMF; eMU *= P.divMF; aMB *= P.divMF; aMU *= P.divMF;
        dMB *= P.divMF * P.eta; dMU *= P.divMF * P.nu;
        const double eu = ds[0] * P.divfac, eb = ds[1] * P.divfac;
        const double au = ds[2] * P.divfac, abv = ds[3] * P.divfac;
        const double du = ds[4] * P.divfac, db = ds[5] * P.divfac;
        out[0] = t;
        out[1] = eMU / 2; out[2] = eMB / 2; out[3] = eu / 2; out[4] = eb / 2;
        out[5] = aMU; out[6] = aMB; out[7] = au; out[8] = abv;
        out[9] = dMU; out[10] = dMB; out[11] = du; out[12] = db;
        out[13] = pow(P.nu * P.nu * P.nu / (dMU + du), 0.25) * P.kzmax;
        out[14] = pow(P.eta * P.eta * P.eta / (dMB + db), 0.25) * P.kzmax;
    }
}

}  // namespace qlgpu
