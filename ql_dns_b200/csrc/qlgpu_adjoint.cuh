// qlgpu_adjoint.cuh -- discrete adjoint of one RK3CN_Elin or RK3CN stage of
// MHD_BQlin (sm_100a kernels).  No counterpart in the reference.
//
// Forward stage (QL_DNS/Integrators/RK3CN_Elin.cpp:86-177 with
// QL_DNS/Models/MHD_BQlin.cpp:117-284), per mode, with R_f = P(fac f) the
// padded inverse transform and T the truncated forward transform (P^H = T):
//   F_b   = T(i b By R_u)
//   F_zeta= T(-i a dBy R_b + ddBy R_bz + i b By R_eta) + (q - 2 Omega) i c u
//   F_eta = T(-i a dBy R_u + i b By R_zeta - 2 dBy R_{i c uz} - ddBy R_uz) - q i c b
//   F_u   = T(i b By R_b) + ilapF (T(2 a b dBy R_bz) + 2 a b q u + 2 Omega i c zeta)
//   u' = E (n1 F + n2 Fprev + u),   E = exp(linC L)            (RK3CN_Elin.cpp:102-104)
//   u' = D (n1 F + n2 Fprev) + C u,  D = 1/(1 - linC L), C = (1 + linC Lold) D
//                                                              (RK3CN.cpp:105-107, Lold the
//                                                               previous stage's operator)
// and for the mean field G_Bx = EMF_x, G_By = -q Bx + EMF_y with the real
// stress profiles  Ex = sum_modes mult (Re(R_bz R_u*) - Re(R_uz R_b*)),
// Ey = sum_modes mult (Re(R_bz R_uy*) - Re(R_uz R_by*)), EMF = rs_fac i kz T(E)
// (half spectrum mirrored), B' = E_B (n1 G + n2 Gprev + B).
//
// The adjoint of a stage maps (lamU', lamB', lamF_out, lamG_out) to
// (lamU, lamB, lamFprev, lamGprev) with the real inner product
// <x, y> = Re sum conj(x) y:  mu = E lamU', lamF = n1 mu + lamF_out,
// lamU = mu + (dR/dU)^H lamF + (dEMF/dU)^H lamG, lamFprev = n2 mu, and the
// mean-field part likewise (Crank-Nicolson: mu = D lamU' and the direct term
// C lamU' in place of mu).  One CTA per mode: 14 inverse transforms (the nine
// forward real-space fields and five back-propagated rhs fields W = P(lamF)),
// a pointwise pass giving the nine real-space adjoints and the mode's
// contribution to the adjoint of the mean-field profiles, nine forward
// transforms, and the spectral chain back to (u, zeta, b, eta).
#pragma once
#include "qlgpu_debug.cuh"
#include "qlgpu_stage.cuh"

namespace qlgpu {

struct AdjStageArgs {
    const cplx* U;         // stage input fluctuations [nxy][4][nz]
    const cplx* lamU_out;  // adjoint of the stage output
    const cplx* lamF_out;  // adjoint of this stage's rhs from the next stage (null: none)
    cplx* lamU_in;         // adjoint of the stage input (written)
    cplx* lamFp;           // n2 mu: adjoint of the previous stage's rhs (null: first stage)
    const double* kx0;     // unsheared kx of every mode during the step
    const double* ky;
    const int* kxi;
    const int* kyi;
    const double* ilap2;   // [Ny/2][nz]
    const cplx* tw;        // transform twiddles [NZ]
    const double* prof;    // [5][NZ]: By, dBy, ddBy, px, py (real space)
    double* bpart;         // [3][NZ][nxy] per-mode adjoint of the mean-field profiles
    double t_s;            // stage time (when t_dev is null)
    const double* t_dev;   // the step's start time on the device: stage time = *t_dev + sc.t_off
    const CnRec* cn;       // RK3CN: the old-operator fields at the stage start
    int integ;             // INTEG_EXP or INTEG_CN
    int pad;
    int* status;           // the handle's status word (debug-build index checks)
    StageConst sc;
};

template <int NZ>
struct AdjGeom {
    using G = Geom<NZ>;
    static constexpr int NG = 16;  // transform groups per CTA (14 inverse, 9 forward transforms)
    static constexpr int THREADS = NG * G::T;
    static constexpr size_t o_tw = 0;
    static constexpr size_t o_prof = o_tw + sizeof(cplx) * NZ;
    static constexpr size_t o_rw = o_prof + sizeof(double) * 5 * NZ;
    static constexpr size_t o_xch = o_rw + sizeof(cplx) * 14 * NZ;
    static constexpr size_t BYTES = o_xch + sizeof(cplx) * NG * G::XSIZE;
    // E of the four fields at every stored index, [4][nz]: in the exchange buffers of
    // groups 14 and 15, which no transform phase uses (14 inverse, 9 forward transforms)
    static constexpr size_t o_etab = o_xch + sizeof(cplx) * 14 * G::XSIZE;
    static_assert(sizeof(double) * 4 * G::nz <= sizeof(cplx) * 2 * G::XSIZE, "E table fits two exchange buffers");
};

// E = exp(linC L_f) of field f at stored index s (RK3CN_Elin.cpp:102-104), L at the stage
// end; for RK3CN D = 1/(1 - linC L_f) (RK3CN.cpp:105).
__device__ __forceinline__ double adj_efac(const DevParams& P, const StageConst& S, double kxe, double ky, double kz2,
                                           int f, int integ) {
    const double L = linop_f<MODEL_BQLIN>(P, lap_end<MODEL_BQLIN>(P, kxe, ky, kz2), f);
    if (integ == INTEG_CN) return __drcp_rn(__dsub_rn(1.0, __dmul_rn(S.linC, L)));
    return exp(__dmul_rn(S.linC, L));
}

// The stage adjoint of one mode (one CTA).  A may live in parameter space (one
// seed per launch) or in shared memory (a launch over many seeds).
template <int NZ>
__device__ __forceinline__ void adj_modes_body(const AdjStageArgs& A, const DevParams& P, int mode) {
    mode = QLGPU_CHECK_INDEX(mode, P.nxy, A.status);
    using G = Geom<NZ>;
    using AG = AdjGeom<NZ>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* tw_s = reinterpret_cast<cplx*>(smem_raw + AG::o_tw);
    double* prof = reinterpret_cast<double*>(smem_raw + AG::o_prof);
    cplx* RW = reinterpret_cast<cplx*>(smem_raw + AG::o_rw);  // [14][NZ]
    const int tid = threadIdx.x;
    const int g = tid / G::T, t = tid % G::T;
    const int lane = tid & 31;
    const unsigned gmask =
        (G::T == 32 ? 0xffffffffu : (((1u << G::T) - 1u) << ((lane / G::T) * G::T)));
    cplx* xch = reinterpret_cast<cplx*>(smem_raw + AG::o_xch) + (size_t)g * G::XSIZE;
    const int nz = P.nz;
    for (int i = tid; i < NZ; i += blockDim.x) tw_s[i] = A.tw[i];
    for (int i = tid; i < 5 * NZ; i += blockDim.x) prof[i] = A.prof[i];
    const StageConst& S = A.sc;
    const double ky = A.ky[mode];
    const double kx0 = A.kx0[mode];
    const int kyi = A.kyi[mode], kxi = A.kxi[mode];
    const double ts = A.t_dev ? __dadd_rn(*A.t_dev, S.t_off) : A.t_s;
    const double a = kx_at(kx0, P.q, ts, ky);
    const double b = ky;
    const double ab = __dmul_rn(a, b);
    const double kxe = __dadd_rn(a, __dmul_rn(__dmul_rn(P.q, S.dt_lin), ky));
    const double fac = P.fac;
    const double mult = (ky == 0.0) ? 1.0 : 2.0;
    const double Om2 = __dmul_rn(2.0, P.Omega);
    const cplx* u = A.U + (size_t)mode * 4 * nz;
    const cplx* lo = A.lamU_out + (size_t)mode * 4 * nz;
    const cplx* lf = A.lamF_out ? A.lamF_out + (size_t)mode * 4 * nz : nullptr;
    const double* il2row = A.ilap2 + (size_t)kyi * nz;
    double* etab = reinterpret_cast<double*>(smem_raw + AG::o_etab);
    for (int i = tid; i < 4 * nz; i += blockDim.x) {
        const int f = i / nz, s = i % nz;
        const int kzi = s <= G::H ? s : s - nz;
        etab[i] = adj_efac(P, S, kxe, ky, kz2val(kzval(kzi, P.kzL)), f, A.integ);
    }
    // RK3CN: kx where the previous stage's operator was evaluated (RK3CN.cpp:119-122;
    // the init form at the run's start, RK3CN.cpp:57), as the forward stage computes it
    double kxo = 0.0;
    int old_init = 0;
    if (A.integ == INTEG_CN) {
        const double tclock = A.t_dev ? *A.t_dev : __dsub_rn(A.t_s, S.t_off);
        old_init = A.cn->old_init;
        if (old_init) kxo = kx_at(kx0, P.q, tclock, ky);
        else kxo = __dadd_rn(kx_at(kx0, P.q, A.cn->t_old, ky), __dmul_rn(__dmul_rn(P.q, A.cn->dtlin_old), ky));
    }
    __syncthreads();

    // lamF of field f at stored index s: n1 E lamU' + lamF_out
    auto lamF = [&](int f, int s, double) -> cplx {
        cplx r = cscale(lo[f * nz + s], __dmul_rn(S.n1, etab[f * nz + s]));
        if (lf) r = cadd(r, lf[f * nz + s]);
        return r;
    };

    // ---- phase 1: fourteen inverse transforms
    if (g < 14) {
        cplx x[G::P];
#pragma unroll
        for (int k2 = 0; k2 < G::P; ++k2) {
            const int k = t + G::T * k2;
            const int s = stored_index<G>(k);
            cplx v = mk(0.0, 0.0);
            if (s >= 0) {
                const double c = kzval(kz_int<G>(k), P.kzL);
                const double kz2 = kz2val(c);
                const bool z0 = (kyi == 0 && s == 0);
                const double il2 = il2row[s];
                if (g < 4) {
                    v = cscale(u[g * nz + s], fac);  // R_u, R_zeta, R_b, R_eta
                } else if (g < 9) {
                    const int f0 = (g == 5 || g == 8) ? 2 : 0;
                    const cplx g0 = u[f0 * nz + s], g1 = u[(f0 + 1) * nz + s];
                    if (g == 7 || g == 8) {
                        v = cscale(cadd(cscale(g0, ab), imul(g1, c)), il2);  // uy, by
                    } else {
                        v = cscale(csub(cscale(g0, __dmul_rn(a, c)), imul(g1, b)), il2);  // uz, bz
                        if (g == 6) v = imul(v, c);                                        // i c uz
                    }
                    v = cscale(v, fac);
                } else if (g == 9) {
                    v = lamF(2, s, kz2);  // W_b
                } else if (g == 10) {
                    v = lamF(1, s, kz2);  // W_zeta
                } else if (g == 11) {
                    v = lamF(3, s, kz2);  // W_eta
                } else {
                    v = lamF(0, s, kz2);  // W_S, W_u2 = P(ilapF lamF_u)
                    if (g == 13) {
                        const double lapF = __dadd_rn(-__dmul_rn(a, a), lap2val(ky, kz2, z0));
                        const double ilapF = (z0 && kxi == 0) ? 1.0 : __drcp_rn(lapF);
                        v = cscale(v, ilapF);
                    }
                }
            }
            x[k2] = v;
        }
        inv_fft<G>(x, xch, tw_s, t, gmask);
#pragma unroll
        for (int j = 0; j < G::P; ++j) RW[g * NZ + zpos<G>(t, j)] = x[j];
    }
    __syncthreads();

    // ---- phase 2: pointwise adjoints in real space (in place: slots 0..8 become lamR)
    const double* By = prof;
    const double* dBy = prof + NZ;
    const double* ddBy = prof + 2 * NZ;
    const double* px = prof + 3 * NZ;
    const double* py = prof + 4 * NZ;
    // lamR = sum of conj(multiplier) W over the terms a field enters (reads slots 0..13 at z)
    auto lam_r = [&](int z, cplx* o) {
        const cplx Ru = RW[0 * NZ + z], Rb = RW[2 * NZ + z];
        const cplx Ruz = RW[4 * NZ + z], Rbz = RW[5 * NZ + z];
        const cplx Ruy = RW[7 * NZ + z], Rby = RW[8 * NZ + z];
        const cplx Wb = RW[9 * NZ + z], Wz = RW[10 * NZ + z], We = RW[11 * NZ + z];
        const cplx WS = RW[12 * NZ + z], Wu2 = RW[13 * NZ + z];
        const double by = By[z], dby = dBy[z], ddby = ddBy[z];
        const double mx = mult * px[z], my = mult * py[z];
        const double bBy = b * by, adBy = a * dby;
        o[0] = cadd(cadd(imul(Wb, -bBy), imul(We, adBy)), cscale(Rbz, mx));
        o[1] = imul(We, -bBy);
        o[2] = csub(cadd(imul(Wz, adBy), imul(WS, -bBy)), cscale(Ruz, mx));
        o[3] = imul(Wz, -bBy);
        o[4] = csub(csub(cscale(We, -ddby), cscale(Rb, mx)), cscale(Rby, my));
        o[5] = cadd(cadd(cscale(Wz, ddby), cscale(Wu2, 2.0 * ab * dby)), cadd(cscale(Ru, mx), cscale(Ruy, my)));
        o[6] = cscale(We, -2.0 * dby);
        o[7] = cscale(Rbz, my);
        o[8] = cscale(Ruz, -my);
    };
    // adjoint of the mean-field profiles at z: Re(conj(multiplier * R) W) per term
    auto prof_adj = [&](int z) {
        const cplx Ru = RW[0 * NZ + z], Rz = RW[1 * NZ + z], Rb = RW[2 * NZ + z], Re_ = RW[3 * NZ + z];
        const cplx Ruz = RW[4 * NZ + z], Rbz = RW[5 * NZ + z], Rik = RW[6 * NZ + z];
        const cplx Wb = RW[9 * NZ + z], Wz = RW[10 * NZ + z], We = RW[11 * NZ + z];
        const cplx WS = RW[12 * NZ + z], Wu2 = RW[13 * NZ + z];
        auto re_cw = [](cplx r, cplx w) { return r.x * w.x + r.y * w.y; };  // Re(conj(r) w)
        auto re_icw = [](cplx r, cplx w) { return r.y * w.x - r.x * w.y; };  // Re(i conj(r) w)
        const double pBy = -b * (re_icw(Ru, Wb) + re_icw(Re_, Wz) + re_icw(Rz, We) + re_icw(Rb, WS));
        const double pdBy = a * (re_icw(Rb, Wz) + re_icw(Ru, We)) - 2.0 * re_cw(Rik, We) + 2.0 * ab * re_cw(Rbz, Wu2);
        const double pddBy = re_cw(Rbz, Wz) - re_cw(Ruz, We);
        const size_t nxy = (size_t)P.nxy;
        A.bpart[(0 * (size_t)NZ + z) * nxy + mode] = pBy;
        A.bpart[(1 * (size_t)NZ + z) * nxy + mode] = pdBy;
        A.bpart[(2 * (size_t)NZ + z) * nxy + mode] = pddBy;
    };
    if constexpr (AG::THREADS >= 2 * NZ) {
        // two threads per z: lamR in the first NZ threads, the profile adjoints in the
        // next NZ; slots 0..8 are overwritten only after both have read them
        const int z = tid % NZ, part = tid / NZ;
        cplx o[9];
        if (part == 0) lam_r(z, o);
        else if (part == 1) prof_adj(z);
        __syncthreads();
        if (part == 0) {
#pragma unroll
            for (int k = 0; k < 9; ++k) RW[k * NZ + z] = o[k];
        }
    } else {
        for (int z = tid; z < NZ; z += blockDim.x) {
            cplx o[9];
            lam_r(z, o);
            prof_adj(z);
#pragma unroll
            for (int k = 0; k < 9; ++k) RW[k * NZ + z] = o[k];
        }
    }
    __syncthreads();

    // ---- phase 3: nine forward transforms, spectral results back into slots 0..8
    if (g < 9) {
        cplx x[G::P];
#pragma unroll
        for (int j = 0; j < G::P; ++j) x[j] = RW[g * NZ + zpos<G>(t, j)];
        fwd_fft<G>(x, xch, tw_s, t, gmask);
#pragma unroll
        for (int k2 = 0; k2 < G::P; ++k2) {
            const int s = stored_index<G>(t + G::T * k2);
            if (s >= 0) RW[g * NZ + s] = x[k2];
        }
    }
    __syncthreads();

    // ---- phase 4: spectral chain to (u, zeta, b, eta), linear terms, RK adjoint
    for (int idx = tid; idx < 4 * nz; idx += blockDim.x) {
        const int f = idx / nz, s = idx % nz;
        const int kzi = s <= G::H ? s : s - nz;
        const double c = kzval(kzi, P.kzL);
        const double kz2 = kz2val(c);
        const bool z0 = (kyi == 0 && s == 0);
        const double il2 = il2row[s];
        const cplx mu = cscale(lo[f * nz + s], etab[idx]);
        cplx r = mu;
        if (A.integ == INTEG_CN) {
            // the direct term (1 + linC Lold) D lamU' (RK3CN.cpp:107)
            const double lo_lap = old_init ? lap_init<MODEL_BQLIN>(P, kxo, lap2val(ky, kz2, z0))
                                           : lap_end<MODEL_BQLIN>(P, kxo, ky, kz2);
            const double Lold = linop_f<MODEL_BQLIN>(P, lo_lap, f);
            r = cscale(mu, __dadd_rn(1.0, __dmul_rn(S.linC, Lold)));
        }
        if (f == 0 || f == 1) {
            // uz = (a c u - i b zeta) il2, i c uz, uy = (a b u + i c zeta) il2
            const cplx luz = cscale(csub(RW[4 * NZ + s], imul(RW[6 * NZ + s], c)), fac);
            const cplx luy = cscale(RW[7 * NZ + s], fac);
            if (f == 0) {
                r = cadd(r, cscale(RW[0 * NZ + s], fac));
                r = cadd(r, cscale(luz, __dmul_rn(a, c) * il2));
                r = cadd(r, cscale(luy, ab * il2));
                // linear terms of F_zeta ((q - 2 Omega) i c u) and F_u (ilapF 2 a b q u)
                r = cadd(r, imul(lamF(1, s, kz2), -(P.q - Om2) * c));
                const double lapF = __dadd_rn(-__dmul_rn(a, a), lap2val(ky, kz2, z0));
                const double ilapF = (z0 && kxi == 0) ? 1.0 : __drcp_rn(lapF);
                r = cadd(r, cscale(lamF(0, s, kz2), ilapF * 2.0 * ab * P.q));
            } else {
                r = cadd(r, cscale(RW[1 * NZ + s], fac));
                r = cadd(r, imul(luz, b * il2));
                r = cadd(r, imul(luy, -c * il2));
                // linear term of F_u: ilapF 2 Omega i c zeta
                const double lapF = __dadd_rn(-__dmul_rn(a, a), lap2val(ky, kz2, z0));
                const double ilapF = (z0 && kxi == 0) ? 1.0 : __drcp_rn(lapF);
                r = cadd(r, imul(lamF(0, s, kz2), -Om2 * c * ilapF));
            }
        } else {
            const cplx lbz = cscale(RW[5 * NZ + s], fac);
            const cplx lby = cscale(RW[8 * NZ + s], fac);
            if (f == 2) {
                r = cadd(r, cscale(RW[2 * NZ + s], fac));
                r = cadd(r, cscale(lbz, __dmul_rn(a, c) * il2));
                r = cadd(r, cscale(lby, ab * il2));
                r = cadd(r, imul(lamF(3, s, kz2), P.q * c));  // linear term of F_eta: -q i c b
            } else {
                r = cadd(r, cscale(RW[3 * NZ + s], fac));
                r = cadd(r, imul(lbz, b * il2));
                r = cadd(r, imul(lby, -c * il2));
            }
        }
        A.lamU_in[(size_t)mode * 4 * nz + f * nz + s] = r;
        if (A.lamFp) A.lamFp[(size_t)mode * 4 * nz + f * nz + s] = cscale(mu, S.n2);
    }
}

template <int NZ>
__global__ void __launch_bounds__(AdjGeom<NZ>::THREADS, 6)
    adj_modes_kernel(const __grid_constant__ AdjStageArgs A, const __grid_constant__ DevParams P) {
    adj_modes_body<NZ>(A, P, blockIdx.x);
}

// ---- the reverse sweep of many seeds at once (same dimensions and parameters):
// every kernel of a reverse step runs once for all seeds, seed = blockIdx.y.
// The per-seed buffers are read from a device table; the position in the sweep
// (step n of a window of `steps`, stage s, buffer parity) is a launch argument.
struct AdjSeedBufs {
    const CnRec* cn_pre;   // [C][3] RK3CN old-operator fields at every stage start (null: RK3CN_Elin)
    const cplx* stU;       // [C][3] recorded stage inputs
    const cplx* stB;       // [C][3] recorded stage mean fields
    const cplx* postU;     // the window's end state
    const double* kx_pre;  // [C] kx0 at every step start
    const double* kx_post; // kx0 at the window end
    const double* t_pre;   // [C + 1] step start times
    cplx* lamU[2];
    cplx* lamB[2];
    cplx* lamF[2];
    cplx* lamG[2];
    double* prof;
    double* bpart;
    double* bsum;
};

struct AdjRevPos {
    const AdjSeedBufs* seeds;
    int n, steps, s;
    int par;  // stages already reversed, mod 2: lamU[par] is the current adjoint state
    long long nlin, nmfe, nxy;
    double weight;  // of AM_b in J
};

// the post-step state of step n and its kx0 (the window end for the last step)
__device__ __forceinline__ const cplx* adj_upost(const AdjSeedBufs& B, const AdjRevPos& X) {
    return X.n + 1 < X.steps ? B.stU + (size_t)(X.n + 1) * 3 * X.nlin : B.postU;
}
__device__ __forceinline__ const double* adj_kxpost(const AdjSeedBufs& B, const AdjRevPos& X) {
    return X.n + 1 < X.steps ? B.kx_pre + (size_t)(X.n + 1) * X.nxy : B.kx_post;
}

template <int NZ>
__global__ void __launch_bounds__(AdjGeom<NZ>::THREADS, 6)
    adj_modes_seeds_kernel(const __grid_constant__ AdjStageArgs base, const __grid_constant__ DevParams P,
                           const __grid_constant__ AdjRevPos X) {
    __shared__ __align__(16) AdjStageArgs sA;
    if (threadIdx.x == 0) {
        const AdjSeedBufs& B = X.seeds[blockIdx.y];
        const int p = X.par;
        sA = base;
        sA.U = B.stU + ((size_t)X.n * 3 + X.s) * X.nlin;
        sA.lamU_out = B.lamU[p];
        sA.lamF_out = X.s == 2 ? nullptr : B.lamF[p];
        sA.lamU_in = B.lamU[p ^ 1];
        sA.lamFp = X.s == 0 ? nullptr : B.lamF[p ^ 1];
        sA.kx0 = B.kx_pre + (size_t)X.n * X.nxy;
        sA.prof = B.prof;
        sA.bpart = B.bpart;
        sA.t_dev = B.t_pre + X.n;
        sA.cn = B.cn_pre ? B.cn_pre + (size_t)X.n * 3 + X.s : nullptr;
    }
    __syncthreads();
    adj_modes_body<NZ>(sA, P, blockIdx.x);
}

// Mean-field part before the mode pass: forward profiles of the stage input
// mean field (By, dBy, ddBy; MHD_BQlin.cpp:122-127), the adjoint stress
// profiles px, py, and the RK / mean-field-rhs adjoint of B:
//   muB = E_B lamB', lamG = n1 muB + lamG_out, lamB = muB - q lamG_y e_x,
//   lamGp = n2 muB,  p(z) = Re sum_{s=1..H} h_s e^{+i k_s z},
//   h_s = rs_fac (-i kz_s) (lamEMF[s] + conj(lamEMF[nz-s])).
// One CTA of 5 transform groups.
struct AdjMfArgs {
    const cplx* B;         // stage input mean field [nmf][nz]
    const cplx* lamB_out;  // adjoint of the stage output mean field
    const cplx* lamG_out;  // adjoint of this stage's mean-field rhs from the next stage (null: none)
    cplx* lamB_in;         // partial adjoint of the stage input mean field (the mode pass adds to By)
    cplx* lamGp;           // n2 muB (null: first stage)
    double* prof;          // [5][NZ] out
    const cplx* tw;
    int integ;             // INTEG_EXP or INTEG_CN
    int pad;
    StageConst sc;
};

template <int NZ>
__device__ __forceinline__ void adj_mf_pre_body(const AdjMfArgs& A, const DevParams& P) {
    using G = Geom<NZ>;
    __shared__ __align__(16) cplx tw_s[NZ];
    __shared__ __align__(16) cplx lamG[2][G::nz];
    __shared__ __align__(16) cplx xchs[5][G::XSIZE];
    const int tid = threadIdx.x;
    const int nz = P.nz;
    const StageConst& S = A.sc;
    for (int i = tid; i < NZ; i += blockDim.x) tw_s[i] = A.tw[i];
    for (int i = tid; i < 2 * nz; i += blockDim.x) {
        const int m = i / nz, s = i % nz;
        const int kzi = s <= G::H ? s : s - nz;
        const double kz2 = kz2val(kzval(kzi, P.kzL));
        const double Lm = P.ql ? __dmul_rn(P.eta, kz2) : 0.0;
        // exp(linC Lm), or D = 1/(1 - linC Lm) and the direct term (1 + linC Lm) D for RK3CN
        const double e = A.integ == INTEG_CN ? __drcp_rn(__dsub_rn(1.0, __dmul_rn(S.linC, Lm)))
                                             : exp(__dmul_rn(S.linC, Lm));
        const cplx muB = cscale(A.lamB_out[m * nz + s], e);
        cplx lg = cscale(muB, S.n1);
        if (A.lamG_out) lg = cadd(lg, A.lamG_out[m * nz + s]);
        lamG[m][s] = lg;
        if (A.lamGp) A.lamGp[m * nz + s] = cscale(muB, S.n2);
        A.lamB_in[m * nz + s] =
            A.integ == INTEG_CN ? cscale(muB, __dadd_rn(1.0, __dmul_rn(S.linC, Lm))) : muB;
    }
    __syncthreads();
    if (tid < 2 * nz && P.ql) {
        // G_By = -q Bx + EMF_y (MHD_BQlin.cpp:274-276)
        if (tid < nz) A.lamB_in[tid] = csub(A.lamB_in[tid], cscale(lamG[1][tid], P.q));
    }
    const int g = tid / G::T, t = tid % G::T, lane = tid & 31;
    const unsigned gmask = (G::T == 32 ? 0xffffffffu : (((1u << G::T) - 1u) << ((lane / G::T) * G::T)));
    if (g < 5) {
        cplx x[G::P];
#pragma unroll
        for (int k2 = 0; k2 < G::P; ++k2) {
            const int k = t + G::T * k2;
            const int s = stored_index<G>(k);
            cplx v = mk(0.0, 0.0);
            if (s >= 0) {
                const double c = kzval(kz_int<G>(k), P.kzL);
                if (g < 3) {
                    v = cscale(A.B[1 * nz + s], P.fac);
                    if (g == 1) v = imul(v, c);
                    if (g == 2) v = cscale(v, kz2val(c));
                } else if (P.ql && s >= 1 && s <= G::H) {
                    const cplx l = lamG[g - 3][s], lm = conjc(lamG[g - 3][nz - s]);
                    v = imul(cadd(l, lm), -c * P.rs_fac);
                }
            }
            x[k2] = v;
        }
        inv_fft<G>(x, xchs[g], tw_s, t, gmask);
#pragma unroll
        for (int j = 0; j < G::P; ++j) A.prof[g * NZ + zpos<G>(t, j)] = x[j].x;
    }
}

template <int NZ>
__global__ void adj_mf_pre_kernel(const __grid_constant__ AdjMfArgs A, const __grid_constant__ DevParams P) {
    adj_mf_pre_body<NZ>(A, P);
}

template <int NZ>
__global__ void adj_mf_pre_seeds_kernel(const __grid_constant__ AdjMfArgs base, const __grid_constant__ DevParams P,
                                        const __grid_constant__ AdjRevPos X) {
    __shared__ __align__(16) AdjMfArgs sM;
    if (threadIdx.x == 0) {
        const AdjSeedBufs& B = X.seeds[blockIdx.y];
        const int p = X.par;
        sM = base;
        sM.B = B.stB + ((size_t)X.n * 3 + X.s) * X.nmfe;
        sM.lamB_out = B.lamB[p];
        sM.lamG_out = X.s == 2 ? nullptr : B.lamG[p];
        sM.lamB_in = B.lamB[p ^ 1];
        sM.lamGp = X.s == 0 ? nullptr : B.lamG[p ^ 1];
        sM.prof = B.prof;
    }
    __syncthreads();
    adj_mf_pre_body<NZ>(sM, P);
}

// Sum of the per-mode profile adjoints over modes, one warp per (profile, z),
// fixed order (lane-strided partial sums, then a shuffle tree).
__device__ __forceinline__ void adj_bsum_body(const double* bpart, int nxy, int n_out, double* bsum) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n_out) return;
    const double* row = bpart + (size_t)w * nxy;
    double s = 0.0;
    for (int m = lane; m < nxy; m += 32) s += row[m];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) bsum[w] = s;
}

__global__ void adj_bsum_kernel(const double* bpart, int nxy, int n_out, double* bsum) {
    adj_bsum_body(bpart, nxy, n_out, bsum);
}

__global__ void adj_bsum_seeds_kernel(const __grid_constant__ AdjRevPos X, int n_out) {
    const AdjSeedBufs& B = X.seeds[blockIdx.y];
    adj_bsum_body(B.bpart, (int)X.nxy, n_out, B.bsum);
}

// lamB_y += fac (T(pBy) - i c T(pdBy) - c^2 T(pddBy)): the adjoint of the
// mean-field profiles of the stage (MHD_BQlin.cpp:122-127).  One CTA.
template <int NZ>
__device__ __forceinline__ void adj_mf_post_body(const double* bsum, const cplx* tw, const DevParams& P,
                                                 cplx* lamB_in) {
    using G = Geom<NZ>;
    __shared__ __align__(16) cplx tw_s[NZ];
    __shared__ __align__(16) cplx xchs[3][G::XSIZE];
    __shared__ __align__(16) cplx spec[3][NZ];
    const int tid = threadIdx.x;
    for (int i = tid; i < NZ; i += blockDim.x) tw_s[i] = tw[i];
    __syncthreads();
    const int g = tid / G::T, t = tid % G::T, lane = tid & 31;
    const unsigned gmask = (G::T == 32 ? 0xffffffffu : (((1u << G::T) - 1u) << ((lane / G::T) * G::T)));
    if (g < 3) {
        cplx x[G::P];
#pragma unroll
        for (int j = 0; j < G::P; ++j) x[j] = mk(bsum[g * NZ + zpos<G>(t, j)], 0.0);
        fwd_fft<G>(x, xchs[g], tw_s, t, gmask);
#pragma unroll
        for (int k2 = 0; k2 < G::P; ++k2) spec[g][t + G::T * k2] = x[k2];
    }
    __syncthreads();
    const int nz = P.nz;
    for (int s = tid; s < nz; s += blockDim.x) {
        const int k = s <= G::H ? s : s + (NZ - nz);
        const int kzi = s <= G::H ? s : s - nz;
        const double c = kzval(kzi, P.kzL);
        cplx v = cadd(cadd(spec[0][k], imul(spec[1][k], -c)), cscale(spec[2][k], kz2val(c)));
        lamB_in[nz + s] = cadd(lamB_in[nz + s], cscale(v, P.fac));
    }
}

template <int NZ>
__global__ void adj_mf_post_kernel(const double* bsum, const cplx* tw, const __grid_constant__ DevParams P,
                                   cplx* lamB_in) {
    adj_mf_post_body<NZ>(bsum, tw, P, lamB_in);
}

template <int NZ>
__global__ void adj_mf_post_seeds_kernel(const cplx* tw, const __grid_constant__ DevParams P,
                                         const __grid_constant__ AdjRevPos X) {
    const AdjSeedBufs& B = X.seeds[blockIdx.y];
    adj_mf_post_body<NZ>(B.bsum, tw, P, B.lamB[X.par ^ 1]);
}

// Gradient of (weight) * AM_b at a post-step state (MHD_BQlin.cpp:388-392,424):
// AM_b = divfac sum mult Re(b conj(by)), by = (a b_y b + i c eta) il2 gives
// d/db = 2 a b_y il2 b + i c il2 eta, d/deta = -i c il2 b.  Adds to lamU.
template <int NZ>
__device__ __forceinline__ void adj_jgrad_body(const cplx* U, const double* kx0, const double* ky, const int* kyi,
                                               const double* ilap2, const DevParams& P, double t_host,
                                               const double* t_dev, double weight, cplx* lamU) {
    using G = Geom<NZ>;
    const int nz = P.nz;
    const double t = t_dev ? *t_dev : t_host;
    const size_t n = (size_t)P.nxy * nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int mode = (int)(i / nz), s = (int)(i % nz);
        const double kyv = ky[mode];
        const double a = kx_at(kx0[mode], P.q, t, kyv);
        const double ab = __dmul_rn(a, kyv);
        const int kzi = s <= G::H ? s : s - nz;
        const double c = kzval(kzi, P.kzL);
        const double il2 = ilap2[(size_t)kyi[mode] * nz + s];
        const double w = weight * P.divfac * (kyv == 0.0 ? 1.0 : 2.0);
        const cplx* u = U + (size_t)mode * 4 * nz;
        const cplx bb = u[2 * nz + s], ee = u[3 * nz + s];
        cplx* l = lamU + (size_t)mode * 4 * nz;
        const cplx gb = cadd(cscale(bb, 2.0 * ab * il2), imul(ee, c * il2));
        const cplx ge = imul(bb, -c * il2);
        l[2 * nz + s] = cadd(l[2 * nz + s], cscale(gb, w));
        l[3 * nz + s] = cadd(l[3 * nz + s], cscale(ge, w));
    }
}

template <int NZ>
__global__ void adj_jgrad_kernel(const cplx* U, const double* kx0, const double* ky, const int* kyi,
                                 const double* ilap2, const __grid_constant__ DevParams P, double t_host,
                                 const double* t_dev, double weight, cplx* lamU) {
    adj_jgrad_body<NZ>(U, kx0, ky, kyi, ilap2, P, t_host, t_dev, weight, lamU);
}

// J's gradient at the post-step state of step n (seed = blockIdx.y)
template <int NZ>
__global__ void adj_jgrad_seeds_kernel(const double* ky, const int* kyi, const double* ilap2,
                                       const __grid_constant__ DevParams P, const __grid_constant__ AdjRevPos X) {
    const AdjSeedBufs& B = X.seeds[blockIdx.y];
    adj_jgrad_body<NZ>(adj_upost(B, X), adj_kxpost(B, X), ky, kyi, ilap2, P, 0.0, B.t_pre + X.n + 1, X.weight,
                       B.lamU[X.par]);
}

// Adjoint of the shearing-box remap (MHD_BQlin.cpp:319-329): the fields of a
// remapped mode were set to zero, so their adjoint is zero.
__device__ __forceinline__ void adj_remap_body(const double* kx0_before, const double* kx0_after, int nxy, int nz,
                                               cplx* lamU) {
    const size_t n = (size_t)nxy * 4 * nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int mode = (int)(i / (4 * (size_t)nz));
        if (kx0_before[mode] != kx0_after[mode]) lamU[i] = mk(0.0, 0.0);
    }
}

__global__ void adj_remap_kernel(const double* kx0_before, const double* kx0_after, int nxy, int nz, cplx* lamU) {
    adj_remap_body(kx0_before, kx0_after, nxy, nz, lamU);
}

__global__ void adj_remap_seeds_kernel(const __grid_constant__ AdjRevPos X, int nz) {
    const AdjSeedBufs& B = X.seeds[blockIdx.y];
    adj_remap_body(B.kx_pre + (size_t)X.n * X.nxy, adj_kxpost(B, X), (int)X.nxy, nz, B.lamU[X.par]);
}

}  // namespace qlgpu
