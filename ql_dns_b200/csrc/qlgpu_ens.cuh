// qlgpu_ens.cuh -- the chunk-queue engine of the batched ensemble (sm_100a):
// MHD_BQlin with RK3CN_Elin or RK3CN, NZ = 16, 32, 64 or 128, many cases in
// one persistent launch.
//
// Work unit.  A chunk is a run of consecutive (kx,ky) modes of one case for
// one RK3 stage.  The host lists every case's chunks of one stage in a fixed
// order (a "round"); the launch walks 3 K rounds.  A CTA takes the next
// ticket from one global counter, waits (bounded) until its case has
// finished the previous stage, runs the chunk, writes the chunk's partial
// stress / diagnostic sums into the chunk's own slot and counts the chunk
// done.  The CTA that completes a case's stage sums the chunk slots in slot
// order (so the result does not depend on which CTA ran which chunk), runs the
// case's mean-field stage and releases the next stage of that case.  No CTA
// ever waits for a whole stage of every case: while one case finishes its
// mean-field stage the others keep every SM busy.
//
// Transforms.  Every z-transform has 8 points per thread: a group of T = NZ/8
// threads holds one length-NZ column, thread t register r holding index
// t + T r in spectral AND in real space.  One routine (xform) computes the
// backward (FFTW_BACKWARD, fftwPlans.cpp:48-51) transform; the forward one is
// conj(xform(conj(x))), and the conjugations are folded into the pointwise
// code around it.  A transform is one register DFT-8, a twiddle, one
// shared-memory exchange and 8/T register DFT-T (T = 16: a radix-2 step on the
// exchanged values and a DFT-8).
//
// Per mode (MHD_BQlin::rhs, QL_DNS/Models/MHD_BQlin.cpp:135-257, fused with
// the stage update of RK3CN_Elin.cpp:102-104 / RK3CN.cpp:105-107): a PAIR of
// groups, role U (velocity side) and role B (magnetic side), runs seven
// transform slots, 14 transforms per mode (the reference does 22):
//
//   slot  U                                     B
//   1 inv R_uz -> KU                            R_bz -> KB
//   2 inv R_u : Ex += Re(KB R_u*)               R_b : Ex -= Re(KU R_b*)
//         acc = -i kx dBy R_u                   acc = -i kx dBy R_b + ddBy KB
//         x = i ky By R_u                       x = i ky By R_b
//   3 fwd x -> F_b (update b)                   x -> S
//   4 inv R_zeta : acc += i ky By R_zeta        R_eta : acc += i ky By R_eta
//   5 inv R_{i kz uz} :                         R_by : Ey -= Re(KU R_by*)
//         acc += -2 dBy R - ddBy KU
//   6 fwd acc -> F_eta (update eta)             acc -> F_zeta (update zeta)
//   7 inv R_uy : Ey += Re(KB R_uy*)             fwd 2 kx ky dBy KB -> F_u = S + ilapF(...)
//
// Slot 7 is an inverse transform in U and a forward one in B: both run the
// same routine.  The stress accumulators Ex, Ey, the held spectrum S and the
// previous right-hand sides live in tensor memory (TMEM) as a per-lane
// scratchpad, so a thread holds only the transform in flight and one
// accumulator in registers.
#pragma once
#include <cstdint>
#include <type_traits>

#include "qlgpu_batch.cuh"
#include "qlgpu_debug.cuh"

namespace qlgpu {
namespace ens {

// 12 warps (3 per scheduler, up to 168 registers) measured 7 % faster than 16 at 128
// registers: fewer spills, and the smaller shared-memory footprint leaves more L1
constexpr int WARPS = 12;
constexpr int THREADS = 32 * WARPS;
// TMEM columns of one lane: Ex (8 doubles), Ey (8 doubles), S (8 complex), acc (8 complex), the
// previous right-hand sides of the two fields the lane updates (8 complex each)
constexpr int TM_EX = 0, TM_EY = 16, TM_S = 32, TM_ACC = 64, TM_FPA = 96, TM_FPB = 128;
constexpr int COLS_PER_WARP = 160;
constexpr int CTAS_PER_SM = 1;  // resident CTAs per SM (their TMEM allocations share the SM's 512 columns)
// TMEM columns per CTA: a power of two >= COLS_PER_WARP * ceil(WARPS / 4) (warps w, w+4, ... share lane
// quarter w%4), at most 512 / CTAS_PER_SM
constexpr int TCOLS = COLS_PER_WARP * ((WARPS + 3) / 4) <= 128 ? 128 : COLS_PER_WARP * ((WARPS + 3) / 4) <= 256 ? 256 : 512;
static_assert(TCOLS * CTAS_PER_SM <= 512, "TMEM columns of the resident CTAs");
static_assert(COLS_PER_WARP * ((WARPS + 3) / 4) <= TCOLS, "TMEM columns of the warps sharing a lane quarter");
constexpr int NEMF = 2;                                  // stress profiles Ex, Ey
constexpr int MAX_PAIRS_PER_WARP = 8;                    // NZ = 16

// Geometry of one NZ class.
template <int NZ_>
struct EG {
    static constexpr int NZ = NZ_;
    static constexpr int T = NZ_ / 8;                 // threads per group (8 points each)
    static constexpr int nz = 1 + 2 * (NZ_ / 3);      // Model.h:34
    static constexpr int H = (nz - 1) / 2;
    static constexpr int GPW = 32 / T;                // groups per warp
    static constexpr int PPW = GPW / 2;               // pairs (modes) per warp
    static constexpr int SWZ = T == 4 ? 1 : (T == 2 ? 3 : 0);  // row swizzle of small groups
    static constexpr int PL = NEMF * NZ_ + 8;         // partial vector (doubles)
    static_assert(8 * T == NZ_ && T >= 2 && T <= 16, "NZ = 16, 32, 64 or 128");
    // dynamic shared memory (bytes): tables, then one region per warp
    static constexpr int NZE = (nz + 1) & ~1;
    static constexpr size_t o_tw = 0;                                        // [8][T] cplx
    static constexpr size_t o_prof = o_tw + 16 * (size_t)NZ_;               // By, dBy, ddBy [3][NZ]
    static constexpr size_t o_kz = o_prof + 8 * 3 * (size_t)NZ_;            // kz value per spectral slot
    static constexpr size_t o_ekz = o_kz + 8 * (size_t)NZ_;                 // [2][NZE] integrating factors
    static constexpr size_t o_warp = o_ekz + 8 * 2 * (size_t)NZE;
    // per pair KU, then KB shifted by T slots: for T <= 4 the two roles of a pair share a quarter
    // warp, and without the shift their K accesses fall on the same banks
    static constexpr int KPAIR = 2 * NZ_ + T;
    static constexpr size_t K_CPLX = (size_t)PPW * KPAIR;                    // per warp: KU, KB of its pairs
    static constexpr size_t STG_CPLX = (size_t)PPW * 4 * nz;                 // staged mode fields
    static constexpr size_t X_CPLX = (size_t)GPW * 8 * T;                    // exchange buffers
    static constexpr size_t X_OFF = K_CPLX + STG_CPLX;                        // per warp: [K | STG | X]
    static constexpr size_t WARP_BYTES = 16 * (X_OFF + X_CPLX);
    static constexpr size_t BYTES = o_warp + WARPS * WARP_BYTES;
};

// Real-space / spectral register classes: index t + T r is in the dealiasing
// gap for every t (dead), stored for every t, or stored for some t.
template <class E>
__device__ __forceinline__ int sidx(int t, int r) {
    const int k = t + E::T * r;
    if (k <= E::H) return k;
    if (k >= E::NZ - E::H) return k - (E::NZ - E::nz);
    return -1;
}
template <class E>
__host__ __device__ constexpr bool rdead(int r) {
    return E::T * r > E::H && E::T * r + E::T - 1 < E::NZ - E::H;
}

// cos / sin (2 pi i / 16)
__device__ __forceinline__ constexpr double c16(int i) {
    return i == 0 ? 1.0 : i == 1 ? QLGPU_C1 : i == 2 ? QLGPU_RSQRT2 : i == 3 ? QLGPU_S1 : i == 4 ? 0.0
         : i == 5 ? -QLGPU_S1 : i == 6 ? -QLGPU_RSQRT2 : -QLGPU_C1;
}
__device__ __forceinline__ constexpr double s16(int i) {
    return i == 0 ? 0.0 : i == 1 ? QLGPU_S1 : i == 2 ? QLGPU_RSQRT2 : i == 3 ? QLGPU_C1 : i == 4 ? 1.0
         : i == 5 ? QLGPU_C1 : i == 6 ? QLGPU_RSQRT2 : QLGPU_S1;
}

// Exchange-buffer slot of (row q, column t) in group g's buffer (cplx units).
template <class E>
__device__ __forceinline__ int xslot(int g, int q, int t) {
    return g * 8 * E::T + E::T * (q ^ (g & E::SWZ)) + ((t + q) & (E::T - 1));
}

// Backward DFT of one column: x[r] = X[t + T r] in, x[r] = y[t + T r] out,
// y[n] = sum_k X[k] exp(+2 pi i n k / NZ).  xg = the warp's exchange buffers,
// g = this thread's group in the warp, tw[q T + t] = exp(2 pi i q t / NZ).
// Warp-collective (every lane of the warp calls it together).
template <class E>
__device__ __forceinline__ void xform(cplx (&x)[8], cplx* xg, const cplx* tw, int g, int t) {
    constexpr int T = E::T;
    dft8<+1>(x);
#pragma unroll
    for (int q = 1; q < 8; ++q) x[q] = cmul(x[q], tw[q * T + t]);
#pragma unroll
    for (int q = 0; q < 8; ++q) xg[xslot<E>(g, q, t)] = x[q];
    __syncwarp();
    if constexpr (T <= 8) {
        constexpr int J = 8 / T;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int q = t + T * j;
            cplx v[T];
#pragma unroll
            for (int s = 0; s < T; ++s) v[s] = xg[xslot<E>(g, q, s)];
            dft<T, +1>(v);
#pragma unroll
            for (int m = 0; m < T; ++m) x[j + J * m] = v[m];
        }
    } else {
        // T = 16: thread (q, h) = (t % 8, t / 8) takes the outputs of parity h of the
        // 16-point transforms over the columns of row q: a radix-2 step then a DFT-8.
        const int q = t & 7, h = t >> 3;
        const double sg = h ? -1.0 : 1.0;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            const cplx za = xg[xslot<E>(g, q, s)];
            const cplx zb = xg[xslot<E>(g, q, s + 8)];
            cplx w = mk(fma(sg, zb.x, za.x), fma(sg, zb.y, za.y));
            if (s != 0) w = cmul(w, mk(h ? c16(s) : 1.0, h ? s16(s) : 0.0));
            x[s] = w;
        }
        dft8<+1>(x);
    }
    __syncwarp();
}

// A store of the new state or right-hand side: read again one stage later, after
// the whole ensemble has streamed through L2, so it is marked evict-first
// (st.global.cs) and leaves L2 to the prefetched fields of the next modes.
__device__ __forceinline__ void st_stream(cplx* p, cplx v) {
    __stcs(reinterpret_cast<double2*>(p), make_double2(v.x, v.y));
}

// ---------------------------------------------------------------------------
// Tensor-memory scratchpad of one thread: Ex (16 columns), Ey (16), S (32).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tm_ld8d(uint32_t a, double (&v)[8]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(a));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __hiloint2double((int)r[2 * i + 1], (int)r[2 * i]);
}
__device__ __forceinline__ void tm_st8d(uint32_t a, const double (&v)[8]) {
    uint32_t r[16];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        r[2 * i] = (uint32_t)__double2loint(v[i]);
        r[2 * i + 1] = (uint32_t)__double2hiint(v[i]);
    }
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};\n" ::"r"(a),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tm_ld8c(uint32_t a, cplx (&v)[8]) {
    double lo[8], hi[8];
    tm_ld8d(a, lo);
    tm_ld8d(a + 16, hi);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        v[i] = mk(lo[2 * i], lo[2 * i + 1]);
        v[i + 4] = mk(hi[2 * i], hi[2 * i + 1]);
    }
}
__device__ __forceinline__ void tm_st8c(uint32_t a, const cplx (&v)[8]) {
    double lo[8], hi[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        lo[2 * i] = v[i].x;
        lo[2 * i + 1] = v[i].y;
        hi[2 * i] = v[i + 4].x;
        hi[2 * i + 1] = v[i + 4].y;
    }
    tm_st8d(a, lo);
    tm_st8d(a + 16, hi);
}
__device__ __forceinline__ void tm_ld4c(uint32_t a, cplx (&v)[4]) {
    double d[8];
    tm_ld8d(a, d);
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = mk(d[2 * i], d[2 * i + 1]);
}
__device__ __forceinline__ void tm_st4c(uint32_t a, const cplx* v) {
    double d[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        d[2 * i] = v[i].x;
        d[2 * i + 1] = v[i].y;
    }
    tm_st8d(a, d);
}
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// mbarrier-tracked bulk copy of a mode's fields into the pair's staging buffer
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// proxy_fence: the destination may hold generic-proxy stores (the previous chunk's sums and
// mean-field scratch reuse the staging buffers), which must be ordered before the async-proxy
// write.  Within a chunk the buffer is only read by generic loads, which have returned before
// the warp barrier that precedes the next copy, so no fence is needed there.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar,
                                          bool proxy_fence) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    if (proxy_fence) asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(d),
                 "l"(src), "r"(bytes), "r"(b)
                 : "memory");
}
// Bounded wait for phase `ph` of the barrier; false when it did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned ph) {
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    for (int it = 0; it < (1 << 22); ++it) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(b), "r"(ph)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Chunk header in shared memory: the case's run constants and stage arguments.
struct ChunkHdr {
    DevParams P;
    StageArgs A;
    // constants of the chunk's stage from the case's clock (thread 0, after the header)
    double tclock, t_new, qt, ts, Om2, cn_t_old, cn_dtlin_old;
    unsigned long long nstep;  // the step's noise counter (driven cases)
    int cn_old_init, diag_due, has_prev, pad2;
    int c, r, ok, top;
    unsigned tk;
    unsigned pre_tk;  // the next ticket, taken after the mode loop
    int pre_ok, pad1;
};

// ---------------------------------------------------------------------------
// Mean-field side of a stage, on the whole CTA (rare: once per case and stage).
// The transforms use the 16-point geometry of qlgpu_fft.cuh; kept out of line
// so that the chunk pipeline's registers are not shared with it.
// ---------------------------------------------------------------------------
// Real-space By, dz By, dz^2 By [3][NZ] of the header's mean field into prof.
template <int NZ>
__device__ __noinline__ void profiles_of(const ChunkHdr& hd, double* prof, cplx* scratch) {
    using G = Geom<NZ>;
    const int tid = threadIdx.x, lane = tid & 31;
    const int go = tid / G::T, to = tid % G::T;
    const unsigned gm = (G::T == 32 ? 0xffffffffu : (((1u << G::T) - 1u) << ((lane / G::T) * G::T)));
    if (go < 3) mean_profiles<G, MODEL_BQLIN>(hd.P, hd.A.mf, prof, scratch + (size_t)go * G::XSIZE, hd.A.tw, go, 3, to,
                                              gm);
}

// The CTA that completed case c's stage r: chunk partials summed in slot order,
// the mean-field stage (stress spectra, mean-field update, clock, diagnostics),
// the next stage's real-space profiles, and the release of stage r + 1.
template <int NZ, int INTEG>
__device__ __noinline__ void top_stage(const EnsLaunch& L, ChunkHdr& hd, int c, int r, int nch, double* scratch,
                                       double tclock, double t_new, bool last, bool diag_due) {
    using G = Geom<NZ>;
    using E = EG<NZ>;
    const int tid = threadIdx.x, lane = tid & 31;
    double* tot = scratch;                     // [PL]
    double* spec = tot + ((E::PL + 1) & ~1);   // [2 NEMF (H+1)]
    cplx* xo = reinterpret_cast<cplx*>(spec + ((2 * NEMF * (G::H + 1) + 1) & ~1));
    double* mfr = reinterpret_cast<double*>(xo + 3 * G::XSIZE);
    // chunk slots in slot order; 32 loads in flight per thread (this sum is on the case's
    // critical path: every CTA waits for the stage it releases)
    constexpr int U = 32;
    for (int idx = tid; idx < E::PL; idx += THREADS) {
        const double* src = hd.A.partials + idx;
        double sum = 0.0;
        for (int jj = 0; jj < nch; jj += U) {
            double v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) v[u] = jj + u < nch ? __ldcg(src + (size_t)(jj + u) * E::PL) : 0.0;
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (jj + u < nch) sum += v[u];
        }
        tot[idx] = sum;
    }
    __syncthreads();
    const int go = tid / G::T, to = tid % G::T;
    const unsigned gm = (G::T == 32 ? 0xffffffffu : (((1u << G::T) - 1u) << ((lane / G::T) * G::T)));
    constexpr int NGO = 3;  // groups taking part in the mean-field transforms
    cplx* xg_o = xo + (size_t)(go < NGO ? go : 0) * G::XSIZE;
    mean_field_stage<G, MODEL_BQLIN, INTEG, NEMF>(hd.A, hd.P, tot, spec, xg_o, hd.A.tw, go < NGO ? go : NGO, NGO, to,
                                                  gm, tclock, t_new, last, diag_due);
    __syncthreads();
    if (go < NGO) mean_profiles<G, MODEL_BQLIN>(hd.P, hd.A.mf, mfr, xg_o, hd.A.tw, go, NGO, to, gm);
    __syncthreads();
    for (int i = tid; i < 3 * NZ; i += THREADS) hd.A.mfr_cache[i] = mfr[i];
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        hd.A.clk->mfr_valid = 1;
        __threadfence();
        if (r == L.nrounds - 1) L.case_end[c] = gtimer();
        st_release_u32(L.epoch + (size_t)c * BATCH_EPOCH_STRIDE, (unsigned)(r + 1));
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// One chunk of MHD_BQlin modes (the per-pair pipeline above) for one stage.
// Returns in every thread; the CTA that completed the case's stage ran the
// mean-field stage and released the case.
// ---------------------------------------------------------------------------
template <int NZ, int INTEG, bool REC>
__device__ __noinline__ void run_chunk(const EnsLaunch& L, ChunkHdr& hd, const RoundItem it, const int r,
                                       uint32_t tmem, uint64_t* bars, unsigned char* bar_ph) {
    using E = EG<NZ>;
    constexpr int T = E::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane / T, t = lane % T, pi = g >> 1, role = g & 1;
    cplx* tw = reinterpret_cast<cplx*>(smem_raw + E::o_tw);
    double* prof = reinterpret_cast<double*>(smem_raw + E::o_prof);
    double* kzc = reinterpret_cast<double*>(smem_raw + E::o_kz);
    double* ekz = reinterpret_cast<double*>(smem_raw + E::o_ekz);
    unsigned char* wbase = smem_raw + E::o_warp + (size_t)warp * E::WARP_BYTES;
    cplx* Kw = reinterpret_cast<cplx*>(wbase);                      // this warp's KU/KB
    cplx* stg = Kw + E::K_CPLX + (size_t)pi * 4 * E::nz;           // this pair's staged fields
    cplx* xg = Kw + E::X_OFF;                                       // this warp's exchange buffers
    uint64_t* bar = bars + warp * MAX_PAIRS_PER_WARP + pi;
    const int c = it.c, j = QLGPU_CHECK_INDEX(it.j, L.ec[it.c].nch, &L.ctl->status);
    const BatchCase* cs = L.cases + c;
    const EnsCase ec = L.ec[c];
    const int s = r % 3, n = r / 3;
    const int swap = (n + L.parity) & 1;

    // ---- header (skipped when this CTA ran the same case and stage last)
    __syncthreads();
    const bool fresh = !(hd.ok && hd.c == c && hd.r == r);
    if (fresh) {
        cta_copy8(&hd.P, &cs->P, (int)sizeof(DevParams));
        cta_copy8(&hd.A, &cs->A[s], (int)sizeof(StageArgs));
    }
    __syncthreads();
    const DevParams& P = hd.P;
    const StageArgs& A = hd.A;
    const StageConst& S = A.sc;
    const int nzd = E::nz;
    // steps that start from buffer 1 read lin_out and write lin_in of the descriptor
    const cplx* lin_in = swap ? A.lin_out : A.lin_in;
    cplx* lin_out = const_cast<cplx*>(swap ? A.lin_in : A.lin_out);
    // ---- the chunk's modes: pass p, pair (warp, pi) -> mode base + p W PPW + warp PPW + pi.  The
    // first mode's staged copy and wavenumbers are requested before the tables are loaded.
    const int mbeg = j * ec.mpc;
    const int mend = min(P.nxy, mbeg + ec.mpc);
    constexpr int MPP = WARPS * E::PPW;  // modes per pass
    const int first = mbeg + warp * E::PPW;
    const unsigned fbytes = 64u * (unsigned)nzd;
    // the pair's barrier was initialised at kernel start; bar_ph holds the parity of its next phase
    unsigned phase = bar_ph[warp * MAX_PAIRS_PER_WARP + pi];
    // pair leader (role U, t = 0) issues the copies of its pair; every pair waits once per pass, so
    // a pair past the chunk's end stages the chunk's last mode (finite values; its stores and sums
    // are switched off)
    const bool leader = (role == 0 && t == 0);
    if (leader && first < mend)
        bulk_load(stg, lin_in + (size_t)min(first + pi, mend - 1) * 4 * nzd, fbytes, bar, true);
    // the mode's wavenumbers are loaded one mode ahead (their latency overlaps the previous mode)
    double nky = 0.0, nkx0 = 0.0;
    int nkyi = 0, nkxi = 0;
    if (first < mend) {
        const int m0 = min(first + pi, mend - 1);
        nky = __ldg(A.ky + m0);
        nkx0 = __ldcg(A.kx0 + m0);
        nkyi = __ldg(A.kyi + m0);
        nkxi = __ldg(A.kxi + m0);
    }
    if (tid == 0) {
        if (fresh) {
            hd.c = c;
            hd.r = r;
            hd.ok = 1;
        }
        const double tc = __ldcg(&A.clk->t);
        hd.tclock = tc;
        hd.cn_t_old = __ldcg(&A.clk->t_old);
        hd.cn_dtlin_old = __ldcg(&A.clk->dtlin_old);
        hd.cn_old_init = __ldcg(&A.clk->old_init);
        const double tn = __dadd_rn(tc, P.dt);
        hd.t_new = tn;
        int dd = 0;
        if (S.last && P.tv_interval > 0.0) {
            const double tv = __dadd_rn(__ldcg(&A.clk->timevar), P.dt);
            dd = __dsub_rn(tv, P.tv_interval) > -1e-8;
        }
        hd.diag_due = dd;
        hd.qt = __dmul_rn(P.q, tn);
        hd.ts = __dadd_rn(tc, S.t_off);
        hd.Om2 = __dmul_rn(2.0, P.Omega);
        hd.has_prev = (S.has_prev && A.Fprev) ? 1 : 0;
        hd.nstep = A.noise ? __ldcg(&A.clk->nstep) : 0ull;
        // optional record of the stage inputs (the adjoint's window recompute): step n = r / 3
        // of the launch, stage s, at the layout of the work-item engine's record
        cplx* rl = cs->rec_lin;
        StageArgs& W = hd.A;
        if (rl) {
            const size_t nlin = (size_t)P.nxy * 4 * nzd, nmfe = (size_t)P.nmf * nzd;
            W.rec_lin = rl + ((size_t)n * 3 + s) * nlin;
            W.rec_mf = cs->rec_mf + ((size_t)n * 3 + s) * nmfe;
            W.rec_kx = s == 0 ? cs->rec_kx + (size_t)n * P.nxy : nullptr;
            W.rec_t = s == 0 ? cs->rec_t + n : nullptr;
            W.rec_cn = cs->rec_cn ? cs->rec_cn + (size_t)n * 3 + s : nullptr;
        } else {
            W.rec_lin = nullptr;
            W.rec_mf = nullptr;
        }
    }
    // ---- tables of the case and stage
    if (fresh) {
        for (int i = tid; i < NZ; i += THREADS) {
            tw[i] = ldc(ec.tw8 + i);
            const int kzi = i <= E::H ? i : i - NZ;
            kzc[i] = kzval(kzi, P.kzL);
        }
        if (INTEG == INTEG_EXP)
            for (int i = tid; i < E::nz; i += THREADS) {
                ekz[i] = __ldg(A.ekz_tab + i);
                ekz[E::NZE + i] = __ldg(A.ekz_tab + E::nz + i);
            }
        const bool cached = __ldcg(&A.clk->mfr_valid) != 0;
        if (cached) {
            for (int i = tid; i < 3 * NZ; i += THREADS) prof[i] = __ldcg(A.mfr_cache + i);
        } else {
            // real-space By, dz By, dz^2 By of the stage input (MHD_BQlin.cpp:122-127); scratch:
            // warp 0's exchange buffers and warp 1's K buffers, which no staged copy writes
            __syncthreads();
            profiles_of<NZ>(hd, prof,
                            reinterpret_cast<cplx*>(smem_raw + E::o_warp) + E::X_OFF);
        }
    }
    __syncthreads();
    // read from shared memory where used, so that they do not hold registers across the mode loop
    const double& tclock = hd.tclock;
    const double& t_new = hd.t_new;
    const double& qt = hd.qt;
    const double& ts = hd.ts;
    const double& Om2 = hd.Om2;
    const double& fac = P.fac;
    const bool last = S.last != 0;
    const bool diag_due = hd.diag_due != 0;
    const bool has_prev = hd.has_prev != 0;
    const double* By = prof;
    const double* dBy = prof + NZ;
    const double* ddBy = prof + 2 * NZ;
    const double* ekz_u = ekz;
    const double* ekz_b = ekz + E::NZE;
    // the stage's mean fields and, in a step's first stage, kx0 and the clock into the record
    // (chunk 0 of the case); stable here because the previous stage, its remap and its mean-field
    // update completed before the stage was released
    if (REC && A.rec_mf && j == 0) {
        const int nmfe = P.nmf * nzd;
        for (int i = tid; i < nmfe; i += THREADS) A.rec_mf[i] = ldc(A.mf + i);
        if (A.rec_kx)
            for (int i = tid; i < P.nxy; i += THREADS) A.rec_kx[i] = __ldcg(A.kx0 + i);
        if (A.rec_t && tid == 0) A.rec_t[0] = __ldcg(&A.clk->t);
        if (A.rec_cn && tid == 0) {
            A.rec_cn->t_old = __ldcg(&A.clk->t_old);
            A.rec_cn->dtlin_old = __ldcg(&A.clk->dtlin_old);
            A.rec_cn->old_init = __ldcg(&A.clk->old_init);
        }
    }

    // TMEM scratchpad of this lane (TM_* column offsets)
    const uint32_t ta = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * COLS_PER_WARP);
    {
        double z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        tm_st8d(ta + TM_EX, z8);
        tm_st8d(ta + TM_EY, z8);
        tm_wait_st();
    }
    double dacc[3] = {0.0, 0.0, 0.0};  // U: eb, AM_b, diss_b; B: eu, AM_u, diss_u

    int m;
    bool ok = true;
    const int lp = role * T + t;  // lane within the pair
    for (int wb = first; wb < mend; wb += MPP) {  // warp-uniform
        const int mraw = wb + pi;
        const bool valid = mraw < mend;
        m = QLGPU_CHECK_INDEX(valid ? mraw : mend - 1, P.nxy, &L.ctl->status);
        // L2 prefetch of the pair's next mode (fields and previous right-hand side)
        if (leader && mraw + MPP < mend) {
            l2_prefetch(lin_in + (size_t)(mraw + MPP) * 4 * nzd, fbytes);
            if (has_prev) l2_prefetch(A.Fprev + (size_t)(mraw + MPP) * 4 * nzd, fbytes);
        }
        const double ky = nky;
        double kx0 = nkx0;
        const int kyi = nkyi, kxi = nkxi;
        if (wb + MPP < mend) {
            const int mn = min(wb + MPP + pi, mend - 1);
            nky = __ldg(A.ky + mn);
            nkx0 = __ldcg(A.kx0 + mn);
            nkyi = __ldg(A.kyi + mn);
            nkxi = __ldg(A.kxi + mn);
        }
        const double a = kx_at(kx0, P.q, ts, ky);
        const double b = ky;
        const double ab = __dmul_rn(a, b);
        const double mult = valid ? ((ky == 0.0) ? 1.0 : 2.0) : 0.0;
        const double kxe = __dadd_rn(a, __dmul_rn(__dmul_rn(P.q, S.dt_lin), ky));
        const double hxy = __dsub_rn(-__dmul_rn(kxe, kxe), __dmul_rn(ky, ky));
        double kxo = 0.0;  // CN: kx at the old operator's time
        if (INTEG == INTEG_CN) {
            if (hd.cn_old_init) kxo = kx_at(kx0, P.q, tclock, ky);
            else kxo = __dadd_rn(kx_at(kx0, P.q, hd.cn_t_old, ky), __dmul_rn(__dmul_rn(P.q, hd.cn_dtlin_old), ky));
        }
        // remap after the step (main.cpp:122-123, MHD_BQlin.cpp:319-329): the mode's new
        // state is zero and kx0 moves by one box wavenumber period
        bool zero = false;
        if (last && P.remap && __dadd_rn(kx0, __dmul_rn(qt, ky)) > P.remap_thresh) {
            zero = true;
            kx0 = __dsub_rn(kx0, P.remap_shift);
        }
        const double* __restrict__ il2row = A.ilap2 + (size_t)kyi * nzd;
        cplx* __restrict__ uo = lin_out + (size_t)m * 4 * nzd;
        cplx* __restrict__ fo = A.Fout ? A.Fout + (size_t)m * 4 * nzd : nullptr;
        const cplx* __restrict__ fpm = has_prev ? A.Fprev + (size_t)m * 4 * nzd : nullptr;
        cplx* KU = Kw + (size_t)pi * E::KPAIR;
        cplx* KB = KU + NZ + T;
        cplx* Kown = role ? KB : KU;
        cplx* Koth = role ? KU : KB;
        const int ksw = pi & E::SWZ;
        auto kslot = [&](int rr) { return T * (rr ^ ksw) + t; };
        const int f0 = role ? 2 : 0;  // u, zeta (U) or b, eta (B)
        // the staged fields of this mode
        if (!mbar_wait(bar, phase)) ok = false;
        phase ^= 1u;
        __syncwarp();
        if (REC && A.rec_lin && valid) {  // record the mode's input fields
            cplx* dst = A.rec_lin + (size_t)m * 4 * nzd;
            for (int i = lp; i < 4 * nzd; i += 2 * T) dst[i] = stg[i];
        }

        cplx x[8];
        // spectral input of a plain inverse transform: field f0 + fa over NZ
        auto load_plain = [&](int fa) {
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) {
                const int sx = sidx<E>(t, rr);
                x[rr] = (!rdead<E>(rr) && sx >= 0) ? cscale(stg[(f0 + fa) * nzd + sx], fac) : mk(0.0, 0.0);
            }
        };
        // the previous right-hand side of field f at this lane's 8 entries: requested before the
        // transform of slot 2 (first updated field) or slot 4 (second), parked in TMEM after it, so the
        // L2 round trip is covered by the transform and the update phase reads TMEM
        auto load_fp = [&](int f, cplx (&fpv)[8]) {
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) {
                const int sx = sidx<E>(t, rr);
                fpv[rr] = (valid && fpm && !rdead<E>(rr) && sx >= 0) ? ldc(fpm + f * nzd + sx) : mk(0.0, 0.0);
            }
        };
        auto update = [&](int f, const cplx (&F)[8], int rr, int sx, double em, const double* ekzt, cplx fp) {
            sx = QLGPU_CHECK_INDEX(sx, nzd, &L.ctl->status);
            const cplx uin = stg[f * nzd + sx];
            cplx nv;
            if (INTEG == INTEG_EXP) {
                const double e = em * ekzt[sx];
                const cplx accu = fpm ? cadd(cadd(cscale(F[rr], S.n1), cscale(fp, S.n2)), uin)
                                      : cadd(cscale(F[rr], S.n1), uin);
                nv = cscale(accu, e);
            } else {
                const int k = t + T * rr;
                const double kz2 = kz2val(kzc[k]);
                const bool z0 = (kyi == 0 && sx == 0);
                const double L = linop_f<MODEL_BQLIN>(P, lap_end<MODEL_BQLIN>(P, kxe, ky, kz2), f);
                const double lo = hd.cn_old_init ? lap_init<MODEL_BQLIN>(P, kxo, lap2val(ky, kz2, z0))
                                                 : lap_end<MODEL_BQLIN>(P, kxo, ky, kz2);
                nv = rk_update<INTEG_CN>(S, L, linop_f<MODEL_BQLIN>(P, lo, f), F[rr], fp, uin, fpm != nullptr);
            }
            if (fo) st_stream(fo + f * nzd + sx, F[rr]);
            st_stream(uo + f * nzd + sx, zero ? mk(0.0, 0.0) : nv);
        };

        // ---- slot 1: z-components R_uz / R_bz -> K: (a c f0 - i b f1) il2 / NZ (MHD_BQlin.cpp:144-146)
        {
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) {
                const int sx = sidx<E>(t, rr);
                cplx v = mk(0.0, 0.0);
                if (!rdead<E>(rr) && sx >= 0) {
                    const double ac = __dmul_rn(a, kzc[t + T * rr]);
                    const cplx g0 = stg[f0 * nzd + sx], g1 = stg[(f0 + 1) * nzd + sx];
                    const double sc = __ldg(il2row + sx) * fac;
                    v = cscale(mk(fma(ac, g0.x, b * g1.y), fma(ac, g0.y, -b * g1.x)), sc);
                }
                x[rr] = v;
            }
            xform<E>(x, xg, tw, g, t);
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) Kown[kslot(rr)] = x[rr];
            __syncwarp();
        }
        // ---- slot 2: R_u / R_b
        {
            load_plain(0);
            if (has_prev) {
                cplx fpq[8];
                load_fp(role ? 0 : 2, fpq);  // U: b, B: u
                xform<E>(x, xg, tw, g, t);
                tm_st8c(ta + TM_FPA, fpq);
            } else {
                xform<E>(x, xg, tw, g, t);
            }
            double ex[8];
            tm_ld8d(ta + TM_EX, ex);
            const double sg = role ? -mult : mult;
            const double kdd = role ? 1.0 : 0.0;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                cplx ah[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int rr = 4 * h + i;
                    const int z = t + T * rr;
                    const cplx ko = Koth[kslot(rr)];
                    const cplx kw = Kown[kslot(rr)];
                    const cplx R = x[rr];
                    ex[rr] = fma(sg, ko.x * R.x + ko.y * R.y, ex[rr]);
                    const double ad = a * dBy[z];
                    const double dd = kdd * ddBy[z];
                    ah[i] = mk(fma(ad, R.y, dd * kw.x), fma(-ad, R.x, dd * kw.y));  // -i a dBy R + kdd ddBy K
                    const double bb = b * By[z];
                    x[rr] = mk(-bb * R.y, -bb * R.x);  // conj(i b By R)
                }
                tm_st4c(ta + TM_ACC + 16 * h, ah);
            }
            tm_st8d(ta + TM_EX, ex);
        }
        // ---- slot 3: forward -> F_b (U) or S (B)
        {
            xform<E>(x, xg, tw, g, t);
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) x[rr] = conjc(x[rr]);
            tm_st4c(ta + TM_S, x);  // S (B) / F_b (U), read in slot 7 and the update phase
            tm_st4c(ta + TM_S + 16, x + 4);
        }
        // ---- slot 4: R_zeta / R_eta: acc += i b By R
        {
            load_plain(1);
            if (has_prev) {
                cplx fpq[8];
                load_fp(role ? 1 : 3, fpq);  // U: eta, B: zeta
                xform<E>(x, xg, tw, g, t);
                tm_st8c(ta + TM_FPB, fpq);
            } else {
                xform<E>(x, xg, tw, g, t);
            }
            tm_wait_st();
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                cplx ah[4];
                tm_ld4c(ta + TM_ACC + 16 * h, ah);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int rr = 4 * h + i;
                    const double bb = b * By[t + T * rr];
                    ah[i] = mk(fma(-bb, x[rr].y, ah[i].x), fma(bb, x[rr].x, ah[i].y));
                }
                tm_st4c(ta + TM_ACC + 16 * h, ah);
            }
        }
        // ---- slot 5: U R_{i kz uz}; B R_by
        {
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) {
                const int sx = sidx<E>(t, rr);
                cplx v = mk(0.0, 0.0);
                if (!rdead<E>(rr) && sx >= 0) {
                    const double cc = kzc[t + T * rr];
                    const cplx g0 = stg[f0 * nzd + sx];
                    const cplx g1 = stg[(f0 + 1) * nzd + sx];
                    const double sc = __ldg(il2row + sx) * fac;
                    // U: i c (a c u - i b zeta) = (b c) zeta + i (a c^2) u
                    // B: (a b) b + i c eta
                    const double p0 = role ? ab : 0.0, q0 = role ? 0.0 : __dmul_rn(a, cc) * cc;
                    const double p1 = role ? 0.0 : b * cc, q1 = role ? cc : 0.0;
                    v = mk(p0 * g0.x - q0 * g0.y + p1 * g1.x - q1 * g1.y, p0 * g0.y + q0 * g0.x + p1 * g1.y + q1 * g1.x);
                    v = cscale(v, sc);
                }
                x[rr] = v;
            }
            xform<E>(x, xg, tw, g, t);
            tm_wait_st();
            double ey[8];
            tm_ld8d(ta + TM_EY, ey);
            const double sgy = role ? -mult : 0.0;
            const double ku = role ? 0.0 : 1.0;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                cplx ah[4];
                tm_ld4c(ta + TM_ACC + 16 * h, ah);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int rr = 4 * h + i;
                    const int z = t + T * rr;
                    const cplx ko = Koth[kslot(rr)];
                    const cplx kw = Kown[kslot(rr)];
                    const cplx R = x[rr];
                    ey[rr] = fma(sgy, ko.x * R.x + ko.y * R.y, ey[rr]);
                    const double d2 = -2.0 * ku * dBy[z], dd = ku * ddBy[z];
                    // the next forward input: conj(acc - 2 ku dBy R - ku ddBy KU)
                    x[rr] = mk(ah[i].x + d2 * R.x - dd * kw.x, -(ah[i].y + d2 * R.y - dd * kw.y));
                }
            }
            tm_st8d(ta + TM_EY, ey);
        }
        // ---- slot 6: forward -> F_eta (U) / F_zeta (B)
        {
            xform<E>(x, xg, tw, g, t);
            const int fl = role ? 0 : 2;           // linear term field
            const double cl = role ? (P.q - Om2) : -P.q;
            if (valid) {
#pragma unroll
                for (int rr = 0; rr < 8; ++rr) {
                    if (rdead<E>(rr)) continue;
                    const int sx = sidx<E>(t, rr);
                    if (sx < 0) continue;
                    const double cc = kzc[t + T * rr];
                    const cplx l0 = stg[fl * nzd + sx];
                    const cplx F = conjc(x[rr]);
                    x[rr] = cadd(F, imul(l0, cl * cc));
                }
            }
            tm_st4c(ta + TM_ACC, x);  // F_eta (U) / F_zeta (B) until the update phase; acc is dead here
            tm_st4c(ta + TM_ACC + 16, x + 4);
        }
        // ---- slot 7: U inverse R_uy (Ey); B forward 2 kx ky dBy KB -> F_u
        {
            if (role == 0) {
#pragma unroll
                for (int rr = 0; rr < 8; ++rr) {
                    const int sx = sidx<E>(t, rr);
                    cplx v = mk(0.0, 0.0);
                    if (!rdead<E>(rr) && sx >= 0) {
                        const double cc = kzc[t + T * rr];
                        const cplx g0 = stg[sx], g1 = stg[nzd + sx];
                        const double sc = __ldg(il2row + sx) * fac;
                        // (a b u + i c zeta) il2 fac (MHD_BQlin.cpp:143)
                        v = cscale(mk(ab * g0.x - cc * g1.y, ab * g0.y + cc * g1.x), sc);
                    }
                    x[rr] = v;
                }
            } else {
                const double ab2 = 2.0 * ab;
#pragma unroll
                for (int rr = 0; rr < 8; ++rr) {
                    const double w = ab2 * dBy[t + T * rr];
                    const cplx kw = Kown[kslot(rr)];
                    x[rr] = mk(w * kw.x, -w * kw.y);  // conj(2 a b dBy R_bz)
                }
            }
            xform<E>(x, xg, tw, g, t);
            tm_wait_st();  // S (slot 3) and Ey (slot 5) are stored before they are read back
            double ey[8];
            tm_ld8d(ta + TM_EY, ey);
            const double rl = __dmul_rn(__dmul_rn(2.0, ab), P.q);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                cplx sv[4];
                tm_ld4c(ta + TM_S + 16 * h, sv);
                if (role == 0) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int rr = 4 * h + i;
                        const cplx ko = Koth[kslot(rr)];
                        ey[rr] = fma(mult, ko.x * x[rr].x + ko.y * x[rr].y, ey[rr]);
                    }
                } else if (valid) {
                    // F_u = S + ilapF ((2 a b q) u + 2 Omega i kz zeta + fwd(...)) (MHD_BQlin.cpp:162)
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int rr = 4 * h + i;
                        if (rdead<E>(rr)) continue;
                        const int sx = sidx<E>(t, rr);
                        if (sx < 0) continue;
                        const double cc = kzc[t + T * rr];
                        const double kz2 = kz2val(cc);
                        const bool z0 = (kyi == 0 && sx == 0);
                        const double lapF = __dadd_rn(-__dmul_rn(a, a), lap2val(ky, kz2, z0));
                        const double ilapF = (z0 && kxi == 0) ? 1.0 : __drcp_rn(lapF);
                        const cplx u0 = stg[sx], z1 = stg[nzd + sx];
                        const cplx F = conjc(x[rr]);
                        const cplx lin = cadd(cadd(F, cscale(u0, rl)), imul(z1, Om2 * cc));
                        x[rr] = cadd(sv[i], cscale(lin, ilapF));
                    }
                }
            }
            tm_st8d(ta + TM_EY, ey);
        }
        // ---- RK updates of the mode's four fields (RK3CN_Elin.cpp:102-104, RK3CN.cpp:105-107) in one
        // phase after the transforms: U updates b (F in TM_S) and eta (TM_ACC), B updates u (registers)
        // and zeta (TM_ACC).  The previous right-hand sides wait in TM_FPA / TM_FPB (slots 2 and 4).
        {
            const int fs = role ? 0 : 2, fa = role ? 1 : 3;
            const double* ekzt = role ? ekz_u : ekz_b;
            cplx fpv[8] = {};
            // the integrating factor of the role's fields, computed while the TMEM loads are in flight
            const double em = (INTEG == INTEG_EXP) ? exp(S.linC * (role ? P.nu : P.cb) * hxy) : 1.0;
            tm_wait_st();  // F (slot 6) is stored before it is read back
            {
                cplx FS[8];
                tm_ld8c(ta + TM_S, FS);
                if (has_prev) tm_ld8c(ta + TM_FPA, fpv);
                if (role) {
#pragma unroll
                    for (int rr = 0; rr < 8; ++rr) FS[rr] = x[rr];
                }
                if (valid) {
#pragma unroll
                    for (int rr = 0; rr < 8; ++rr) {
                        if (rdead<E>(rr)) continue;
                        const int sx = sidx<E>(t, rr);
                        if (sx >= 0) update(fs, FS, rr, sx, em, ekzt, fpv[rr]);
                    }
                }
            }
            if (has_prev) tm_ld8c(ta + TM_FPB, fpv);
            {
                cplx FA[8];
                tm_ld8c(ta + TM_ACC, FA);
                if (valid) {
#pragma unroll
                    for (int rr = 0; rr < 8; ++rr) {
                        if (rdead<E>(rr)) continue;
                        const int sx = sidx<E>(t, rr);
                        if (sx >= 0) update(fa, FA, rr, sx, em, ekzt, fpv[rr]);
                    }
                }
            }
        }
        // ---- after the mode: remap bookkeeping, next mode's copy, diagnostics
        if (zero && valid && role == 0 && t == 0) A.kx0[m] = kx0;
        // the next mode's 1/lap2 row into L1 (a read-only table): its loads in slots 1, 5, 7 hit L1
        if (wb + MPP < mend && lp * 16 < nzd) {
            const double* row = A.ilap2 + (size_t)nkyi * nzd + 16 * lp;
            asm volatile("prefetch.global.L1 [%0];\n" ::"l"(row));
        }
        __syncwarp();  // every lane is done with the staging buffer and K
        {
            const int wn = wb + MPP;
            if (leader && wn < mend)
                bulk_load(stg, lin_in + (size_t)min(wn + pi, mend - 1) * 4 * nzd, fbytes, bar, false);
        }
        if (A.noise) {
            // Model::DrivingNoise after the step (main.cpp:111-113), before the diagnostics see it
            if (valid && !zero)
                noise_mode(A.noise, hd.nstep, uo, nzd, lp, 2 * T, m, kx0, ky, kxi, kyi, P.q, tclock, P.kzL);
            __syncwarp();
        }
        if (diag_due && valid && !zero) {
            // Calc_Energy_AM_Diss per mode at t_new (MHD_BQlin.cpp:365-407): U sums the magnetic
            // terms, B the velocity terms, from the new state just stored by the pair
            const double an = kx_at(kx0, P.q, t_new, ky);
            const double abn = __dmul_rn(an, ky);
            const double md = (ky == 0.0) ? 1.0 : 2.0;
            const double vis = role ? P.nu : P.eta;
            const int fd = role ? 0 : 2;
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) {
                if (rdead<E>(rr)) continue;
                const int sx = sidx<E>(t, rr);
                if (sx < 0) continue;
                const double cc = kzc[t + T * rr];
                const bool z0 = (kyi == 0 && sx == 0);
                const double lap2 = lap2val(ky, kz2val(cc), z0);
                const double il2 = ilap2val(lap2, z0);
                const double lapF = __dadd_rn(-__dmul_rn(an, an), lap2);
                const double l2 = __dmul_rn(lapF, il2);
                const cplx f0v = ldc(uo + fd * nzd + sx), f1v = ldc(uo + (fd + 1) * nzd + sx);
                const double n0 = f0v.x * f0v.x + f0v.y * f0v.y, n1 = f1v.x * f1v.x + f1v.y * f1v.y;
                const double e = l2 * n0 - il2 * n1;
                const cplx yv = cscale(cadd(cscale(f0v, abn), imul(f1v, cc)), il2);
                dacc[0] += md * e;
                dacc[1] += md * (f0v.x * yv.x + f0v.y * yv.y);
                dacc[2] += md * vis * (-lapF * e);
            }
        }
    }
    if (leader) bar_ph[warp * MAX_PAIRS_PER_WARP + pi] = (unsigned char)phase;
    // the CTA's next ticket, taken now so that the atomic's latency overlaps the sums below.
    // Holding it cannot deadlock: what is left of this chunk (sums, count, mean-field stage)
    // never waits, so the smallest unfinished ticket is always running or about to run.
    unsigned nxt = 0;
    if (tid == 0) nxt = atomicAdd(L.next, 1u);
    if (!ok && (lane & (2 * T - 1)) == 0) {
        if (atomicOr(&L.ctl->status, QLGPU_STATUS_TIMEOUT) == 0) {
            L.ctl->fail_case = c;
            L.ctl->fail_stage = r;
            L.ctl->fail_where = 1;
        }
        atomicExch(&L.ctl->abort, 1);
    }

    // ---- CTA sums of the chunk: stress profiles (groups in lane order, then warps in order)
    __syncthreads();
    double* red = reinterpret_cast<double*>(smem_raw + E::o_warp);  // [WARPS][NEMF][NZ] then [WARPS][6]
    {
        tm_wait_st();
        double ex[8], ey[8];
        tm_ld8d(ta + TM_EX, ex);
        tm_ld8d(ta + TM_EY, ey);
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
            double sx = 0.0, sy = 0.0;
#pragma unroll
            for (int gg = 0; gg < E::GPW; ++gg) {
                sx += __shfl_sync(0xffffffffu, ex[rr], gg * T + t);
                sy += __shfl_sync(0xffffffffu, ey[rr], gg * T + t);
            }
            if (g == 0) {
                red[(warp * NEMF + 0) * NZ + t + T * rr] = sx;
                red[(warp * NEMF + 1) * NZ + t + T * rr] = sy;
            }
        }
    }
    double* dred = red + (size_t)WARPS * NEMF * NZ;
    if (diag_due) {
        // U lanes hold (eb, AM_b, diss_b), B lanes (eu, AM_u, diss_u): sum each role over the
        // warp by a fixed shuffle tree over the lanes of that role
        double v6[6];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            v6[2 * q] = role ? dacc[q] : 0.0;      // velocity terms: slots 0, 2, 4
            v6[2 * q + 1] = role ? 0.0 : dacc[q];  // magnetic terms: slots 1, 3, 5
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            double v = v6[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) dred[warp * 6 + q] = v;
        }
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const BatchCase* bc = L.cases + c;
    double* part = hd.A.partials + (size_t)j * E::PL;
    for (int idx = tid; idx < NEMF * NZ; idx += THREADS) {
        double sum = 0.0;
#pragma unroll 4
        for (int w = 0; w < WARPS; ++w) sum += red[w * NEMF * NZ + idx];
        part[idx] = sum;
    }
    if (tid < 6) {
        double sum = 0.0;
        if (diag_due)
            for (int w = 0; w < WARPS; ++w) sum += dred[w * 6 + tid];
        part[NEMF * NZ + tid] = sum;
    }
    (void)bc;

    // ---- count the chunk; the CTA that completes the case's stage runs the mean-field stage
    if (tid == 0) {
        hd.pre_tk = nxt;
        hd.pre_ok = 1;
    }
    __threadfence();
    __syncthreads();
    unsigned* ep = L.epoch + (size_t)c * BATCH_EPOCH_STRIDE;
    if (tid == 0) {
        const unsigned dn = atomicAdd(ep + 1, 1u) + 1u;
        hd.top = (dn == (unsigned)((r + 1) * ec.nch)) ? 1 : 0;
    }
    __syncthreads();
    if (!hd.top) return;
    __threadfence();
    const unsigned long long t0 = (L.trace && tid == 0) ? gtimer() : 0ull;
    top_stage<NZ, INTEG>(L, hd, c, r, ec.nch, reinterpret_cast<double*>(smem_raw + E::o_warp), tclock, t_new, last,
                         diag_due);
    if (L.trace && tid == 0) L.trace[4 * (size_t)blockIdx.x + 2] += gtimer() - t0;
}

// ---------------------------------------------------------------------------
// The persistent kernel: tickets in order, one chunk per ticket.
// ---------------------------------------------------------------------------
template <int INTEG, bool REC>
__global__ void __launch_bounds__(THREADS, CTAS_PER_SM) ens_kernel(const __grid_constant__ EnsLaunch L) {
    __shared__ ChunkHdr hd;
    __shared__ __align__(8) uint64_t bars[WARPS * MAX_PAIRS_PER_WARP];
    __shared__ unsigned char bar_ph[WARPS * MAX_PAIRS_PER_WARP];
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        hd.ok = 0;
        hd.pre_ok = 0;
        if (blockIdx.x == 0) L.ctl->t_start = gtimer();
    }
    // the staging barriers are initialised once per launch (a live barrier is never re-initialised);
    // the chunks carry each barrier's phase parity in bar_ph
    if (tid < WARPS * MAX_PAIRS_PER_WARP) {
        mbar_init(&bars[tid]);
        bar_ph[tid] = 0;
    }
    if (warp == 0) tmem_alloc(&s_tmem, (uint32_t)TCOLS);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tmem = s_tmem;
    const unsigned total = (unsigned)L.R * (unsigned)L.nrounds;
    unsigned long long tw_sum = 0, tc_sum = 0, nchunks = 0;  // trace (thread 0)
    for (;;) {
        __syncthreads();  // the previous chunk is done with the header
        if (tid == 0) {
            unsigned tk = total;
            const unsigned long long t0 = L.trace ? gtimer() : 0ull;
            if (!ld_volatile_i32(&L.ctl->abort)) tk = hd.pre_ok ? hd.pre_tk : atomicAdd(L.next, 1u);
            hd.pre_ok = 0;
            if (tk < total) {
                // the case's previous stage must be complete (bounded wait)
                const int r = (int)(tk / (unsigned)L.R);
                const int c = L.round[tk % (unsigned)L.R].c;
                if (!batch_wait(L.epoch + (size_t)c * BATCH_EPOCH_STRIDE, (unsigned)r, L.ctl, L.wait_ns, c,
                                (unsigned)r))
                    tk = total;
            }
            hd.tk = tk;
            if (L.trace) tw_sum += gtimer() - t0;
        }
        __syncthreads();
        const unsigned tk = hd.tk;
        if (tk >= total) break;
        const int r = (int)(tk / (unsigned)L.R);
        RoundItem it = L.round[tk % (unsigned)L.R];
        it.c = QLGPU_CHECK_INDEX(it.c, L.ncases, &L.ctl->status);
        const unsigned long long t1 = (L.trace && tid == 0) ? gtimer() : 0ull;
        switch (L.ec[it.c].NZ) {
            case 16: run_chunk<16, INTEG, REC>(L, hd, it, r, tmem, bars, bar_ph); break;
            case 32: run_chunk<32, INTEG, REC>(L, hd, it, r, tmem, bars, bar_ph); break;
            case 64: run_chunk<64, INTEG, REC>(L, hd, it, r, tmem, bars, bar_ph); break;
            default: run_chunk<128, INTEG, REC>(L, hd, it, r, tmem, bars, bar_ph); break;
        }
        if (L.trace && tid == 0) {
            tc_sum += gtimer() - t1;
            ++nchunks;
        }
    }
    if (L.trace && tid == 0) {
        unsigned long long* tr = L.trace + 4 * (size_t)blockIdx.x;
        tr[0] = tw_sum;
        tr[1] = tc_sum;
        tr[3] = nchunks;
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc(s_tmem, (uint32_t)TCOLS);
}

// Dynamic shared memory of an NZ class
inline size_t chunk_smem(int NZ) {
    switch (NZ) {
        case 16: return EG<16>::BYTES;
        case 32: return EG<32>::BYTES;
        case 64: return EG<64>::BYTES;
        default: return EG<128>::BYTES;
    }
}
// Modes per pass of a CTA for an NZ class
inline int pass_modes(int NZ) { return WARPS * (32 / (NZ / 8)) / 2; }

}  // namespace ens
}  // namespace qlgpu
