// qlgpu_batch.cuh -- the persistent kernel of a batched ensemble: many
// independent quasi-linear cases (different mode grids, NZ, viscosities, mean
// fields) stepped for many RK3 steps by ONE cooperative launch.
//
// Every CTA owns a short list of work items (case c, CTA number i of the n
// CTAs given to c) chosen on the host.  Per stage it runs stage_body() for each
// item, i.e. the same fused stage as the single-case kernel, with the CTA
// index and count of the item in place of blockIdx / gridDim.  The last CTA of
// a case to publish its partial sums runs the case's mean-field stage and then
// releases the case's stage counter; the other CTAs of the case wait for that
// counter before their next stage of the case.  There is no grid-wide barrier:
// cases advance independently, each at the pace of its own CTAs.
//
// Every wait is bounded (wait_ns, and an iteration cap): a CTA that gives up
// sets QLGPU_STATUS_TIMEOUT and the abort word, and every CTA then leaves its
// step loop, frees its TMEM and returns.  The host launches the kernel with the
// cooperative attribute, so all CTAs are co-resident or the launch fails.
#pragma once
#include "qlgpu_kernel.cuh"

namespace qlgpu {

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile_i32(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// Wait (one thread) until *epoch >= target.  False when the launch was aborted
// or the wait exceeded wait_ns (then the abort word is set here).
static __device__ __noinline__ bool batch_wait(const unsigned* epoch, unsigned target, BatchCtl* ctl, long long wait_ns,
                                               int c, unsigned k) {
    const unsigned long long t0 = gtimer();
    // at least ~32 ns per iteration: the cap ends the wait even if the timer misbehaves
    const long long max_iter = wait_ns / 32 + 1024;
    unsigned ns = 32;
    for (long long it = 0; it < max_iter; ++it) {
        if ((int)(ld_acquire_u32(epoch) - target) >= 0) return true;
        if (ld_volatile_i32(&ctl->abort)) return false;
        if ((long long)(gtimer() - t0) > wait_ns) break;
        __nanosleep(ns);
        if (ns < 512) ns <<= 1;
    }
    if (atomicOr(&ctl->status, QLGPU_STATUS_TIMEOUT) == 0) {
        ctl->fail_case = c;
        ctl->fail_stage = (int)k;
    }
    atomicExch(&ctl->abort, 1);
    return false;
}

// Copy n bytes (a multiple of 8) from global to shared memory with the whole CTA.
__device__ __forceinline__ void cta_copy8(void* dst, const void* src, int n) {
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
    for (int i = threadIdx.x; i < n / 8; i += blockDim.x) d[i] = __ldcg(s + i);
}

// One stage of one work item of a given NZ; returns true in the CTA that
// completed the case's stage.  Kept out of line: one function per NZ class
// keeps the compile time of the kernel linear in the number of classes.  The
// shared-memory objects are declared here so that every access stays a
// shared-space access.
// Field staging in the persistent kernel: only for transforms of up to 8 points
// per thread (NZ <= 64).  At NZ = 128 the staging buffers cost the warp per SM
// that the 255-register CTA could still hold; the batch measured 8% faster
// without them (the single-case kernel keeps them: 6% faster with).
template <int NZ>
struct BatchStaging {
    static constexpr bool ON = Geom<NZ>::P <= 8;
};

template <int NZ, int MODEL, int INTEG, int MAXNZ>
__device__ __noinline__ bool batch_item_stage(const BatchCase* cs, int s, int swap, int cta, int ncta, uint32_t tmem,
                                              int n) {
    static_assert(sizeof(StageArgs) % 8 == 0 && sizeof(DevParams) % 8 == 0, "8-byte copies");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ StageShared ss;
    __shared__ __align__(16) StageArgs sA;
    __shared__ __align__(16) DevParams sP;
    __syncthreads();  // the previous item is done with sA / sP
    cta_copy8(&sP, &cs->P, (int)sizeof(DevParams));
    cta_copy8(&sA, &cs->A[s], (int)sizeof(StageArgs));
    __syncthreads();
    if (threadIdx.x == 0) {
        ss.tmem = tmem;
        if (swap) {
            const cplx* in = sA.lin_in;
            sA.lin_in = sA.lin_out;
            sA.lin_out = const_cast<cplx*>(in);
        }
        cplx* rl = cs->rec_lin;
        if (rl) {
            const size_t nlin = (size_t)sP.nxy * 4 * sP.nz, nmfe = (size_t)sP.nmf * sP.nz;
            sA.rec_lin = rl + ((size_t)n * 3 + s) * nlin;
            sA.rec_mf = cs->rec_mf + ((size_t)n * 3 + s) * nmfe;
            sA.rec_kx = s == 0 ? cs->rec_kx + (size_t)n * sP.nxy : nullptr;
            sA.rec_t = s == 0 ? cs->rec_t + n : nullptr;
            sA.rec_cn = cs->rec_cn ? cs->rec_cn + (size_t)n * 3 + s : nullptr;
        }
    }
    __syncthreads();
    return stage_body<NZ, MODEL, INTEG, true, BatchStaging<NZ>::ON>(sA, sP, cta, ncta, smem_raw, ss);
}

// MAXNZ: the largest NZ class the kernel steps.  With TMEM one CTA runs per
// SM; classes up to NZ = 64 hold 8 points per thread, fit 128 registers and
// run 16-warp CTAs, the NZ = 128 / 256 classes (16 points per thread) 8-warp CTAs.
template <int MAXNZ>
struct BatchOcc {
    static constexpr int MAX_THREADS = MAXNZ <= 64 ? 512 : 256;
};

template <int MODEL, int INTEG, int MAXNZ>
__global__ void __launch_bounds__(BatchOcc<MAXNZ>::MAX_THREADS, 1) batch_kernel(BatchLaunch L) {
    __shared__ uint32_t s_tmem;
    __shared__ int s_ok;
    __shared__ BatchSlot s_items[BATCH_MAX_SLOTS];
    __shared__ int s_top[BATCH_MAX_SLOTS];
    const int tid = threadIdx.x, warp = tid >> 5;
    const BatchCta* me = L.ctas + blockIdx.x;
    const int nitems = min(me->nslots, BATCH_MAX_SLOTS);
    const int tcols = me->tcols;
    if (tid < nitems * 4) reinterpret_cast<int*>(s_items)[tid] = reinterpret_cast<const int*>(me->slot)[tid];
    if (blockIdx.x == 0 && tid == 0) L.ctl->t_start = gtimer();
    if (tcols > 0 && warp == 0) tmem_alloc(&s_tmem, (uint32_t)tcols);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tmem = tcols > 0 ? s_tmem : 0u;
    bool ok = true;
    unsigned k = 0;  // stages completed by every case in this launch
    for (int n = 0; n < L.nsteps && ok; ++n) {
        const int swap = (n + L.parity) & 1;
        for (int s = 0; s < 3 && ok; ++s, ++k) {
            // all items of this CTA publish stage k before the CTA waits for any of them
            for (int i = 0; i < nitems; ++i) {
                const BatchSlot it = s_items[i];
                const BatchCase* cs = L.cases + QLGPU_CHECK_INDEX(it.c, L.ncases, &L.ctl->status);
                bool top = false;
                if (it.NZ == 16) {
                    top = batch_item_stage<16, MODEL, INTEG, MAXNZ>(cs, s, swap, it.cta, it.ncta, tmem, n);
                } else if (it.NZ == 32) {
                    top = batch_item_stage<32, MODEL, INTEG, MAXNZ>(cs, s, swap, it.cta, it.ncta, tmem, n);
                } else if (it.NZ == 64) {
                    top = batch_item_stage<64, MODEL, INTEG, MAXNZ>(cs, s, swap, it.cta, it.ncta, tmem, n);
                } else if constexpr (MAXNZ >= 128) {
                    if (it.NZ == 128)
                        top = batch_item_stage<128, MODEL, INTEG, MAXNZ>(cs, s, swap, it.cta, it.ncta, tmem, n);
                    else if (it.NZ == 256)
                        top = batch_item_stage<256, MODEL, INTEG, MAXNZ>(cs, s, swap, it.cta, it.ncta, tmem, n);
                }
                if (tid == 0) s_top[i] = top ? 1 : 0;
                if (top) {
                    __syncthreads();
                    if (tid == 0) {
                        __threadfence();
                        if (n == L.nsteps - 1 && s == 2) L.case_end[it.c] = gtimer();
                        st_release_u32(L.epoch + (size_t)it.c * BATCH_EPOCH_STRIDE, k + 1);
                    }
                }
            }
            __syncthreads();
            if (tid == 0) {
                s_ok = 1;
                for (int i = 0; i < nitems && s_ok; ++i) {
                    if (s_top[i]) continue;
                    const int c = s_items[i].c;
                    if (!batch_wait(L.epoch + (size_t)c * BATCH_EPOCH_STRIDE, k + 1, L.ctl, L.wait_ns, c, k)) s_ok = 0;
                }
                __threadfence();
            }
            __syncthreads();
            ok = s_ok != 0;
        }
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if (tcols > 0 && warp == 0) tmem_dealloc(s_tmem, (uint32_t)tcols);
}

}  // namespace qlgpu
