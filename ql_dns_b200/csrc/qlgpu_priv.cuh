// qlgpu_priv.cuh -- per-thread private scratch buffers for the stage kernel.
//
// Each thread of a transform group keeps a few length-P complex vectors for
// the whole per-mode pipeline (real-space z / x components of the
// fluctuations, a partial right-hand side, the stress accumulators).  They are
// only ever touched by the thread that owns them, in chunks of 4 complex
// values (16 32-bit words).  Two backings with the same interface:
//
//   PrivSmem : shared memory, laid out [buffer][element][32 lanes] so that a
//              warp-wide access is one conflict-free 512-byte sweep;
//   PrivTmem : Blackwell tensor memory (TMEM) used as a per-lane scratchpad.
//              Warp w owns TMEM lanes 32*(w%4)..+31 (the 32x32b access
//              shape); each thread's buffers are consecutive 32-bit columns
//              of its own lane.  tcgen05.ld / tcgen05.st are warp-wide
//              (.sync.aligned), so every call must be warp-convergent.
#pragma once
#include <cstdint>

#include "qlgpu_fft.cuh"

namespace qlgpu {

template <class G, int NB>
struct PrivSmem {
    static constexpr bool kTmem = false;
    cplx* base;  // this warp's region: NB * P * 32 cplx
    int lane;
    __device__ __forceinline__ void init(cplx* warp_base, int l) {
        base = warp_base;
        lane = l;
    }
    __device__ __forceinline__ void ld4(int b, int c, cplx* v) const {
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] = base[((b * G::P) + 4 * c + i) * 32 + lane];
    }
    __device__ __forceinline__ void st4(int b, int c, const cplx* v) const {
#pragma unroll
        for (int i = 0; i < 4; ++i) base[((b * G::P) + 4 * c + i) * 32 + lane] = v[i];
    }
    __device__ __forceinline__ void st_fence() const {}
    __host__ __device__ static constexpr size_t smem_bytes_per_warp() { return sizeof(cplx) * NB * G::P * 32; }
    __host__ __device__ static constexpr int tmem_cols_per_warp() { return 0; }
};

template <class G, int NB>
struct PrivTmem {
    static constexpr bool kTmem = true;
    static constexpr int COLS = NB * 4 * G::P;  // 32-bit columns per thread
    uint32_t taddr;                             // lane-quarter base + this warp's column offset
    __device__ __forceinline__ void init(uint32_t tmem_base, int warp) {
        taddr = tmem_base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * COLS);
    }
    __device__ __forceinline__ void ld4(int b, int c, cplx* v) const {
        const uint32_t a = taddr + (uint32_t)(b * 4 * G::P + 16 * c);
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15])
            : "r"(a));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            v[i].x = __hiloint2double((int)r[4 * i + 1], (int)r[4 * i + 0]);
            v[i].y = __hiloint2double((int)r[4 * i + 3], (int)r[4 * i + 2]);
        }
    }
    __device__ __forceinline__ void st4(int b, int c, const cplx* v) const {
        const uint32_t a = taddr + (uint32_t)(b * 4 * G::P + 16 * c);
        uint32_t r[16];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            r[4 * i + 0] = (uint32_t)__double2loint(v[i].x);
            r[4 * i + 1] = (uint32_t)__double2hiint(v[i].x);
            r[4 * i + 2] = (uint32_t)__double2loint(v[i].y);
            r[4 * i + 3] = (uint32_t)__double2hiint(v[i].y);
        }
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
            "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};\n" ::"r"(a),
            "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
            "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
            : "memory");
    }
    // Stores must complete before the same columns are read back.
    __device__ __forceinline__ void st_fence() const { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
    __host__ __device__ static constexpr size_t smem_bytes_per_warp() { return 0; }
    __host__ __device__ static constexpr int tmem_cols_per_warp() { return COLS; }
};

__device__ __forceinline__ void tmem_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// One full warp allocates ncols (power of two, 32..512) and writes the base to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(d), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(base), "r"(ncols) : "memory");
}

}  // namespace qlgpu
