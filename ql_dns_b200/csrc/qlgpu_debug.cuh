// qlgpu_debug.cuh -- the QLGPU_DEBUG build: device bounds checks and canary
// guard zones (the stand-in for a memory checker on a pool where none runs).
//
// QLGPU_CHECK_INDEX(i, n, status) is i in a release build.  With -DQLGPU_DEBUG
// it checks 0 <= i < n; a failed check sets QLGPU_STATUS_BOUNDS in the given
// status word and yields 0, so the access stays inside the buffer and the
// kernel runs on (no trap).  The host reports the bit as QLGPU_ERR_STATUS.
//
// Guard zones: in a debug build every device buffer is followed by
// QLGPU_GUARD_BYTES bytes filled with QLGPU_GUARD_BYTE; guard_check_kernel
// scans a list of zones after each launch and sets QLGPU_STATUS_CANARY where a
// byte changed (an out-of-bounds store that the index checks missed).
#pragma once
#include <cuda_runtime.h>

#include "qlgpu_types.h"

#ifdef QLGPU_DEBUG
#define QLGPU_GUARD_BYTES 256
#define QLGPU_DEBUG_BUILD 1
#else
#define QLGPU_GUARD_BYTES 0
#define QLGPU_DEBUG_BUILD 0
#endif
#define QLGPU_GUARD_BYTE 0xA5

namespace qlgpu {

__device__ __forceinline__ long long dbg_index(long long i, long long n, int* status) {
    if (i < 0 || i >= n) {
        if (status) atomicOr(status, QLGPU_STATUS_BOUNDS);
        return 0;
    }
    return i;
}

// A stored kz index: -1 (a dropped wavenumber) or 0 <= s < nz.
__device__ __forceinline__ int dbg_stored(int s, int nz, int* status) {
    if (s < -1 || s >= nz) {
        if (status) atomicOr(status, QLGPU_STATUS_BOUNDS);
        return -1;
    }
    return s;
}

#ifdef QLGPU_DEBUG
#define QLGPU_CHECK_INDEX(i, n, status) ((decltype(i))::qlgpu::dbg_index((long long)(i), (long long)(n), (status)))
#define QLGPU_CHECK_STORED(s, nz, status) (::qlgpu::dbg_stored((s), (nz), (status)))
#else
#define QLGPU_CHECK_INDEX(i, n, status) (i)
#define QLGPU_CHECK_STORED(s, nz, status) (s)
#endif

// One guard zone: QLGPU_GUARD_BYTES bytes at p.
struct GuardZone {
    const unsigned char* p;
};

}  // namespace qlgpu
