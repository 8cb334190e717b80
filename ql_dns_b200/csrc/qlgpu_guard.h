// qlgpu_guard.h -- canary guard zones after the device buffers of the
// QLGPU_DEBUG build (host side; the check kernel is in qlgpu_guard.cu).
//
// A handle that allocates a buffer of n bytes asks for n + QLGPU_GUARD_BYTES
// and registers the zone that follows the buffer.  guard_arm fills every zone
// with QLGPU_GUARD_BYTE; guard_check scans them in one kernel and returns
// QLGPU_STATUS_CANARY if any byte changed.  In a release build
// QLGPU_GUARD_BYTES is 0 and all of it is a no-op.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "qlgpu_debug.cuh"

namespace qlgpu {

struct GuardList {
    std::vector<GuardZone> zones;
    GuardZone* d_zones = nullptr;  // device copy of `zones`
    int* d_flag = nullptr;         // set by the check kernel
    int armed = 0;                 // zones in d_zones
};

// Registers the zone after a buffer of `bytes` at `buf` (debug build only).
inline void guard_add(GuardList& g, const void* buf, size_t bytes) {
    if (QLGPU_GUARD_BYTES == 0 || !buf) return;
    g.zones.push_back(GuardZone{static_cast<const unsigned char*>(buf) + bytes});
}

// Fills every registered zone with the pattern (after the buffers were zeroed).
cudaError_t guard_arm(GuardList& g, cudaStream_t s);
// Scans the zones; *bits = QLGPU_STATUS_CANARY if one changed, else 0.  Synchronises s.
cudaError_t guard_check(GuardList& g, cudaStream_t s, int* bits);
void guard_release(GuardList& g);
// Overwrites the first byte of zone `i` from the host (the test of the check itself).
cudaError_t guard_poke(GuardList& g, int i, cudaStream_t s);

}  // namespace qlgpu
