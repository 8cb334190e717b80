// qlgpu_guard.cu -- the check kernel of the canary guard zones (qlgpu_guard.h).
#include "qlgpu_guard.h"

namespace qlgpu {
namespace {

__global__ void guard_check_kernel(const GuardZone* z, int nz, int* flag) {
    const int zi = blockIdx.x;
    if (zi >= nz) return;
    const unsigned char* p = z[zi].p;
    for (int i = threadIdx.x; i < QLGPU_GUARD_BYTES; i += blockDim.x)
        if (p[i] != (unsigned char)QLGPU_GUARD_BYTE) atomicOr(flag, QLGPU_STATUS_CANARY);
}

}  // namespace

cudaError_t guard_arm(GuardList& g, cudaStream_t s) {
    if (QLGPU_GUARD_BYTES == 0 || g.zones.empty()) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    if ((int)g.zones.size() != g.armed) {
        if (g.d_zones) cudaFree(g.d_zones);
        g.d_zones = nullptr;
        e = cudaMalloc(&g.d_zones, sizeof(GuardZone) * g.zones.size());
        if (e != cudaSuccess) return e;
        if (!g.d_flag && (e = cudaMalloc(&g.d_flag, sizeof(int))) != cudaSuccess) return e;
        e = cudaMemcpyAsync(g.d_zones, g.zones.data(), sizeof(GuardZone) * g.zones.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        g.armed = (int)g.zones.size();
    }
    for (const GuardZone& z : g.zones) {
        e = cudaMemsetAsync(const_cast<unsigned char*>(z.p), QLGPU_GUARD_BYTE, QLGPU_GUARD_BYTES, s);
        if (e != cudaSuccess) return e;
    }
    return cudaMemsetAsync(g.d_flag, 0, sizeof(int), s);
}

cudaError_t guard_check(GuardList& g, cudaStream_t s, int* bits) {
    *bits = 0;
    if (QLGPU_GUARD_BYTES == 0 || g.zones.empty()) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    if (g.armed != (int)g.zones.size() && (e = guard_arm(g, s)) != cudaSuccess) return e;
    guard_check_kernel<<<g.armed, 128, 0, s>>>(g.d_zones, g.armed, g.d_flag);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int f = 0;
    if ((e = cudaMemcpyAsync(&f, g.d_flag, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    *bits = f;
    return cudaSuccess;
}

void guard_release(GuardList& g) {
    if (g.d_zones) cudaFree(g.d_zones);
    if (g.d_flag) cudaFree(g.d_flag);
    g.d_zones = nullptr;
    g.d_flag = nullptr;
    g.zones.clear();
    g.armed = 0;
}

cudaError_t guard_poke(GuardList& g, int i, cudaStream_t s) {
    if (i < 0 || i >= (int)g.zones.size()) return cudaErrorInvalidValue;
    return cudaMemsetAsync(const_cast<unsigned char*>(g.zones[i].p), 0x00, 1, s);
}

}  // namespace qlgpu
