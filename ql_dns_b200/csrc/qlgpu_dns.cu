// qlgpu_dns.cu -- host side of the 3-D shearing-box MHD DNS (include/qlgpu_dns.h).
//
// A handle owns the state [nxy][6][nz], two rhs buffers of the same shape, the
// transform scratch X [6][Kyn][Mx][NZ], P [9][Kyn][Mx][NZ] and T [9][nxy][nz],
// and a device clock.  One step is 3 x (A, B, C, D) + the kx0 remap + the clock
// advance (qlgpu_dns.cuh), captured once in a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qlgpu.h"
#include "../../include/qlgpu_dns.h"
#include "qlgpu_dns.cuh"
#include "qlgpu_guard.h"
#include "qlgpu_host.h"

using namespace qlgpu;
using namespace qlgpu::dns;

namespace {

using KernFn = void (*)(DnsArgs);

template <int NZ>
bool pick_zx(int MX, KernFn* inv, KernFn* fwd, size_t* s_inv, size_t* s_fwd, int ncol) {
    switch (MX) {
        case 16: *inv = dns_inv_zx<NZ, 16>; *fwd = dns_fwd_xz<16, NZ>;
                 *s_inv = InvZX<NZ, 16>::smem(ncol); *s_fwd = FwdXZ<16, NZ>::smem(ncol); return true;
        case 32: *inv = dns_inv_zx<NZ, 32>; *fwd = dns_fwd_xz<32, NZ>;
                 *s_inv = InvZX<NZ, 32>::smem(ncol); *s_fwd = FwdXZ<32, NZ>::smem(ncol); return true;
        case 64: *inv = dns_inv_zx<NZ, 64>; *fwd = dns_fwd_xz<64, NZ>;
                 *s_inv = InvZX<NZ, 64>::smem(ncol); *s_fwd = FwdXZ<64, NZ>::smem(ncol); return true;
        default: return false;
    }
}

bool pick_kernels(int NZ, int MX, int MY, int ncol, KernFn* inv, KernFn* fwd, KernFn* phys, size_t* s_inv,
                  size_t* s_fwd, size_t* s_phys, int* zc, int* phys_threads) {
    bool ok = false;
    switch (NZ) {
        case 16: ok = pick_zx<16>(MX, inv, fwd, s_inv, s_fwd, ncol); break;
        case 32: ok = pick_zx<32>(MX, inv, fwd, s_inv, s_fwd, ncol); break;
        case 64: ok = pick_zx<64>(MX, inv, fwd, s_inv, s_fwd, ncol); break;
        default: return false;
    }
    if (!ok) return false;
    switch (MY) {
        case 16: *phys = dns_phys<16>; *s_phys = Phys<16>::smem(); *zc = Phys<16>::ZC; *phys_threads = Phys<16>::THREADS; break;
        case 32: *phys = dns_phys<32>; *s_phys = Phys<32>::smem(); *zc = Phys<32>::ZC; *phys_threads = Phys<32>::THREADS; break;
        case 64: *phys = dns_phys<64>; *s_phys = Phys<64>::smem(); *zc = Phys<64>::ZC; *phys_threads = Phys<64>::THREADS; break;
        case 128: *phys = dns_phys<128>; *s_phys = Phys<128>::smem(); *zc = Phys<128>::ZC; *phys_threads = Phys<128>::THREADS; break;
        case 256: *phys = dns_phys<256>; *s_phys = Phys<256>::smem(); *zc = Phys<256>::ZC; *phys_threads = Phys<256>::THREADS; break;
        default: return false;
    }
    return true;
}

thread_local std::string g_err;

}  // namespace

struct qlgpu_dns {
    qlgpu_dns_params p;
    int device = 0;
    cudaStream_t stream = nullptr;
    int nxy = 0, nz = 0, nx = 0, ny = 0, Kyn = 0, ncol = 0;
    DnsArgs a{};
    DnsStage st[3]{};
    KernFn k_inv = nullptr, k_fwd = nullptr, k_phys = nullptr;
    size_t s_inv = 0, s_fwd = 0, s_phys = 0;
    int zc = 16, phys_threads = 256;
    double t = 0.0;
    double divf = 0.0, kzmax = 0.0;
    double* d_part = nullptr;
    double* d_rec = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::vector<double> kx_tab;
    std::string err;
    qlgpu::GuardList guards;  // debug build: canary zones after the device buffers
};

static int fail(qlgpu_dns* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    g_err = msg;
    return code;
}

static int cuda_fail(qlgpu_dns* h, cudaError_t e, const char* where) {
    return fail(h, QLGPU_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define DNS_CK(h, call)                                  \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

static void release(qlgpu_dns* h) {
    if (!h) return;
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    void* bufs[] = {h->a.lin, h->a.kx0, h->a.X, h->a.P, h->a.T, h->a.F[0], h->a.F[1], h->a.clock,
                    h->a.status, (void*)h->a.ky, (void*)h->a.kz, (void*)h->a.twz, (void*)h->a.twx,
                    (void*)h->a.twy, h->d_part, h->d_rec};
    for (void* b : bufs)
        if (b) cudaFree(b);
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    guard_release(h->guards);
    if (h->stream) cudaStreamDestroy(h->stream);
}

static bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void make_stages(qlgpu_dns* h) {
    const double dt = h->p.dt;
    const bool cn = h->p.integrator == QLGPU_INTEG_RK3CN;
    const double lc = cn ? dt / 2 : dt;
    const double a0 = 8.0 / 15.0, a1 = 5.0 / 12.0, a2 = 3.0 / 4.0, b1 = -17.0 / 60.0, b2 = -5.0 / 12.0;
    const double p1 = 8.0 / 15.0, p2 = 2.0 / 3.0;
    // RK3CN_Elin.cpp:89-91,122-125,155-158 (RK3CN.cpp alike with dt/2)
    DnsStage s0{}, s1{}, s2{};
    s0.t_off = 0.0; s0.dt_lin = dt * p1; s0.linC = lc * a0; s0.n1 = a0 * dt; s0.n2 = 0.0; s0.tn_off = dt * p1;
    s0.cur = 0; s0.prev = 1; s0.has_prev = 0;
    s1.t_off = dt * p1; s1.dt_lin = dt * (p2 - p1); s1.linC = lc * (a1 + b1); s1.n1 = a1 * dt; s1.n2 = b1 * dt;
    s1.tn_off = dt * p2; s1.cur = 1; s1.prev = 0; s1.has_prev = 1;
    s2.t_off = dt * p2; s2.dt_lin = dt * (1.0 - p2); s2.linC = lc * (a2 + b2); s2.n1 = a2 * dt; s2.n2 = b2 * dt;
    s2.tn_off = dt; s2.cur = 0; s2.prev = 1; s2.has_prev = 1; s2.last = 1;
    h->st[0] = s0; h->st[1] = s1; h->st[2] = s2;
}

// One launch of the step with programmatic dependent launch: the kernel may be
// scheduled while the previous one drains (it waits in pdl_start before it touches
// global memory), which hides the launch gap between the short kernels of a stage.
template <typename... Args>
static cudaError_t launch_pdl(void (*k)(Args...), dim3 grid, int block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = grid;
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

// Products of the current state: launches A, B, C.
static cudaError_t enqueue_products(qlgpu_dns* h) {
    const DnsArgs& a = h->a;
    cudaError_t e = launch_pdl(h->k_inv, dim3(h->Kyn, 6), BLOCK, h->s_inv, h->stream, a);
    if (e == cudaSuccess)
        e = launch_pdl(h->k_phys, dim3(h->p.Mx, h->p.NZ / h->zc), h->phys_threads, h->s_phys, h->stream, a);
    if (e == cudaSuccess) e = launch_pdl(h->k_fwd, dim3(h->Kyn, NPROD), BLOCK, h->s_fwd, h->stream, a);
    return e;
}

static cudaError_t enqueue_step(qlgpu_dns* h) {
    const int n = h->nxy * h->nz;
    for (int s = 0; s < 3; ++s) {
        cudaError_t e = enqueue_products(h);
        if (e == cudaSuccess)
            e = launch_pdl(dns_update, dim3((n + BLOCK - 1) / BLOCK), BLOCK, 0, h->stream, h->a, h->st[s]);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = launch_pdl(dns_remap_kx, dim3((h->nxy + 255) / 256), 256, 0, h->stream, h->a);
    if (e == cudaSuccess) e = launch_pdl(dns_advance_clock, dim3(1), 32, 0, h->stream, h->a);
    return e;
}

static cudaError_t enqueue_diag(qlgpu_dns* h) {
    dns_diag_modes<<<(h->nxy * 32 + 255) / 256, 256, 0, h->stream>>>(h->a, h->d_part);
    dns_diag_final<<<1, 256, 0, h->stream>>>(h->a, h->d_part, h->divf, h->kzmax, h->d_rec);
    return cudaGetLastError();
}

extern "C" {

int qlgpu_dns_create(const qlgpu_dns_params* p, int device, qlgpu_dns_t** out) {
    if (!p || !out) return fail(nullptr, QLGPU_ERR_ARG, "null argument");
    *out = nullptr;
    if (p->integrator != QLGPU_INTEG_RK3CN_ELIN && p->integrator != QLGPU_INTEG_RK3CN)
        return fail(nullptr, QLGPU_ERR_ARG, "integrator must be 0 (RK3CN_Elin) or 1 (RK3CN)");
    if (!pow2(p->Mx) || !pow2(p->My) || !pow2(p->NZ) || p->Mx < 16 || p->Mx > 64 || p->NZ < 16 || p->NZ > 64 ||
        p->My < 16 || p->My > 256)
        return fail(nullptr, QLGPU_ERR_UNSUPPORTED, "grid: Mx, NZ in {16, 32, 64}, My in {16, ..., 256}");
    if (!(p->dt > 0) || !(p->L[0] > 0) || !(p->L[1] > 0) || !(p->L[2] > 0) || p->viscosity_order < 0 ||
        !(p->nu >= 0) || !(p->eta >= 0))
        return fail(nullptr, QLGPU_ERR_ARG, "dt, L must be > 0; nu, eta, viscosity_order >= 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(nullptr, QLGPU_ERR_NODEVICE, "no CUDA device");
    qlgpu_dns* h = new qlgpu_dns();
    h->p = *p;
    if (device < 0) cudaGetDevice(&device);
    h->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { int r = cuda_fail(h, e, "cudaSetDevice"); delete h; return r; }
    // the mode set of the QL layout (Kdata.cpp:30-46) with nx = 2 floor(Mx/3)+2, ny = 2 floor(My/3)+2
    qlgpu_params qp{};
    qp.model = QLGPU_MODEL_MHD_FULLQLIN;
    qp.integrator = p->integrator;
    qp.nx = 2 * (p->Mx / 3) + 2;
    qp.ny = 2 * (p->My / 3) + 2;
    qp.NZ = p->NZ;
    for (int i = 0; i < 3; ++i) qp.L[i] = p->L[i];
    h->nx = qp.nx;
    h->ny = qp.ny;
    h->Kyn = qp.ny / 2;
    h->ncol = qp.nx - 1;
    h->nxy = h->ncol * h->Kyn;
    h->nz = stored_nz(p->NZ);
    if (!pick_kernels(p->NZ, p->Mx, p->My, h->ncol, &h->k_inv, &h->k_fwd, &h->k_phys, &h->s_inv, &h->s_fwd,
                      &h->s_phys, &h->zc, &h->phys_threads)) {
        delete h;
        return fail(nullptr, QLGPU_ERR_UNSUPPORTED, "grid combination not built");
    }
    std::vector<double> kx, ky;
    std::vector<int> kxi, kyi;
    ktables(qp, kx, ky, kxi, kyi);
    h->kx_tab = kx;
    const int nzl = (h->nz - 1) / 2;
    const double kzL = 2 * kPI / p->L[2];
    std::vector<double> kz(h->nz);
    for (int s = 0; s < h->nz; ++s) kz[s] = (s <= nzl ? s : (-2 * nzl + s - 1)) * kzL;  // Kdata.cpp:74-78
    DnsArgs& a = h->a;
    a.nxy = h->nxy; a.nz = h->nz; a.ncol = h->ncol; a.Kyn = h->Kyn; a.nx = h->nx;
    a.Mx = p->Mx; a.My = p->My; a.NZ = p->NZ;
    a.order_half = p->viscosity_order / 2;
    a.remap = p->remap;
    a.integ = p->integrator;
    a.dkx = 2 * kPI / p->L[0];
    a.q = p->q; a.omega = p->omega; a.nu = p->nu; a.eta = p->eta; a.B0z = p->B0z;
    a.scale = 1.0 / ((double)p->Mx * (double)p->My * (double)p->NZ);
    a.kmask = p->dealias_xy ? (p->Mx / 3.0) * a.dkx : 1e300;
    a.dt = p->dt;
    a.remap_thresh = (h->nx - 1) / 2.0 * a.dkx;
    a.remap_shift = (double)(h->nx - 1) * a.dkx;
    const double norm = (double)p->Mx * (double)p->My * (double)p->NZ;
    h->divf = p->L[2] / (norm * norm);
    h->kzmax = 2 * kPI / p->L[2] * (p->NZ / 3);
    make_stages(h);
    const size_t ns = (size_t)h->nxy * 6 * h->nz;
    const size_t plane = (size_t)h->Kyn * p->Mx * p->NZ;
    auto alloc = [&](void** ptr, size_t bytes) { return cudaMalloc(ptr, bytes); };
    int rc = QLGPU_OK;
#define DNS_AL(ptr, bytes)                                                         \
    if (rc == QLGPU_OK) {                                                          \
        cudaError_t e2 = alloc((void**)&(ptr), (bytes) + QLGPU_GUARD_BYTES);       \
        if (e2 != cudaSuccess) rc = cuda_fail(h, e2, "cudaMalloc " #ptr);          \
        else guard_add(h->guards, (ptr), (bytes));                                 \
    }
    DNS_AL(a.lin, ns * sizeof(cplx));
    DNS_AL(a.F[0], ns * sizeof(cplx));
    DNS_AL(a.F[1], ns * sizeof(cplx));
    DNS_AL(a.kx0, h->nxy * sizeof(double));
    DNS_AL(a.X, 6 * plane * sizeof(cplx));
    DNS_AL(a.P, NPROD * plane * sizeof(cplx));
    DNS_AL(a.T, (size_t)NPROD * h->nxy * h->nz * sizeof(cplx));
    DNS_AL(a.clock, 2 * sizeof(double));
    DNS_AL(a.status, sizeof(int));
    DNS_AL(a.ky, h->nxy * sizeof(double));
    DNS_AL(a.kz, h->nz * sizeof(double));
    DNS_AL(a.twz, 2 * p->NZ * sizeof(double));
    DNS_AL(a.twx, 2 * p->Mx * sizeof(double));
    DNS_AL(a.twy, 2 * p->My * sizeof(double));
    DNS_AL(h->d_part, (size_t)h->nxy * 6 * sizeof(double));
    DNS_AL(h->d_rec, 15 * sizeof(double));
#undef DNS_AL
    if (rc == QLGPU_OK) {
        std::vector<double> twz = twiddles(p->NZ, group_threads(p->NZ));
        std::vector<double> twx = twiddles(p->Mx, group_threads(p->Mx));
        std::vector<double> twy = twiddles(p->My, group_threads(p->My));
        cudaError_t e3 = cudaSuccess;
        if (e3 == cudaSuccess) e3 = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (e3 == cudaSuccess) e3 = cudaMemcpy((void*)a.ky, ky.data(), h->nxy * sizeof(double), cudaMemcpyHostToDevice);
        if (e3 == cudaSuccess) e3 = cudaMemcpy((void*)a.kz, kz.data(), h->nz * sizeof(double), cudaMemcpyHostToDevice);
        if (e3 == cudaSuccess) e3 = cudaMemcpy((void*)a.twz, twz.data(), twz.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e3 == cudaSuccess) e3 = cudaMemcpy((void*)a.twx, twx.data(), twx.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e3 == cudaSuccess) e3 = cudaMemcpy((void*)a.twy, twy.data(), twy.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e3 == cudaSuccess) e3 = cudaMemcpy(a.kx0, kx.data(), h->nxy * sizeof(double), cudaMemcpyHostToDevice);
        if (e3 == cudaSuccess) e3 = cudaMemset(a.lin, 0, ns * sizeof(cplx));
        if (e3 == cudaSuccess) e3 = cudaMemset(a.F[0], 0, ns * sizeof(cplx));
        if (e3 == cudaSuccess) e3 = cudaMemset(a.F[1], 0, ns * sizeof(cplx));
        if (e3 == cudaSuccess) e3 = cudaMemset(a.clock, 0, 2 * sizeof(double));
        if (e3 == cudaSuccess) e3 = cudaMemset(a.status, 0, sizeof(int));
        if (e3 == cudaSuccess) e3 = ensure_smem_attr((const void*)h->k_inv, h->s_inv);
        if (e3 == cudaSuccess) e3 = ensure_smem_attr((const void*)h->k_fwd, h->s_fwd);
        if (e3 == cudaSuccess) e3 = ensure_smem_attr((const void*)h->k_phys, h->s_phys);
        if (e3 == cudaSuccess) e3 = cudaEventCreate(&h->ev[0]);
        if (e3 == cudaSuccess) e3 = cudaEventCreate(&h->ev[1]);
        if (e3 == cudaSuccess) e3 = guard_arm(h->guards, h->stream);
        if (e3 != cudaSuccess) rc = cuda_fail(h, e3, "dns setup");
    }
    if (rc != QLGPU_OK) {
        std::string m = h->err;
        release(h);
        delete h;
        g_err = m;
        return rc;
    }
    *out = h;
    return QLGPU_OK;
}

int qlgpu_dns_destroy(qlgpu_dns_t* h) {
    if (!h) return QLGPU_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    release(h);
    delete h;
    return QLGPU_OK;
}

int qlgpu_dns_dims(const qlgpu_dns_t* h, int* nxy, int* nz, int* nx, int* ny) {
    if (!h) return QLGPU_ERR_ARG;
    if (nxy) *nxy = h->nxy;
    if (nz) *nz = h->nz;
    if (nx) *nx = h->nx;
    if (ny) *ny = h->ny;
    return QLGPU_OK;
}

int qlgpu_dns_set_state(qlgpu_dns_t* h, double t, const double* lin, const double* kx0) {
    if (!h || !lin) return fail(h, QLGPU_ERR_ARG, "null argument");
    if (!std::isfinite(t)) return fail(h, QLGPU_ERR_ARG, "t must be finite");
    DNS_CK(h, cudaSetDevice(h->device));
    const size_t ns = (size_t)h->nxy * 6 * h->nz;
    const double* kx = kx0 ? kx0 : h->kx_tab.data();
    if (kx0) {
        // every kx0 on the lattice of 2 pi/Lx, and the columns of each ky plane in distinct
        // x bins (kx0 mod Mx): the remap keeps nx-1 consecutive integers per plane
        std::vector<int> used((size_t)h->Kyn * h->p.Mx, -1);
        for (int i = 0; i < h->nxy; ++i) {
            const double m = std::nearbyint(kx[i] / h->a.dkx);
            if (!std::isfinite(kx[i]) || std::fabs(kx[i] - m * h->a.dkx) > 1e-9 * std::max(1.0, std::fabs(kx[i])))
                return fail(h, QLGPU_ERR_ARG, "kx0 is not a multiple of 2 pi / Lx");
            const int b = (int)(((long long)m % h->p.Mx + h->p.Mx) % h->p.Mx);
            int& u = used[(size_t)(i % h->Kyn) * h->p.Mx + b];
            if (u >= 0) return fail(h, QLGPU_ERR_ARG, "two columns of one ky plane share an x bin (kx0 mod Mx)");
            u = i;
        }
    }
    DNS_CK(h, cudaMemcpyAsync(h->a.lin, lin, ns * sizeof(cplx), cudaMemcpyHostToDevice, h->stream));
    DNS_CK(h, cudaMemcpyAsync(h->a.kx0, kx, h->nxy * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    double clk[2] = {t, 0.0};
    DNS_CK(h, cudaMemcpyAsync(h->a.clock, clk, sizeof(clk), cudaMemcpyHostToDevice, h->stream));
    DNS_CK(h, cudaMemsetAsync(h->a.status, 0, sizeof(int), h->stream));
    DNS_CK(h, cudaStreamSynchronize(h->stream));
    h->t = t;
    return QLGPU_OK;
}

int qlgpu_dns_get_state(qlgpu_dns_t* h, double* t, double* lin, double* kx0) {
    if (!h) return fail(h, QLGPU_ERR_ARG, "null handle");
    DNS_CK(h, cudaSetDevice(h->device));
    const size_t ns = (size_t)h->nxy * 6 * h->nz;
    if (lin) DNS_CK(h, cudaMemcpyAsync(lin, h->a.lin, ns * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
    if (kx0) DNS_CK(h, cudaMemcpyAsync(kx0, h->a.kx0, h->nxy * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    DNS_CK(h, cudaStreamSynchronize(h->stream));
    if (t) *t = h->t;
    return QLGPU_OK;
}

static int ensure_graph(qlgpu_dns* h) {
    if (h->gexec) return QLGPU_OK;
    const char* env = getenv("QLGPU_DNS_GRAPH");
    if (env && env[0] == '0') return QLGPU_OK;
    DNS_CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_step(h);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
    if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(h, e, "dns step capture"); }
    if (e2 != cudaSuccess) return cuda_fail(h, e2, "cudaStreamEndCapture");
    h->graph = g;
    DNS_CK(h, cudaGraphInstantiate(&h->gexec, g, 0));
    return QLGPU_OK;
}

static int launch_steps(qlgpu_dns* h, int nsteps) {
    int rc = ensure_graph(h);
    if (rc != QLGPU_OK) return rc;
    for (int i = 0; i < nsteps; ++i) {
        if (h->gexec)
            DNS_CK(h, cudaGraphLaunch(h->gexec, h->stream));
        else
            DNS_CK(h, enqueue_step(h));
        h->t = h->t + h->p.dt;  // main.cpp:116, the same sum as the device clock
    }
    return QLGPU_OK;
}

// The status word after a call's launches (bit 1: non-finite state); in the debug build also
// the index checks' bit and the guard zones after every buffer.
static int check_status(qlgpu_dns* h) {
    int st = 0, g = 0;
    DNS_CK(h, cudaMemcpyAsync(&st, h->a.status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    DNS_CK(h, cudaStreamSynchronize(h->stream));
    DNS_CK(h, guard_check(h->guards, h->stream, &g));
    st |= g;
    if (st & (QLGPU_STATUS_BOUNDS | QLGPU_STATUS_CANARY))
        return fail(h, QLGPU_ERR_STATUS,
                    (st & QLGPU_STATUS_BOUNDS) ? "debug build: an index check failed"
                                               : "debug build: a guard zone was overwritten");
    if (st) return fail(h, QLGPU_ERR_STATUS, "non-finite DNS state");
    return QLGPU_OK;
}

int qlgpu_dns_step(qlgpu_dns_t* h, int nsteps, int diag_every, double* diag_out, int max_diag, int* ndiag) {
    if (!h || nsteps < 0 || diag_every < 0) return fail(h, QLGPU_ERR_ARG, "bad argument");
    if (diag_every > 0 && (!diag_out || max_diag < nsteps / diag_every))
        return fail(h, QLGPU_ERR_ARG, "diag_out too small");
    DNS_CK(h, cudaSetDevice(h->device));
    int nd = 0;
    if (diag_every <= 0) {
        int rc = launch_steps(h, nsteps);
        if (rc != QLGPU_OK) return rc;
    } else {
        for (int i = 0; i < nsteps; ++i) {
            int rc = launch_steps(h, 1);
            if (rc != QLGPU_OK) return rc;
            if ((i + 1) % diag_every == 0) {
                DNS_CK(h, enqueue_diag(h));
                DNS_CK(h, cudaMemcpyAsync(diag_out + 15 * (size_t)nd, h->d_rec, 15 * sizeof(double),
                                          cudaMemcpyDeviceToHost, h->stream));
                ++nd;
            }
        }
    }
    if (ndiag) *ndiag = nd;
    return check_status(h);
}

int qlgpu_dns_step_timed(qlgpu_dns_t* h, int nsteps, float* ms) {
    if (!h || nsteps < 1 || !ms) return fail(h, QLGPU_ERR_ARG, "bad argument");
    DNS_CK(h, cudaSetDevice(h->device));
    int rc = ensure_graph(h);
    if (rc != QLGPU_OK) return rc;
    DNS_CK(h, cudaEventRecord(h->ev[0], h->stream));
    rc = launch_steps(h, nsteps);
    if (rc != QLGPU_OK) return rc;
    DNS_CK(h, cudaEventRecord(h->ev[1], h->stream));
    DNS_CK(h, cudaEventSynchronize(h->ev[1]));
    DNS_CK(h, cudaEventElapsedTime(ms, h->ev[0], h->ev[1]));
    return check_status(h);
}

int qlgpu_dns_diagnostics(qlgpu_dns_t* h, double* out15) {
    if (!h || !out15) return fail(h, QLGPU_ERR_ARG, "null argument");
    DNS_CK(h, cudaSetDevice(h->device));
    DNS_CK(h, enqueue_diag(h));
    DNS_CK(h, cudaMemcpyAsync(out15, h->d_rec, 15 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    DNS_CK(h, cudaStreamSynchronize(h->stream));
    return QLGPU_OK;
}

int qlgpu_dns_rhs(qlgpu_dns_t* h, double t, double* F) {
    if (!h || !F) return fail(h, QLGPU_ERR_ARG, "null argument");
    DNS_CK(h, cudaSetDevice(h->device));
    DNS_CK(h, enqueue_products(h));
    DnsStage s{};
    s.rhs_only = 1;
    s.t_abs = t;
    s.cur = 0;
    const int n = h->nxy * h->nz;
    dns_update<<<(n + BLOCK - 1) / BLOCK, BLOCK, 0, h->stream>>>(h->a, s);
    DNS_CK(h, cudaGetLastError());
    const size_t ns = (size_t)h->nxy * 6 * h->nz;
    DNS_CK(h, cudaMemcpyAsync(F, h->a.F[0], ns * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
    DNS_CK(h, cudaStreamSynchronize(h->stream));
    return QLGPU_DEBUG_BUILD ? check_status(h) : QLGPU_OK;
}

int qlgpu_dns_status(qlgpu_dns_t* h, int* status) {
    if (!h || !status) return fail(h, QLGPU_ERR_ARG, "null argument");
    DNS_CK(h, cudaSetDevice(h->device));
    DNS_CK(h, cudaMemcpyAsync(status, h->a.status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    DNS_CK(h, cudaStreamSynchronize(h->stream));
    return QLGPU_OK;
}

int qlgpu_dns_last_error(const qlgpu_dns_t* h, char* buf, int buflen) {
    if (!buf || buflen <= 0) return QLGPU_ERR_ARG;
    const std::string& m = h ? h->err : g_err;
    std::strncpy(buf, m.c_str(), buflen - 1);
    buf[buflen - 1] = 0;
    return QLGPU_OK;
}

void* qlgpu_dns_stream(qlgpu_dns_t* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"
