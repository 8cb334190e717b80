// qlgpu.cu -- host side of the C ABI in include/qlgpu.h: handle lifetime,
// wavenumber tables, device buffers, stage launches and the main-loop
// bookkeeping of QL_DNS/main.cpp:108-133.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/qlgpu.h"
#include "qlgpu_handle.h"
#include "qlgpu_host.h"
#include "qlgpu_kernel.cuh"
#include "qlgpu_forcing.cuh"

using namespace qlgpu;

namespace {

thread_local std::string g_create_error;

}  // namespace

namespace {

int fail(qlgpu_t* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}

#define QLGPU_CK(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(h, QLGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int reset_clock(qlgpu_t* h, double t) {
    DevClock c;
    std::memset(&c, 0, sizeof(c));
    c.t = t;
    c.timevar = 0.0;
    c.old_init = 1;
    QLGPU_CK(cudaMemcpyAsync(h->d_clk, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream));
    return QLGPU_OK;
}

StageArgs base_args(qlgpu_t* h) {
    StageArgs A;
    std::memset(&A, 0, sizeof(A));
    A.mf = h->d_mf;
    A.kx0 = h->d_kx0;
    A.ky = h->d_ky;
    A.kxi = h->d_kxi;
    A.kyi = h->d_kyi;
    A.tw = h->d_tw;
    A.ilap2 = h->d_ilap2;
    A.partials = h->d_partials;
    A.gpartials = h->d_gpartials;
    A.clk = h->d_clk;
    A.diag_ring = h->d_diag;
    A.diag_cap = h->diag_cap;
    A.trace = h->d_trace;
    A.mfr_cache = h->d_mfr;
    return A;
}

// One RK3 step = three stage launches (RK3CN_Elin::Step / RK3CN::Step).
// ev (optional): 4 events recorded before stage 1 and after each stage.
}  // namespace

// One RK3 step = three stage launches (RK3CN_Elin::Step / RK3CN::Step).  ev
// (optional): 4 events recorded before stage 1 and after each stage.  hook
// (optional) is called before each stage launch with the stage index (the
// adjoint records the stage inputs there).
void qlgpu_enqueue_step(qlgpu_t* h, cudaEvent_t* ev, const std::function<void(int)>& hook) {
    cplx* Fbuf[3] = {h->d_F1, h->d_F2, nullptr};
    const cplx* Fprev[3] = {nullptr, h->d_F1, h->d_F2};
    cplx* Fmf[3] = {h->d_Fmf1, h->d_Fmf2, h->d_Fmf1};
    const cplx* Fmfp[3] = {nullptr, h->d_Fmf1, h->d_Fmf2};
    if (ev) cudaEventRecord(ev[0], h->stream);
    for (int s = 0; s < 3; ++s) {
        StageArgs A = base_args(h);
        A.lin_in = h->d_lin[h->cur];
        A.lin_out = h->d_lin[h->cur ^ 1];
        A.Fprev = Fprev[s];
        A.Fout = Fbuf[s];
        A.Fmf_prev = Fmfp[s];
        A.Fmf_out = (s < 2) ? Fmf[s] : nullptr;
        A.sc = h->sc[s];
        if (A.trace) A.trace += 32 * s;
        A.ekz_tab = h->ekz_dynamic ? nullptr : h->d_ekz + (size_t)s * 2 * h->nz;
        if (hook) hook(s);
        h->var.launch(A, h->dp, h->grid, h->block, h->smem, h->stream);
        if (ev) cudaEventRecord(ev[s + 1], h->stream);
        h->cur ^= 1;
    }
}

namespace {

void enqueue_step(qlgpu_t* h, cudaEvent_t* ev = nullptr) { qlgpu_enqueue_step(h, ev, nullptr); }

int ensure_diag(qlgpu_t* h, int cap) {
    if (cap <= h->diag_cap) return QLGPU_OK;
    if (h->d_diag) cudaFree(h->d_diag);
    h->d_diag = nullptr;
    QLGPU_CK(cudaMalloc(&h->d_diag, sizeof(double) * 15 * (size_t)cap));
    h->diag_cap = cap;
    return QLGPU_OK;
}

int check_launch(qlgpu_t* h) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, QLGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return QLGPU_OK;
}

}  // namespace

// Debug build: after a call's launches, the device index checks' status bits (the clock's
// and the adjoint kernels') and the guard zones after every buffer.  A release build
// returns at once.
int qlgpu_debug_verify(qlgpu_t* h) {
#ifdef QLGPU_DEBUG
    int st = 0, sa = 0, g = 0;
    QLGPU_CK(cudaMemcpyAsync(&st, &h->d_clk->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaMemcpyAsync(&sa, h->d_dbg, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(guard_check(h->guards, h->stream, &g));
    st = ((st | sa) & QLGPU_STATUS_BOUNDS) | g;
    if (st) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "debug build: device status 0x%x (%s)", st,
                      (st & QLGPU_STATUS_BOUNDS) ? "an index check failed" : "a guard zone was overwritten");
        return fail(h, QLGPU_ERR_STATUS, buf);
    }
#else
    (void)h;
#endif
    return QLGPU_OK;
}

extern "C" {

const char* qlgpu_version(void) { return "qlgpu 0.1 (sm_100a, FP64)"; }

int qlgpu_last_error(const qlgpu_t* h, char* buf, int buflen) {
    const std::string& s = h ? h->err : g_create_error;
    if (buf && buflen > 0) {
        std::snprintf(buf, (size_t)buflen, "%s", s.c_str());
    }
    return (int)s.size();
}

int qlgpu_create(const qlgpu_params* pp, int device, qlgpu_t** out) {
    qlgpu_t* h = nullptr;
    if (!pp || !out) return fail(nullptr, QLGPU_ERR_ARG, "null argument");
    *out = nullptr;
    const qlgpu_params& p = *pp;
    {
        std::string msg;
        const int prc = check_params(p, &msg);
        if (prc != QLGPU_OK) return fail(nullptr, prc, msg);
    }
    Variant var;
    const char* ps = std::getenv("QLGPU_PRIV_SMEM");
    const bool use_tmem = !(ps && ps[0] == '1');
    if (!pick_variant(p.NZ, p.model, p.integrator, use_tmem, &var))
        return fail(nullptr, QLGPU_ERR_UNSUPPORTED,
                    "unsupported NZ: must be a power of two in [16, 256]");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(nullptr, QLGPU_ERR_NODEVICE, "no CUDA device");
    h = new (std::nothrow) qlgpu_handle();
    if (!h) return fail(nullptr, QLGPU_ERR_ARG, "out of host memory");
    h->p = p;
    h->var = var;
    if (device < 0) cudaGetDevice(&device);
    h->device = device;
    int rc;
    auto bail = [&](int code) {
        g_create_error = h->err;
        qlgpu_destroy(h);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess) {
        h->err = "cudaSetDevice failed";
        return bail(QLGPU_ERR_NODEVICE);
    }
    h->NZ = p.NZ;
    h->nz = stored_nz(p.NZ);
    h->nxy = mode_count(p);
    h->nmf = mean_field_count(p);
    h->dp = make_devparams(p);
    for (int s = 0; s < 3; ++s) h->sc[s] = stage_const(p, s);
    const DevParams& d = h->dp;

    ktables(p, h->kx_tab, h->ky_tab, h->kxi_tab, h->kyi_tab);
    // Launch geometry: as many CTAs as fit, at most one mode per group
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        h->err = "cudaGetDeviceProperties failed";
        return bail(QLGPU_ERR_CUDA);
    }
    // CTA width: the number of warps (up to 16 or 8, as compiled) that maximises resident
    // warps per SM, given shared memory, registers and (for the TMEM store) 512 TMEM columns per SM.
    int best_w = 1, best_res = -1, best_per_sm = 1;
    for (int w = var.max_warps; w >= 1; --w) {
        const size_t sm_bytes = var.smem(w);
        if (sm_bytes > (size_t)prop.sharedMemPerBlockOptin) continue;
        if (ensure_smem_attr(var.kernel(), sm_bytes) !=
            cudaSuccess)
            continue;
        const int tc = var.tmem(w);
        if (tc > 512) continue;
        int want = tc > 0 ? 512 / tc : 32;
        const size_t per_cta = sm_bytes + 1024;
        while (want > 1 && per_cta * want > (size_t)prop.sharedMemPerMultiprocessor) --want;
        int pct = (int)((100.0 * per_cta * want) / (double)prop.sharedMemPerMultiprocessor + 0.999);
        if (pct > 100) pct = 100;
        cudaFuncSetAttribute(var.kernel(), cudaFuncAttributePreferredSharedMemoryCarveout, pct);
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, var.kernel(), 32 * w, sm_bytes);
        if (tc > 0 && occ > 512 / tc) occ = 512 / tc;
        if (occ < 1) continue;
        // warps that hold work at once: the CTAs the modes need (one mode per pair of
        // groups), capped by what the GPU holds.  Narrower CTAs win ties: the same
        // warps spread over more SMs.
        const int modes_per_cta = w * (32 / var.T) / 2;
        const long need = (h->nxy + modes_per_cta - 1) / modes_per_cta;
        const long cap = (long)prop.multiProcessorCount * occ;
        const int res = (int)((need < cap ? need : cap) * w);
        if (best_res < 0 || res >= best_res * 0.98) {
            best_res = res;
            best_w = w;
            best_per_sm = occ;
        }
    }
    h->warps = best_w;
    h->block = 32 * h->warps;
    h->smem = var.smem(h->warps);
    if (ensure_smem_attr(var.kernel(), h->smem) != cudaSuccess) {
        h->err = "shared memory request too large";
        return bail(QLGPU_ERR_CUDA);
    }
    {
        int want = var.tmem(h->warps) > 0 ? 512 / var.tmem(h->warps) : 32;
        const size_t per_cta = h->smem + 1024;
        while (want > 1 && per_cta * want > (size_t)prop.sharedMemPerMultiprocessor) --want;
        int pct = (int)((100.0 * per_cta * want) / (double)prop.sharedMemPerMultiprocessor + 0.999);
        if (pct > 100) pct = 100;
        cudaFuncSetAttribute(var.kernel(), cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    }
    h->tmem_cols = var.tmem(h->warps);
    int per_sm = best_per_sm;
    h->per_sm = per_sm;
    // one mode per pair of transform groups
    const int modes_per_cta = h->warps * (32 / var.T) / 2;
    int need = (h->nxy + modes_per_cta - 1) / modes_per_cta;
    int cap = prop.multiProcessorCount * per_sm;
    h->grid = need < cap ? need : cap;
    if (h->grid > 64 * RED_GROUP) h->grid = 64 * RED_GROUP;
    if (h->grid < 1) h->grid = 1;
    const int ngroups = (h->grid + RED_GROUP - 1) / RED_GROUP;

    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        h->err = "stream create failed";
        return bail(QLGPU_ERR_CUDA);
    }
    const size_t nlin = (size_t)h->nxy * 4 * h->nz, nmfe = (size_t)h->nmf * h->nz;
#define QLGPU_ALLOC(ptr, bytes)                                                      \
    if (cudaMalloc(&(ptr), (bytes) + QLGPU_GUARD_BYTES) != cudaSuccess) {             \
        h->err = "cudaMalloc failed for " #ptr;                                      \
        return bail(QLGPU_ERR_CUDA);                                                 \
    }                                                                                \
    guard_add(h->guards, (ptr), (bytes));                                            \
    cudaMemsetAsync((ptr), 0, (bytes), h->stream);
    QLGPU_ALLOC(h->d_lin[0], nlin * sizeof(cplx));
    QLGPU_ALLOC(h->d_lin[1], nlin * sizeof(cplx));
    QLGPU_ALLOC(h->d_F1, nlin * sizeof(cplx));
    QLGPU_ALLOC(h->d_F2, nlin * sizeof(cplx));
    QLGPU_ALLOC(h->d_mf, nmfe * sizeof(cplx));
    QLGPU_ALLOC(h->d_Fmf1, nmfe * sizeof(cplx));
    QLGPU_ALLOC(h->d_Fmf2, nmfe * sizeof(cplx));
    QLGPU_ALLOC(h->d_kx0, h->nxy * sizeof(double));
    QLGPU_ALLOC(h->d_ky, h->nxy * sizeof(double));
    QLGPU_ALLOC(h->d_kxi, h->nxy * sizeof(int));
    QLGPU_ALLOC(h->d_kyi, h->nxy * sizeof(int));
    QLGPU_ALLOC(h->d_tw, h->NZ * sizeof(cplx));
    QLGPU_ALLOC(h->d_partials, (size_t)h->grid * var.PL * sizeof(double));
    QLGPU_ALLOC(h->d_gpartials, (size_t)ngroups * var.PL * sizeof(double));
    QLGPU_ALLOC(h->d_clk, sizeof(DevClock));
    QLGPU_ALLOC(h->d_out15, 15 * sizeof(double));
    QLGPU_ALLOC(h->d_ilap2, (size_t)(p.ny / 2) * h->nz * sizeof(double));
    QLGPU_ALLOC(h->d_mfr, (size_t)8 * h->NZ * sizeof(double));
    QLGPU_ALLOC(h->d_ekz, (size_t)6 * h->nz * sizeof(double));
    QLGPU_ALLOC(h->d_dbg, sizeof(int));
    const std::vector<double> tw = twiddles(h->NZ, var.T);
    cudaMemcpyAsync(h->d_tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    h->il2_tab = ilap2_table(p, h->nz);
    h->ekz_tab = ekz_table(p, d);
    cudaMemcpyAsync(h->d_ekz, h->ekz_tab.data(), h->ekz_tab.size() * sizeof(double), cudaMemcpyHostToDevice,
                    h->stream);
    cudaMemcpyAsync(h->d_ilap2, h->il2_tab.data(), h->il2_tab.size() * sizeof(double), cudaMemcpyHostToDevice,
                    h->stream);
    cudaMemcpyAsync(h->d_kx0, h->kx_tab.data(), h->nxy * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_ky, h->ky_tab.data(), h->nxy * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_kxi, h->kxi_tab.data(), h->nxy * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_kyi, h->kyi_tab.data(), h->nxy * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    {
        const char* tr = std::getenv("QLGPU_TRACE");
        if (tr && tr[0] == '1') {
            QLGPU_ALLOC(h->d_trace, 3 * 32 * sizeof(unsigned long long));
        }
    }
#undef QLGPU_ALLOC
    if (guard_arm(h->guards, h->stream) != cudaSuccess) {
        h->err = "guard zones";
        return bail(QLGPU_ERR_CUDA);
    }
    rc = reset_clock(h, 0.0);
    if (rc) return bail(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        h->err = "initialisation failed";
        return bail(QLGPU_ERR_CUDA);
    }
    *out = h;
    return QLGPU_OK;
}

int qlgpu_destroy(qlgpu_t* h) {
    if (!h) return QLGPU_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    void* bufs[] = {h->d_lin[0], h->d_lin[1], h->d_F1, h->d_F2, h->d_mf, h->d_Fmf1, h->d_Fmf2,
                    h->d_kx0, h->d_ky, h->d_kxi, h->d_kyi, h->d_tw, h->d_partials, h->d_gpartials,
                    h->d_clk, h->d_diag, h->d_out15, h->d_linop, h->d_ilap2, h->d_trace,
                    h->d_mfr, h->d_ekz, h->d_forcing, h->d_kx0_prev, h->d_dbg};
    for (void* b : bufs)
        if (b) cudaFree(b);
    for (cudaEvent_t e : h->ev)
        if (e) cudaEventDestroy(e);
    guard_release(h->guards);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return QLGPU_OK;
}

int qlgpu_dims(const qlgpu_t* h, int* nxy, int* nlin, int* nz, int* nmf) {
    if (!h) return QLGPU_ERR_ARG;
    if (nxy) *nxy = h->nxy;
    if (nlin) *nlin = 4;
    if (nz) *nz = h->nz;
    if (nmf) *nmf = h->nmf;
    return QLGPU_OK;
}

static int set_state_impl(qlgpu_t* h, double t, const void* lin, const void* mf, const void* kx0, cudaMemcpyKind k) {
    if (!h || !lin || !mf) return fail(h, QLGPU_ERR_ARG, "null state pointer");
    QLGPU_CK(cudaSetDevice(h->device));
    const size_t nlin = (size_t)h->nxy * 4 * h->nz, nmfe = (size_t)h->nmf * h->nz;
    h->cur = 0;
    QLGPU_CK(cudaMemcpyAsync(h->d_lin[0], lin, nlin * sizeof(cplx), k, h->stream));
    QLGPU_CK(cudaMemcpyAsync(h->d_mf, mf, nmfe * sizeof(cplx), k, h->stream));
    if (kx0) QLGPU_CK(cudaMemcpyAsync(h->d_kx0, kx0, h->nxy * sizeof(double), k, h->stream));
    else
        QLGPU_CK(cudaMemcpyAsync(h->d_kx0, h->kx_tab.data(), h->nxy * sizeof(double), cudaMemcpyHostToDevice,
                                 h->stream));
    int rc = reset_clock(h, t);
    if (rc) return rc;
    // the integrator and model start afresh: no steps, zero mean-field profiles of a previous rhs
    h->dt_sum = 0.0;
    h->steps_taken = 0;
    if (h->d_forcing) QLGPU_CK(cudaMemsetAsync(h->d_forcing, 0, 9 * sizeof(double), h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    return QLGPU_OK;
}

static int get_state_impl(qlgpu_t* h, double* t, void* lin, void* mf, void* kx0, cudaMemcpyKind k) {
    if (!h) return QLGPU_ERR_ARG;
    QLGPU_CK(cudaSetDevice(h->device));
    const size_t nlin = (size_t)h->nxy * 4 * h->nz, nmfe = (size_t)h->nmf * h->nz;
    if (lin) QLGPU_CK(cudaMemcpyAsync(lin, h->d_lin[h->cur], nlin * sizeof(cplx), k, h->stream));
    if (mf) QLGPU_CK(cudaMemcpyAsync(mf, h->d_mf, nmfe * sizeof(cplx), k, h->stream));
    if (kx0) QLGPU_CK(cudaMemcpyAsync(kx0, h->d_kx0, h->nxy * sizeof(double), k, h->stream));
    double tt = 0;
    QLGPU_CK(cudaMemcpyAsync(&tt, &h->d_clk->t, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    if (t) *t = tt;
    return QLGPU_OK;
}

int qlgpu_set_state(qlgpu_t* h, double t, const double* lin, const double* mf, const double* kx0) {
    return set_state_impl(h, t, lin, mf, kx0, cudaMemcpyHostToDevice);
}
int qlgpu_get_state(qlgpu_t* h, double* t, double* lin, double* mf, double* kx0) {
    return get_state_impl(h, t, lin, mf, kx0, cudaMemcpyDeviceToHost);
}
int qlgpu_set_state_device(qlgpu_t* h, double t, const void* lin, const void* mf, const void* kx0) {
    return set_state_impl(h, t, lin, mf, kx0, cudaMemcpyDeviceToDevice);
}
int qlgpu_get_state_device(qlgpu_t* h, double* t, void* lin, void* mf, void* kx0) {
    return get_state_impl(h, t, lin, mf, kx0, cudaMemcpyDeviceToDevice);
}

// Steps with driving noise and / or the CFL time step (main.cpp:108-133 with
// RK3CN_Elin.cpp:76-80): per step the host reads the mean-field maxima, sets dt
// and the stage constants, enqueues the three stages (the stage-3 input's
// maxima are taken before stage 3: the profiles the last rhs computed), then
// the noise; a record after every diag_every-th step through diag_kernel.
static int step_forced(qlgpu_t* h, int nsteps, int diag_every, double* diag_out, int max_diag, int* ndiag) {
    if (!h->d_forcing) {
        QLGPU_CK(cudaMalloc(&h->d_forcing, 9 * sizeof(double)));
        QLGPU_CK(cudaMemsetAsync(h->d_forcing, 0, 9 * sizeof(double), h->stream));
    }
    if (h->noise_f != 0.0 && !h->d_kx0_prev) QLGPU_CK(cudaMalloc(&h->d_kx0_prev, h->nxy * sizeof(double)));
    if (diag_every > 0) {
        int rc = ensure_diag(h, max_diag > 0 ? max_diag : 1);
        if (rc) return rc;
    }
    const double fac = 1.0 / h->NZ;  // fftwPlans.cpp:30
    const double Ns[3] = {(double)h->p.nx, (double)((h->p.ny / 2) * 2), (double)h->NZ};
    const double dealias[3] = {2.0, 2.0, 3.0};
    double kmax = 0;  // MHD_BQlin.cpp:69-74
    for (int i = 0; i < 3; ++i) kmax = std::max(kmax, 2 * kPI / h->p.L[i] * (Ns[i] / dealias[i]));
    double t = 0;
    QLGPU_CK(cudaMemcpyAsync(&t, &h->d_clk->t, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    const double tv_saved = h->dp.tv_interval;
    h->dp.tv_interval = 0.0;  // records come from diag_kernel here
    h->ekz_dynamic = h->cfl > 0;
    int nd = 0, rc = QLGPU_OK;
    for (int n = 0; n < nsteps && rc == QLGPU_OK; ++n) {
        double dt = h->p.dt;
        if (h->cfl > 0) {
            mf_absmax2_kernel<<<1, 256, 0, h->stream>>>(h->d_mf, 1, h->nz, h->NZ, fac, h->d_forcing + 4);
            double m[8];
            QLGPU_CK(cudaMemcpyAsync(m, h->d_forcing, sizeof(m), cudaMemcpyDeviceToHost, h->stream));
            QLGPU_CK(cudaStreamSynchronize(h->stream));
            const double c = h->p.model == QLGPU_MODEL_MHD_BQLIN
                                 ? kmax * std::sqrt(m[1]) + kmax * std::sqrt(m[4]) + h->p.q
                                 : kmax * (std::sqrt(m[1]) + std::sqrt(m[0]) + std::sqrt(m[2]) + std::sqrt(m[3])) +
                                       h->p.q;
            dt = h->cfl / c;  // RK3CN_Elin.cpp:77-79
            if (dt > h->dt_max) dt = h->dt_max;
        }
        qlgpu_params pp = h->p;
        pp.dt = dt;
        h->dp.dt = dt;
        for (int s = 0; s < 3; ++s) h->sc[s] = stage_const(pp, s);
        if (h->noise_f != 0.0) {
            QLGPU_CK(cudaMemcpyAsync(h->d_kx0_prev, h->d_kx0, h->nxy * sizeof(double), cudaMemcpyDeviceToDevice,
                                     h->stream));
        }
        qlgpu_enqueue_step(h, nullptr, [&](int s) {
            if (s == 2 && h->cfl > 0)
                mf_absmax2_kernel<<<1, 256, 0, h->stream>>>(h->d_mf, h->nmf, h->nz, h->NZ, fac, h->d_forcing);
        });
        if (h->noise_f != 0.0) {
            NoiseArgs a;
            a.lin = h->d_lin[h->cur];
            a.kx0_prev = h->d_kx0_prev;
            a.kx0_now = h->d_kx0;
            a.ky = h->d_ky;
            a.kxi = h->d_kxi;
            a.kyi = h->d_kyi;
            a.nxy = h->nxy;
            a.nz = h->nz;
            a.q = h->p.q;
            a.t = t;
            a.kzL = 2 * kPI / h->p.L[2];
            a.step = h->steps_taken;
            a.ns = noise_spec(h->p, h->NZ, dt, h->noise_f, h->noise_klo, h->noise_khi, h->noise_seed,
                              h->noise_only_vel, h->noise_only_mag);
            const int n_el = h->nxy * h->nz;
            noise_kernel<<<(n_el + 255) / 256, 256, 0, h->stream>>>(a);
        }
        t = t + dt;  // main.cpp:116, the device clock's sum
        h->dt_sum += dt;
        ++h->steps_taken;
        if (diag_every > 0 && (n + 1) % diag_every == 0 && nd < max_diag) {
            h->var.diag(h->d_lin[h->cur], h->d_mf, h->d_kx0, h->d_ky, h->d_kxi, h->d_kyi, h->dp, t,
                        h->d_diag + 15 * (size_t)nd, h->stream);
            ++nd;
        }
        rc = check_launch(h);
    }
    h->dp.tv_interval = tv_saved;
    h->dp.dt = h->p.dt;
    for (int s = 0; s < 3; ++s) h->sc[s] = stage_const(h->p, s);
    h->ekz_dynamic = false;
    if (rc) return rc;
    DevClock c;
    QLGPU_CK(cudaMemcpyAsync(&c, h->d_clk, sizeof(DevClock), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    if (nd > 0) QLGPU_CK(cudaMemcpy(diag_out, h->d_diag, sizeof(double) * 15 * (size_t)nd, cudaMemcpyDeviceToHost));
    if (ndiag) *ndiag = nd;
    if (c.status & (QLGPU_STATUS_NONFINITE | QLGPU_STATUS_UNSTABLE))
        return fail(h, QLGPU_ERR_STATUS, "device status set: non-finite or unstable solution");
    return qlgpu_debug_verify(h);
}

int qlgpu_set_noise(qlgpu_t* h, double f_noise, double k_low, double k_high, unsigned long long seed) {
    if (!h) return QLGPU_ERR_ARG;
    if (!std::isfinite(f_noise) || !(k_low >= 0) || !(k_high >= k_low))
        return fail(h, QLGPU_ERR_ARG, "noise: finite f_noise, 0 <= k_low <= k_high");
    h->noise_f = f_noise;
    h->noise_klo = k_low;
    h->noise_khi = k_high;
    h->noise_seed = seed;
    return QLGPU_OK;
}

int qlgpu_debug_build(void) { return QLGPU_DEBUG_BUILD; }

int qlgpu_debug_guard_poke(qlgpu_t* h, int zone) {
    if (!h) return QLGPU_ERR_ARG;
    if (!QLGPU_DEBUG_BUILD) return fail(h, QLGPU_ERR_UNSUPPORTED, "guard zones exist in the debug build only");
    if (zone < 0 || zone >= (int)h->guards.zones.size()) return fail(h, QLGPU_ERR_ARG, "no such guard zone");
    QLGPU_CK(cudaSetDevice(h->device));
    QLGPU_CK(guard_poke(h->guards, zone, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    return QLGPU_OK;
}

int qlgpu_set_noise_fields(qlgpu_t* h, int drive_only_velocity, int drive_only_magnetic) {
    if (!h) return QLGPU_ERR_ARG;
    if ((drive_only_velocity || drive_only_magnetic) && h->p.model != QLGPU_MODEL_MHD_FULLQLIN)
        return fail(h, QLGPU_ERR_UNSUPPORTED, "drive_only_velocity / drive_only_magnetic are MHD_FullQlin inputs");
    h->noise_only_vel = drive_only_velocity != 0;
    h->noise_only_mag = drive_only_magnetic != 0;
    return QLGPU_OK;
}

int qlgpu_set_cfl(qlgpu_t* h, double cfl, double dt_max) {
    if (!h) return QLGPU_ERR_ARG;
    if (!(cfl >= 0) || (cfl > 0 && !(dt_max > 0))) return fail(h, QLGPU_ERR_ARG, "cfl >= 0 and dt_max > 0");
    h->cfl = cfl;
    h->dt_max = dt_max;
    return QLGPU_OK;
}

int qlgpu_mean_time_step(qlgpu_t* h, double* dt_mean) {
    if (!h || !dt_mean) return QLGPU_ERR_ARG;
    *dt_mean = h->steps_taken ? h->dt_sum / (double)h->steps_taken : h->p.dt;
    return QLGPU_OK;
}

int qlgpu_step(qlgpu_t* h, int nsteps, int diag_every, double* diag_out, int max_diag, int* ndiag) {
    if (!h) return QLGPU_ERR_ARG;
    if (nsteps < 0) return fail(h, QLGPU_ERR_ARG, "nsteps < 0");
    if (diag_every > 0 && (!diag_out || max_diag < 0)) return fail(h, QLGPU_ERR_ARG, "diag_out required");
    QLGPU_CK(cudaSetDevice(h->device));
    if (h->noise_f != 0.0 || h->cfl > 0) return step_forced(h, nsteps, diag_every, diag_out, max_diag, ndiag);
    h->dt_sum += nsteps * h->p.dt;
    h->steps_taken += (unsigned long long)nsteps;
    const double interval = diag_every > 0 ? diag_every * h->p.dt : 0.0;
    if (interval != h->dp.tv_interval) h->dp.tv_interval = interval;
    if (diag_every > 0) {
        int rc = ensure_diag(h, max_diag > 0 ? max_diag : 1);
        if (rc) return rc;
        // restart the record counter for this call
        int zero = 0;
        QLGPU_CK(cudaMemcpyAsync(&h->d_clk->ndiag, &zero, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    }
    for (int n = 0; n < nsteps; ++n) {
        enqueue_step(h);
        if ((n & 63) == 63) {
            int rc = check_launch(h);
            if (rc) return rc;
        }
    }
    int rc = check_launch(h);
    if (rc) return rc;
    DevClock c;
    QLGPU_CK(cudaMemcpyAsync(&c, h->d_clk, sizeof(DevClock), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    int nrec = 0;
    if (diag_every > 0) {
        nrec = c.ndiag < max_diag ? c.ndiag : max_diag;
        if (nrec > 0)
            QLGPU_CK(cudaMemcpy(diag_out, h->d_diag, sizeof(double) * 15 * (size_t)nrec, cudaMemcpyDeviceToHost));
    }
    if (ndiag) *ndiag = nrec;
    if (c.status & (QLGPU_STATUS_NONFINITE | QLGPU_STATUS_UNSTABLE | QLGPU_STATUS_DIAG_FULL)) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "device status 0x%x: %s", c.status,
                      (c.status & QLGPU_STATUS_NONFINITE)  ? "solution contains NaN or Inf (solution.cpp:194)"
                      : (c.status & QLGPU_STATUS_UNSTABLE) ? "solution is very large, probably unstable (solution.cpp:184)"
                                                           : "diagnostic records dropped (max_diag too small)");
        return fail(h, QLGPU_ERR_STATUS, buf);
    }
    return qlgpu_debug_verify(h);
}

int qlgpu_step_timed(qlgpu_t* h, float* stage_ms) {
    if (!h || !stage_ms) return QLGPU_ERR_ARG;
    QLGPU_CK(cudaSetDevice(h->device));
    for (int i = 0; i < 4; ++i)
        if (!h->ev[i]) QLGPU_CK(cudaEventCreate(&h->ev[i]));
    h->dp.tv_interval = 0.0;
    enqueue_step(h, h->ev);
    int rc = check_launch(h);
    if (rc) return rc;
    QLGPU_CK(cudaEventSynchronize(h->ev[3]));
    for (int s = 0; s < 3; ++s) QLGPU_CK(cudaEventElapsedTime(&stage_ms[s], h->ev[s], h->ev[s + 1]));
    int st = 0;
    QLGPU_CK(cudaMemcpy(&st, &h->d_clk->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st & (QLGPU_STATUS_NONFINITE | QLGPU_STATUS_UNSTABLE)) return fail(h, QLGPU_ERR_STATUS, "device status set");
    return qlgpu_debug_verify(h);
}

int qlgpu_diagnostics(qlgpu_t* h, double* out15) {
    if (!h || !out15) return QLGPU_ERR_ARG;
    QLGPU_CK(cudaSetDevice(h->device));
    double t = 0;
    QLGPU_CK(cudaMemcpyAsync(&t, &h->d_clk->t, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    h->var.diag(h->d_lin[h->cur], h->d_mf, h->d_kx0, h->d_ky, h->d_kxi, h->d_kyi, h->dp, t, h->d_out15, h->stream);
    int rc = check_launch(h);
    if (rc) return rc;
    QLGPU_CK(cudaMemcpyAsync(out15, h->d_out15, 15 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    return qlgpu_debug_verify(h);
}

int qlgpu_rhs(qlgpu_t* h, double t, double dt_lin, const double* lin_in, const double* mf_in, double* lin_rhs,
              double* mf_rhs, double* linop) {
    if (!h || !lin_in || !mf_in || !lin_rhs || !mf_rhs) return fail(h, QLGPU_ERR_ARG, "null argument");
    QLGPU_CK(cudaSetDevice(h->device));
    const size_t nlin = (size_t)h->nxy * 4 * h->nz, nmfe = (size_t)h->nmf * h->nz;
    if (linop && !h->d_linop) QLGPU_CK(cudaMalloc(&h->d_linop, nlin * sizeof(double)));
    // Scratch: F1 holds the input copy, F2 the rhs, Fmf2 the input MF copy, Fmf1 the MF rhs.
    // The model reads the mean field from A.mf, so the handle's mean field is saved and restored.
    QLGPU_CK(cudaMemcpyAsync(h->d_F1, lin_in, nlin * sizeof(cplx), cudaMemcpyHostToDevice, h->stream));
    QLGPU_CK(cudaMemcpyAsync(h->d_Fmf2, h->d_mf, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, h->stream));
    QLGPU_CK(cudaMemcpyAsync(h->d_mf, mf_in, nmfe * sizeof(cplx), cudaMemcpyHostToDevice, h->stream));
    StageArgs A = base_args(h);
    A.lin_in = h->d_F1;
    A.lin_out = h->d_F2;
    A.Fmf_out = h->d_Fmf1;
    A.rhs_only = 1;
    A.linop_out = linop ? h->d_linop : nullptr;
    A.sc.t_off = t;
    A.sc.abs_time = 1;
    A.sc.dt_lin = dt_lin;
    h->var.launch(A, h->dp, h->grid, h->block, h->smem, h->stream);
    int rc = check_launch(h);
    if (rc) return rc;
    QLGPU_CK(cudaMemcpyAsync(lin_rhs, h->d_F2, nlin * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaMemcpyAsync(mf_rhs, h->d_Fmf1, nmfe * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
    if (linop) QLGPU_CK(cudaMemcpyAsync(linop, h->d_linop, nlin * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaMemcpyAsync(h->d_mf, h->d_Fmf2, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    return qlgpu_debug_verify(h);
}

int qlgpu_status(qlgpu_t* h, int* status) {
    if (!h || !status) return QLGPU_ERR_ARG;
    QLGPU_CK(cudaSetDevice(h->device));
    QLGPU_CK(cudaMemcpyAsync(status, &h->d_clk->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    return QLGPU_OK;
}

int qlgpu_time(qlgpu_t* h, double* t) {
    if (!h || !t) return QLGPU_ERR_ARG;
    QLGPU_CK(cudaSetDevice(h->device));
    QLGPU_CK(cudaMemcpyAsync(t, &h->d_clk->t, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    return QLGPU_OK;
}

int qlgpu_trace(qlgpu_t* h, unsigned long long* out96) {
    if (!h || !out96) return QLGPU_ERR_ARG;
    if (!h->d_trace) return fail(h, QLGPU_ERR_UNSUPPORTED, "tracing is off (set QLGPU_TRACE=1 before qlgpu_create)");
    QLGPU_CK(cudaSetDevice(h->device));
    QLGPU_CK(cudaMemcpyAsync(out96, h->d_trace, 96 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
    QLGPU_CK(cudaStreamSynchronize(h->stream));
    return QLGPU_OK;
}

int qlgpu_launch_info(const qlgpu_t* h, int* info8) {
    if (!h || !info8) return QLGPU_ERR_ARG;
    info8[0] = h->grid;
    info8[1] = h->block;
    info8[2] = (int)h->smem;
    info8[3] = h->per_sm;
    info8[4] = h->tmem_cols;
    info8[5] = h->var.T;
    info8[6] = h->nxy;
    info8[7] = h->warps;
    return QLGPU_OK;
}

int qlgpu_kernel_attrs(const qlgpu_t* h, int* attrs8) {
    if (!h || !attrs8) return QLGPU_ERR_ARG;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, h->var.kernel()) != cudaSuccess) return QLGPU_ERR_CUDA;
    int occ0 = 0, occs = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ0, h->var.kernel(), h->block, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occs, h->var.kernel(), h->block, h->smem);
    attrs8[0] = fa.numRegs;
    attrs8[1] = (int)fa.sharedSizeBytes;
    attrs8[2] = (int)fa.localSizeBytes;
    attrs8[3] = fa.maxThreadsPerBlock;
    attrs8[4] = occ0;
    attrs8[5] = occs;
    attrs8[6] = fa.maxDynamicSharedSizeBytes;
    attrs8[7] = fa.preferredShmemCarveout;
    return QLGPU_OK;
}

int qlgpu_stream(qlgpu_t* h, void** stream) {
    if (!h || !stream) return QLGPU_ERR_ARG;
    *stream = (void*)h->stream;
    return QLGPU_OK;
}

}  // extern "C"

// ============================================================================
// qlgpu_rhs_noalloc: Model::rhs on caller-owned device buffers with no device
// allocation at all.
//
// Some callers cannot allocate device memory while they run this step: code
// executing inside a pre-sized memory pool or arena that forbids cudaMalloc
// after start-up, callers that own every device buffer themselves (a host
// framework passing in pointers it manages), and latency-critical loops where
// an allocation (and the implicit device synchronisation of cudaFree) is not
// acceptable.  For them the scratch the stage kernel needs (wavenumber and
// twiddle tables, per-CTA partial sums, the reduction counters) lives in one
// file-scope device array of a fixed size, loaded with the library and held by
// every GPU that loads it until the process exits.
// ============================================================================
#include <mutex>

namespace {

// Fixed scratch for qlgpu_rhs_noalloc (4 MiB per device).
#define QLGPU_NOALLOC_SCRATCH_BYTES (4u << 20)
#define QLGPU_NOALLOC_MAX_MODES 8192
#define QLGPU_NOALLOC_MAX_KY 128
#define QLGPU_NOALLOC_MAX_GRID 256

static __device__ __align__(256) unsigned char g_noalloc_scratch[QLGPU_NOALLOC_SCRATCH_BYTES];

// Per device, looked up once: the device address of g_noalloc_scratch (in host
// code the symbol g_noalloc_scratch is only a host-side stand-in; handing it to
// a kernel would read the wrong memory), the SM count and the opt-in shared
// memory per CTA.  The cache lives for the process: after cudaDeviceReset the
// context is new and the cached address is stale.
std::mutex g_noalloc_mutex;
struct NoallocDevice {
    void* ptr = nullptr;
    int sms = 0;
    int smem_optin = 0;
};
NoallocDevice g_noalloc_dev[64];

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct NoallocLayout {
    size_t tw, ky, kxi, kyi, kx0, il2, partials, gpartials, clk, end;
};

NoallocLayout noalloc_layout(int NZ, int nxy, int nyh, int nz, int grid, int PL) {
    NoallocLayout L;
    size_t o = 0;
    L.tw = o; o = align256(o + sizeof(cplx) * NZ);
    L.ky = o; o = align256(o + sizeof(double) * nxy);
    L.kxi = o; o = align256(o + sizeof(int) * nxy);
    L.kyi = o; o = align256(o + sizeof(int) * nxy);
    L.kx0 = o; o = align256(o + sizeof(double) * nxy);
    L.il2 = o; o = align256(o + sizeof(double) * (size_t)nyh * nz);
    L.partials = o; o = align256(o + sizeof(double) * (size_t)grid * PL);
    L.gpartials = o; o = align256(o + sizeof(double) * (size_t)((grid + RED_GROUP - 1) / RED_GROUP) * PL);
    L.clk = o; o = align256(o + sizeof(DevClock));
    L.end = o;
    return L;
}

// Fills the wavenumber tables (Kdata.cpp:24-46,100-119), the twiddles of the
// transform layout and the default kx0, and zeroes the reduction counters.
__global__ void noalloc_tables_kernel(unsigned char* base, NoallocLayout L, int NZ, int T, int nx, int ny, int nz,
                                      double kxL, double kyL, double kzL, int fill_kx0) {
    const int nxy = (nx - 1) * (ny / 2);
    const int nyh = ny / 2, nxh = nx / 2;
    cplx* tw = reinterpret_cast<cplx*>(base + L.tw);
    double* ky = reinterpret_cast<double*>(base + L.ky);
    int* kxi = reinterpret_cast<int*>(base + L.kxi);
    int* kyi = reinterpret_cast<int*>(base + L.kyi);
    double* kx0 = reinterpret_cast<double*>(base + L.kx0);
    double* il2 = reinterpret_cast<double*>(base + L.il2);
    DevClock* clk = reinterpret_cast<DevClock*>(base + L.clk);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const int P = NZ / T;
    for (int i = tid; i < NZ; i += nth) {
        const int n2 = i / T, t = i % T;
        const int m = (n2 * t) % NZ;
        double sn, cs;
        sincospi(2.0 * (double)m / (double)NZ, &sn, &cs);
        tw[i] = mk(cs, sn);
    }
    (void)P;
    for (int i = tid; i < nxy; i += nth) {
        // mode index j + (Ny/2) i with the kx Nyquist column dropped
        const int col = i / nyh, j = i % nyh;
        const int ix = col < nxh ? col : col + 1;  // skip the Nyquist index nx/2
        const int kxint = ix < nxh ? ix : (-2 * nxh + ix);
        ky[i] = j * kyL;
        kxi[i] = kxint;
        kyi[i] = j;
        if (fill_kx0) kx0[i] = kxint * kxL;
    }
    const int nzl = (nz - 1) / 2;
    for (int i = tid; i < nyh * nz; i += nth) {
        const int j = i / nz, s = i % nz;
        const double kyr = j * kyL;
        const int kzi = s <= nzl ? s : (-2 * nzl + s - 1);
        const double c = kzi * kzL;
        const double kz2 = -(c * c);
        double v = 1 / (-kyr * kyr + kz2);
        if (kyr == 0 && s == 0) v = 1;
        il2[i] = v;
    }
    unsigned* w = reinterpret_cast<unsigned*>(clk);
    for (int i = tid; i < (int)(sizeof(DevClock) / sizeof(unsigned)); i += nth) w[i] = 0u;
}

}  // namespace

extern "C" int qlgpu_rhs_noalloc(const qlgpu_params* pp, double t, double dt_lin, const void* lin_in,
                                 const void* mf_in, const void* kx0, void* lin_rhs, void* mf_rhs, void* linop,
                                 void* stream) {
    if (!pp || !lin_in || !mf_in || !lin_rhs || !mf_rhs) return fail(nullptr, QLGPU_ERR_ARG, "null argument");
    const qlgpu_params& p = *pp;
    if (p.model != QLGPU_MODEL_MHD_BQLIN && p.model != QLGPU_MODEL_MHD_FULLQLIN)
        return fail(nullptr, QLGPU_ERR_ARG, "unknown model");
    if (p.nx < 2 || (p.nx % 2) || p.ny < 2 || (p.ny % 2))
        return fail(nullptr, QLGPU_ERR_ARG, "nx and ny must be even and >= 2");
    if (!(p.L[0] > 0 && p.L[1] > 0 && p.L[2] > 0)) return fail(nullptr, QLGPU_ERR_ARG, "box lengths must be > 0");
    if (p.model == QLGPU_MODEL_MHD_BQLIN && p.nu == 0.0)
        return fail(nullptr, QLGPU_ERR_ARG, "MHD_BQlin divides by nu (MHD_BQlin.cpp:251); nu must be nonzero");
    {
        // the kernel moves complex values as 16-byte vectors and requests whole modes into L2
        const uintptr_t bits = (uintptr_t)lin_in | (uintptr_t)mf_in | (uintptr_t)kx0 | (uintptr_t)lin_rhs |
                               (uintptr_t)mf_rhs | (uintptr_t)linop;
        if (bits & 15) return fail(nullptr, QLGPU_ERR_ARG, "device pointers must be 16-byte aligned");
    }
    Variant var;
    if (!pick_variant(p.NZ, p.model, QLGPU_INTEG_RK3CN_ELIN, true, &var))
        return fail(nullptr, QLGPU_ERR_UNSUPPORTED, "unsupported NZ: must be a power of two in [16, 256]");
    const int nz = 1 + 2 * int(p.NZ / 3.0), nxy = (p.nx - 1) * (p.ny / 2), nyh = p.ny / 2;
    const int nmf = p.model == QLGPU_MODEL_MHD_BQLIN ? 2 : 4;
    if (nxy > QLGPU_NOALLOC_MAX_MODES || nyh > QLGPU_NOALLOC_MAX_KY)
        return fail(nullptr, QLGPU_ERR_ARG,
                    "too large for the fixed no-allocation scratch: at most 8192 (kx,ky) modes and ny <= 256 "
                    "(use qlgpu_create / qlgpu_rhs for larger grids)");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return fail(nullptr, QLGPU_ERR_NODEVICE, "no CUDA device");
    NoallocDevice nd;
    {
        // One-time set-up on this device: the device address of the scratch array and the
        // two device attributes the launch geometry needs.
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        NoallocDevice& c = g_noalloc_dev[dev];
        if (!c.ptr) {
            void* ptr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                return fail(nullptr, QLGPU_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            int sms = 0, optin = 0;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
                return fail(nullptr, QLGPU_ERR_CUDA, "device attributes");
            c.sms = sms;
            c.smem_optin = optin;
            c.ptr = ptr;
        }
        nd = c;
    }
    void* base = nd.ptr;
    // Launch geometry: as in qlgpu_create, at most one CTA per SM and one mode per pair of groups.
    int warps = 8;
    while (warps > 1 && var.smem(warps) > (size_t)nd.smem_optin) warps >>= 1;
    const size_t smem = var.smem(warps);
    if (ensure_smem_attr(var.kernel(), smem) != cudaSuccess)
        return fail(nullptr, QLGPU_ERR_CUDA, "shared memory request too large");
    const int modes_per_cta = warps * (32 / var.T) / 2;
    int grid = (nxy + modes_per_cta - 1) / modes_per_cta;
    if (grid > nd.sms) grid = nd.sms;
    if (grid > QLGPU_NOALLOC_MAX_GRID) grid = QLGPU_NOALLOC_MAX_GRID;
    const NoallocLayout L = noalloc_layout(p.NZ, nxy, nyh, nz, grid, var.PL);
    if (L.end > QLGPU_NOALLOC_SCRATCH_BYTES)
        return fail(nullptr, QLGPU_ERR_ARG, "case exceeds the 4 MiB no-allocation scratch");
    // Run constants (as qlgpu_create)
    DevParams d;
    std::memset(&d, 0, sizeof(d));
    d.nxy = nxy; d.nz = nz; d.NZ = p.NZ; d.nmf = nmf;
    d.q = p.q;
    d.Omega = p.model == QLGPU_MODEL_MHD_BQLIN ? 2.0 / 3.0 * p.q : p.omega;
    d.nu = p.nu; d.eta = p.eta;
    d.etanu = p.model == QLGPU_MODEL_MHD_BQLIN ? p.eta / p.nu : p.eta;
    d.cb = p.model == QLGPU_MODEL_MHD_BQLIN ? (p.eta / p.nu) * p.nu : p.eta;
    d.factored = (p.model == QLGPU_MODEL_MHD_BQLIN || p.viscosity_order / 2 == 1) ? 1 : 0;
    d.B0z = p.B0z;
    d.visc_half = p.viscosity_order / 2;
    d.ql = p.quasilinear ? 1 : 0;
    d.remap = p.remap ? 1 : 0;
    d.kzL = 2 * kPI / p.L[2];
    d.fac = 1.0 / p.NZ;
    const int Nx = p.nx, Ny = (p.ny / 2) * 2;
    d.rs_fac = 1.0 / (Ny * Nx) / (Ny * Nx);
    d.dt = p.dt;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* b = static_cast<unsigned char*>(base);
    noalloc_tables_kernel<<<32, 256, 0, st>>>(b, L, p.NZ, var.T, p.nx, p.ny, nz, 2 * kPI / p.L[0], 2 * kPI / p.L[1],
                                             d.kzL, kx0 ? 0 : 1);
    StageArgs A;
    std::memset(&A, 0, sizeof(A));
    A.lin_in = static_cast<const cplx*>(lin_in);
    A.lin_out = static_cast<cplx*>(lin_rhs);
    A.mf = const_cast<cplx*>(static_cast<const cplx*>(mf_in));  // read only in rhs mode
    A.Fmf_out = static_cast<cplx*>(mf_rhs);
    A.kx0 = kx0 ? const_cast<double*>(static_cast<const double*>(kx0)) : reinterpret_cast<double*>(b + L.kx0);
    A.ky = reinterpret_cast<const double*>(b + L.ky);
    A.kxi = reinterpret_cast<const int*>(b + L.kxi);
    A.kyi = reinterpret_cast<const int*>(b + L.kyi);
    A.tw = reinterpret_cast<const cplx*>(b + L.tw);
    A.ilap2 = reinterpret_cast<const double*>(b + L.il2);
    A.partials = reinterpret_cast<double*>(b + L.partials);
    A.gpartials = reinterpret_cast<double*>(b + L.gpartials);
    A.clk = reinterpret_cast<DevClock*>(b + L.clk);
    A.rhs_only = 1;
    A.linop_out = static_cast<double*>(linop);
    A.sc.t_off = t;
    A.sc.abs_time = 1;
    A.sc.dt_lin = dt_lin;
    var.launch(A, d, grid, 32 * warps, smem, st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(nullptr, QLGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return QLGPU_OK;
}
