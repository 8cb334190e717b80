// qlgpu_adjoint.cu -- gradient of the time-averaged Maxwell stress with
// respect to the initial fluctuation field: the forward MHD_BQlin run
// (RK3CN_Elin or RK3CN) with checkpoints, then the discrete adjoint of every step in
// reverse, with the stages of each checkpoint window recomputed
// (qlgpu_adjoint_maxwell in include/qlgpu.h; kernels in qlgpu_adjoint.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qlgpu.h"
#include "qlgpu_adjoint.cuh"
#include "qlgpu_batch_internal.h"
#include "qlgpu_handle.h"

using namespace qlgpu;

namespace {

struct AdjOps {
    void (*mf_pre)(const AdjMfArgs&, const DevParams&, cudaStream_t);
    void (*modes)(const AdjStageArgs&, const DevParams&, int nxy, cudaStream_t);
    void (*mf_post)(const double*, const cplx*, const DevParams&, cplx*, cudaStream_t);
    void (*jgrad)(const cplx*, const double*, const double*, const int*, const double*, const DevParams&, double,
                  const double*, double, cplx*, cudaStream_t);
    const void* modes_kernel;
    size_t modes_smem;
    // one launch for all seeds of a batch (seed = blockIdx.y)
    void (*mf_pre_s)(const AdjMfArgs&, const DevParams&, const AdjRevPos&, int, cudaStream_t);
    void (*modes_s)(const AdjStageArgs&, const DevParams&, const AdjRevPos&, int nxy, int, cudaStream_t);
    void (*mf_post_s)(const cplx*, const DevParams&, const AdjRevPos&, int, cudaStream_t);
    void (*jgrad_s)(const double*, const int*, const double*, const DevParams&, const AdjRevPos&, int, cudaStream_t);
    const void* modes_seeds_kernel;
};

template <int NZ>
void ops_mf_pre(const AdjMfArgs& A, const DevParams& P, cudaStream_t st) {
    adj_mf_pre_kernel<NZ><<<1, 128, 0, st>>>(A, P);
}
template <int NZ>
void ops_modes(const AdjStageArgs& A, const DevParams& P, int nxy, cudaStream_t st) {
    adj_modes_kernel<NZ><<<nxy, AdjGeom<NZ>::THREADS, AdjGeom<NZ>::BYTES, st>>>(A, P);
}
template <int NZ>
void ops_mf_post(const double* bsum, const cplx* tw, const DevParams& P, cplx* lamB, cudaStream_t st) {
    adj_mf_post_kernel<NZ><<<1, 64, 0, st>>>(bsum, tw, P, lamB);
}
template <int NZ>
void ops_jgrad(const cplx* U, const double* kx0, const double* ky, const int* kyi, const double* il2,
               const DevParams& P, double t, const double* t_dev, double w, cplx* lam, cudaStream_t st) {
    adj_jgrad_kernel<NZ><<<148, 256, 0, st>>>(U, kx0, ky, kyi, il2, P, t, t_dev, w, lam);
}
template <int NZ>
void ops_mf_pre_s(const AdjMfArgs& M, const DevParams& P, const AdjRevPos& X, int ns, cudaStream_t st) {
    adj_mf_pre_seeds_kernel<NZ><<<dim3(1, ns), 128, 0, st>>>(M, P, X);
}
template <int NZ>
void ops_modes_s(const AdjStageArgs& A, const DevParams& P, const AdjRevPos& X, int nxy, int ns, cudaStream_t st) {
    adj_modes_seeds_kernel<NZ><<<dim3(nxy, ns), AdjGeom<NZ>::THREADS, AdjGeom<NZ>::BYTES, st>>>(A, P, X);
}
template <int NZ>
void ops_mf_post_s(const cplx* tw, const DevParams& P, const AdjRevPos& X, int ns, cudaStream_t st) {
    adj_mf_post_seeds_kernel<NZ><<<dim3(1, ns), 64, 0, st>>>(tw, P, X);
}
template <int NZ>
void ops_jgrad_s(const double* ky, const int* kyi, const double* il2, const DevParams& P, const AdjRevPos& X, int ns,
                 cudaStream_t st) {
    adj_jgrad_seeds_kernel<NZ><<<dim3(148, ns), 256, 0, st>>>(ky, kyi, il2, P, X);
}
template <int NZ>
AdjOps make_ops() {
    AdjOps o;
    o.mf_pre = &ops_mf_pre<NZ>;
    o.modes = &ops_modes<NZ>;
    o.mf_post = &ops_mf_post<NZ>;
    o.jgrad = &ops_jgrad<NZ>;
    o.modes_kernel = reinterpret_cast<const void*>(&adj_modes_kernel<NZ>);
    o.modes_smem = AdjGeom<NZ>::BYTES;
    o.mf_pre_s = &ops_mf_pre_s<NZ>;
    o.modes_s = &ops_modes_s<NZ>;
    o.mf_post_s = &ops_mf_post_s<NZ>;
    o.jgrad_s = &ops_jgrad_s<NZ>;
    o.modes_seeds_kernel = reinterpret_cast<const void*>(&adj_modes_seeds_kernel<NZ>);
    return o;
}
bool pick_ops(int NZ, AdjOps* o) {
    switch (NZ) {
        case 16: *o = make_ops<16>(); return true;
        case 32: *o = make_ops<32>(); return true;
        case 64: *o = make_ops<64>(); return true;
        case 128: *o = make_ops<128>(); return true;
        case 256: *o = make_ops<256>(); return true;
        default: return false;
    }
}

int afail(qlgpu_t* h, int code, const std::string& msg) {
    h->err = msg;
    return code;
}

int adj_integ(const qlgpu_t* h) { return h->p.integrator == QLGPU_INTEG_RK3CN ? INTEG_CN : INTEG_EXP; }

// the stage-start record of RK3CN copies the clock's bytes from t_old (CnRec's layout)
static_assert(offsetof(DevClock, dtlin_old) == offsetof(DevClock, t_old) + 8 &&
                  offsetof(DevClock, old_init) == offsetof(DevClock, t_old) + 16 && sizeof(CnRec) == 24,
              "CnRec mirrors DevClock from t_old");

#define QA_CK(call)                                                                                \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return afail(h, QLGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device allocations of one call, freed on every exit path.
struct Pool {
    std::vector<void*> ptrs;
    ~Pool() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t get(T** out, size_t count) {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, sizeof(T) * (count ? count : 1));
        if (e == cudaSuccess) {
            ptrs.push_back(p);
            e = cudaMemset(p, 0, sizeof(T) * (count ? count : 1));
        }
        *out = static_cast<T*>(p);
        return e;
    }
};


// One seed's adjoint: the buffers and the position of its sweeps.  The phases
// below only enqueue work on the handle's stream (except where a host copy is
// needed), so several jobs, one per handle, advance together on their own
// streams: qlgpu_adjoint_maxwell_batch interleaves them phase by phase.
struct AdjJob {
    qlgpu_t* h = nullptr;
    AdjOps ops{};
    int N = 0, C = 0, NC = 0;
    size_t nlin = 0, nmfe = 0, nxy = 0;
    Pool pool;
    cplx *ck_lin = nullptr, *ck_mf = nullptr;
    double* ck_kx0 = nullptr;
    DevClock* ck_clk = nullptr;
    cplx *fin_lin = nullptr, *fin_mf = nullptr;
    double* fin_kx0 = nullptr;
    DevClock* fin_clk = nullptr;
    int fin_cur = 0;
    std::vector<double> rec;
    DevClock cend{};
    cplx *stU = nullptr, *stB = nullptr, *postU = nullptr;
    double *kx_pre = nullptr, *kx_post = nullptr, *t_pre = nullptr;
    CnRec* cn_pre = nullptr;  // RK3CN: the old-operator clock fields at every stage start of the window
    cplx *lamU[2] = {nullptr, nullptr}, *lamB[2] = {nullptr, nullptr};
    cplx *lamF[2] = {nullptr, nullptr}, *lamG[2] = {nullptr, nullptr};
    double *prof = nullptr, *bpart = nullptr, *bsum = nullptr;
    int iu = 0, ib = 0;
    double J = 0.0;
    // full-window graphs (replayed for every window of C steps when C is even)
    cudaGraphExec_t g_fwd = nullptr, g_rec = nullptr, g_bwd = nullptr;
    ~AdjJob() {
        for (cudaGraphExec_t g : {g_fwd, g_rec, g_bwd})
            if (g) cudaGraphExecDestroy(g);
    }
};

int adj_begin(AdjJob& j, qlgpu_t* h, double t0, const double* lin0, const double* mf0, const double* kx0, int nsteps,
              int checkpoint_every) {
    j.h = h;
    if (!lin0 || !mf0 || nsteps < 1 || checkpoint_every < 1)
        return afail(h, QLGPU_ERR_ARG, "null argument, nsteps < 1 or checkpoint_every < 1");
    if (h->p.model != QLGPU_MODEL_MHD_BQLIN)
        return afail(h, QLGPU_ERR_UNSUPPORTED, "the adjoint covers MHD_BQlin (RK3CN_Elin or RK3CN)");
    if (h->noise_f != 0.0 || h->cfl > 0) return afail(h, QLGPU_ERR_UNSUPPORTED, "the adjoint runs at fixed dt, no noise");
    if (!pick_ops(h->NZ, &j.ops)) return afail(h, QLGPU_ERR_UNSUPPORTED, "unsupported NZ");
    QA_CK(cudaSetDevice(h->device));
    QA_CK(ensure_smem_attr(j.ops.modes_kernel, j.ops.modes_smem));
    QA_CK(ensure_smem_attr(j.ops.modes_seeds_kernel, j.ops.modes_smem));
    int rc = qlgpu_set_state(h, t0, lin0, mf0, kx0);
    if (rc) return rc;
    j.N = nsteps;
    j.C = std::min(checkpoint_every, nsteps);
    j.NC = (j.N + j.C - 1) / j.C;
    j.nlin = (size_t)h->nxy * 4 * h->nz;
    j.nmfe = (size_t)h->nmf * h->nz;
    j.nxy = (size_t)h->nxy;
    QA_CK(j.pool.get(&j.ck_lin, (size_t)j.NC * j.nlin));
    QA_CK(j.pool.get(&j.ck_mf, (size_t)j.NC * j.nmfe));
    QA_CK(j.pool.get(&j.ck_kx0, (size_t)j.NC * j.nxy));
    QA_CK(j.pool.get(&j.ck_clk, (size_t)j.NC));
    QA_CK(j.pool.get(&j.fin_lin, j.nlin));
    QA_CK(j.pool.get(&j.fin_mf, j.nmfe));
    QA_CK(j.pool.get(&j.fin_kx0, j.nxy));
    QA_CK(j.pool.get(&j.fin_clk, 1));
    if (h->diag_cap < j.N) {
        if (h->d_diag) cudaFree(h->d_diag);
        h->d_diag = nullptr;
        h->diag_cap = 0;
        QA_CK(cudaMalloc(&h->d_diag, sizeof(double) * 15 * (size_t)j.N));
        h->diag_cap = j.N;
    }
    const int zero = 0;
    QA_CK(cudaMemcpyAsync(&h->d_clk->ndiag, &zero, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    h->dp.tv_interval = h->p.dt;  // the AM_b record of every step
    return QLGPU_OK;
}

// checkpoint c of the forward sweep (the state at the start of window c)
int adj_checkpoint(AdjJob& j, int c) {
    qlgpu_t* h = j.h;
    cudaStream_t st = h->stream;
    QA_CK(cudaMemcpyAsync(j.ck_lin + c * j.nlin, h->d_lin[h->cur], j.nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.ck_mf + c * j.nmfe, h->d_mf, j.nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.ck_kx0 + c * j.nxy, h->d_kx0, j.nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.ck_clk + c, h->d_clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, st));
    return QLGPU_OK;
}

int adj_forward_step(AdjJob& j, int) {
    qlgpu_enqueue_step(j.h, nullptr, nullptr);
    return QLGPU_OK;
}

int adj_forward_end(AdjJob& j) {
    qlgpu_t* h = j.h;
    cudaStream_t st = h->stream;
    QA_CK(cudaGetLastError());
    j.rec.assign((size_t)15 * j.N, 0.0);
    QA_CK(cudaMemcpyAsync(j.rec.data(), h->d_diag, j.rec.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    QA_CK(cudaMemcpyAsync(&j.cend, h->d_clk, sizeof(DevClock), cudaMemcpyDeviceToHost, st));
    QA_CK(cudaMemcpyAsync(j.fin_lin, h->d_lin[h->cur], j.nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.fin_mf, h->d_mf, j.nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.fin_kx0, h->d_kx0, j.nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.fin_clk, h->d_clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, st));
    j.fin_cur = h->cur;
    return QLGPU_OK;
}

int adj_alloc_backward(AdjJob& j);

// after the stream is synchronised: J and the backward buffers
int adj_forward_finish(AdjJob& j) {
    qlgpu_t* h = j.h;
    h->dp.tv_interval = 0.0;
    if (j.cend.status & (QLGPU_STATUS_NONFINITE | QLGPU_STATUS_UNSTABLE))
        return afail(h, QLGPU_ERR_STATUS, "forward run: non-finite or unstable solution");
    if (j.cend.ndiag != j.N) return afail(h, QLGPU_ERR_STATUS, "forward run: missing diagnostic records");
    double s = 0.0;
    for (int n = 0; n < j.N; ++n) s += j.rec[(size_t)15 * n + 8];  // AM_b (MHD_BQlin.cpp:459)
    j.J = s / j.N;
    return adj_alloc_backward(j);
}

int adj_alloc_backward(AdjJob& j) {
    qlgpu_t* h = j.h;
    QA_CK(j.pool.get(&j.stU, (size_t)j.C * 3 * j.nlin));
    QA_CK(j.pool.get(&j.stB, (size_t)j.C * 3 * j.nmfe));
    QA_CK(j.pool.get(&j.postU, j.nlin));
    QA_CK(j.pool.get(&j.kx_pre, (size_t)j.C * j.nxy));
    QA_CK(j.pool.get(&j.kx_post, j.nxy));
    QA_CK(j.pool.get(&j.t_pre, (size_t)j.C + 1));
    QA_CK(j.pool.get(&j.cn_pre, (size_t)j.C * 3));
    for (int i = 0; i < 2; ++i) {
        QA_CK(j.pool.get(&j.lamU[i], j.nlin));
        QA_CK(j.pool.get(&j.lamB[i], j.nmfe));
        QA_CK(j.pool.get(&j.lamF[i], j.nlin));
        QA_CK(j.pool.get(&j.lamG[i], j.nmfe));
    }
    QA_CK(j.pool.get(&j.prof, (size_t)5 * h->NZ));
    QA_CK(j.pool.get(&j.bpart, (size_t)3 * h->NZ * j.nxy));
    QA_CK(j.pool.get(&j.bsum, (size_t)3 * h->NZ));
    return QLGPU_OK;
}

int window_steps(const AdjJob& j, int w) { return std::min(j.N, w * j.C + j.C) - w * j.C; }

// restore checkpoint w before recomputing its window
int adj_window_begin(AdjJob& j, int w) {
    qlgpu_t* h = j.h;
    cudaStream_t st = h->stream;
    h->cur = 0;
    QA_CK(cudaMemcpyAsync(h->d_lin[0], j.ck_lin + w * j.nlin, j.nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_mf, j.ck_mf + w * j.nmfe, j.nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_kx0, j.ck_kx0 + w * j.nxy, j.nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_clk, j.ck_clk + w, sizeof(DevClock), cudaMemcpyDeviceToDevice, st));
    // the mean-field profile cache holds a later mean field: recompute it in the first stage
    const int zero = 0;
    QA_CK(cudaMemcpyAsync(&h->d_clk->mfr_valid, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
    return QLGPU_OK;
}

// recompute step n of the window, recording every stage's input
int adj_recompute_step(AdjJob& j, int n) {
    qlgpu_t* h = j.h;
    cudaStream_t st = h->stream;
    QA_CK(cudaMemcpyAsync(j.kx_pre + n * j.nxy, h->d_kx0, j.nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.t_pre + n, &h->d_clk->t, sizeof(double), cudaMemcpyDeviceToDevice, st));
    cudaError_t herr = cudaSuccess;
    qlgpu_enqueue_step(h, nullptr, [&](int s) {
        const cudaError_t e1 = cudaMemcpyAsync(j.stU + ((size_t)n * 3 + s) * j.nlin, h->d_lin[h->cur],
                                               j.nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
        const cudaError_t e2 = cudaMemcpyAsync(j.stB + ((size_t)n * 3 + s) * j.nmfe, h->d_mf, j.nmfe * sizeof(cplx),
                                               cudaMemcpyDeviceToDevice, st);
        // t_old, dtlin_old, old_init of the clock (the layout of CnRec)
        const cudaError_t e3 = cudaMemcpyAsync(j.cn_pre + (size_t)n * 3 + s, &h->d_clk->t_old, sizeof(CnRec),
                                               cudaMemcpyDeviceToDevice, st);
        if (herr == cudaSuccess) herr = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
    });
    QA_CK(herr);
    return QLGPU_OK;
}

int adj_window_end(AdjJob& j, int w) {
    qlgpu_t* h = j.h;
    cudaStream_t st = h->stream;
    const int steps = window_steps(j, w);
    QA_CK(cudaMemcpyAsync(j.postU, h->d_lin[h->cur], j.nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.kx_post, h->d_kx0, j.nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(j.t_pre + steps, &h->d_clk->t, sizeof(double), cudaMemcpyDeviceToDevice, st));
    return QLGPU_OK;
}

// the adjoint of step n of a window of `steps` steps (stream-ordered after
// adj_window_end; the step times are read on the device from t_pre)
int adj_backward_step(AdjJob& j, int steps, int n) {
    qlgpu_t* h = j.h;
    cudaStream_t st = h->stream;
    const cplx* Upost = (n + 1 < steps) ? j.stU + (size_t)(n + 1) * 3 * j.nlin : j.postU;
    const double* kxa = (n + 1 < steps) ? j.kx_pre + (n + 1) * j.nxy : j.kx_post;
    // J = (1/N) sum AM_b(post-step state), recorded after the remap (main.cpp:122-130)
    j.ops.jgrad(Upost, kxa, h->d_ky, h->d_kyi, h->d_ilap2, h->dp, 0.0, j.t_pre + n + 1, 1.0 / j.N, j.lamU[j.iu], st);
    adj_remap_kernel<<<148, 256, 0, st>>>(j.kx_pre + n * j.nxy, kxa, h->nxy, h->nz, j.lamU[j.iu]);
    for (int s = 2; s >= 0; --s) {
        const StageConst& S = h->sc[s];
        AdjMfArgs M;
        std::memset(&M, 0, sizeof(M));
        M.B = j.stB + ((size_t)n * 3 + s) * j.nmfe;
        M.lamB_out = j.lamB[j.ib];
        M.lamG_out = (s == 2) ? nullptr : j.lamG[0];
        M.lamB_in = j.lamB[j.ib ^ 1];
        M.lamGp = (s == 0) ? nullptr : j.lamG[1];
        M.prof = j.prof;
        M.tw = h->d_tw;
        M.sc = S;
        M.integ = adj_integ(h);
        j.ops.mf_pre(M, h->dp, st);
        AdjStageArgs A;
        std::memset(&A, 0, sizeof(A));
        A.status = h->d_dbg;
        A.U = j.stU + ((size_t)n * 3 + s) * j.nlin;
        A.lamU_out = j.lamU[j.iu];
        A.lamF_out = (s == 2) ? nullptr : j.lamF[0];
        A.lamU_in = j.lamU[j.iu ^ 1];
        A.lamFp = (s == 0) ? nullptr : j.lamF[1];
        A.kx0 = j.kx_pre + n * j.nxy;
        A.ky = h->d_ky;
        A.kxi = h->d_kxi;
        A.kyi = h->d_kyi;
        A.ilap2 = h->d_ilap2;
        A.tw = h->d_tw;
        A.prof = j.prof;
        A.bpart = j.bpart;
        A.t_dev = j.t_pre + n;
        A.cn = j.cn_pre + (size_t)n * 3 + s;
        A.integ = adj_integ(h);
        A.sc = S;
        j.ops.modes(A, h->dp, h->nxy, st);
        const int nout = 3 * h->NZ;
        adj_bsum_kernel<<<(nout + 7) / 8, 256, 0, st>>>(j.bpart, h->nxy, nout, j.bsum);
        j.ops.mf_post(j.bsum, h->d_tw, h->dp, j.lamB[j.ib ^ 1], st);
        j.iu ^= 1;
        j.ib ^= 1;
        std::swap(j.lamF[0], j.lamF[1]);
        std::swap(j.lamG[0], j.lamG[1]);
    }
    QA_CK(cudaGetLastError());
    return QLGPU_OK;
}

// The reverse sweep of all seeds of a batch on one stream: the same kernels as
// adj_backward_step, each launched once with one grid row per seed.  Every
// seed's arithmetic is that of adj_backward_step (results bit for bit equal).
struct SeedReverse {
    qlgpu_t* h = nullptr;  // the first seed's handle: tables, parameters, error text
    AdjOps ops{};
    const AdjSeedBufs* d_seeds = nullptr;
    int nseeds = 0;
    int par = 0;  // stages reversed so far, mod 2
    size_t nlin = 0, nmfe = 0, nxy = 0;
    double weight = 0.0;
};

int adj_backward_step_seeds(SeedReverse& R, cudaStream_t st, int steps, int n) {
    qlgpu_t* h = R.h;
    const int ns = R.nseeds;
    AdjRevPos X;
    X.seeds = R.d_seeds;
    X.n = n;
    X.steps = steps;
    X.s = 2;
    X.par = R.par;
    X.nlin = (long long)R.nlin;
    X.nmfe = (long long)R.nmfe;
    X.nxy = (long long)R.nxy;
    X.weight = R.weight;
    R.ops.jgrad_s(h->d_ky, h->d_kyi, h->d_ilap2, h->dp, X, ns, st);
    adj_remap_seeds_kernel<<<dim3(148, ns), 256, 0, st>>>(X, h->nz);
    for (int s = 2; s >= 0; --s) {
        X.s = s;
        X.par = R.par;
        AdjMfArgs M;
        std::memset(&M, 0, sizeof(M));
        M.tw = h->d_tw;
        M.sc = h->sc[s];
        M.integ = adj_integ(h);
        R.ops.mf_pre_s(M, h->dp, X, ns, st);
        AdjStageArgs A;
        std::memset(&A, 0, sizeof(A));
        A.status = h->d_dbg;
        A.ky = h->d_ky;
        A.kxi = h->d_kxi;
        A.kyi = h->d_kyi;
        A.ilap2 = h->d_ilap2;
        A.tw = h->d_tw;
        A.integ = adj_integ(h);
        A.sc = h->sc[s];
        R.ops.modes_s(A, h->dp, X, h->nxy, ns, st);
        const int nout = 3 * h->NZ;
        adj_bsum_seeds_kernel<<<dim3((nout + 7) / 8, ns), 256, 0, st>>>(X, nout);
        R.ops.mf_post_s(h->d_tw, h->dp, X, ns, st);
        R.par ^= 1;
    }
    QA_CK(cudaGetLastError());
    return QLGPU_OK;
}

// gradients out, and the handle left at the end of the forward run
int adj_finish(AdjJob& j, double* grad_lin, double* grad_mf) {
    qlgpu_t* h = j.h;
    cudaStream_t st = h->stream;
    QA_CK(cudaMemcpyAsync(grad_lin, j.lamU[j.iu], j.nlin * sizeof(cplx), cudaMemcpyDeviceToHost, st));
    if (grad_mf) QA_CK(cudaMemcpyAsync(grad_mf, j.lamB[j.ib], j.nmfe * sizeof(cplx), cudaMemcpyDeviceToHost, st));
    h->cur = j.fin_cur;
    QA_CK(cudaMemcpyAsync(h->d_lin[h->cur], j.fin_lin, j.nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_mf, j.fin_mf, j.nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_kx0, j.fin_kx0, j.nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_clk, j.fin_clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, st));
    return QLGPU_OK;
}

int sync_job(AdjJob& j) {
    qlgpu_t* h = j.h;
    QA_CK(cudaStreamSynchronize(h->stream));
    return QLGPU_OK;
}

// The seeds' forward sweep and window recompute in the persistent batch kernel
// (one launch per window for all seeds, the recompute recording every stage's
// input through the kernel's record pointers); the reverse sweep on the batch's
// stream, every kernel launched once for all seeds (per seed on its handle's
// stream when the seeds differ in a parameter).  The batch's reduction order differs from
// the single-case kernel's, so each seed's results agree with
// qlgpu_adjoint_maxwell to round-off rather than bit for bit.
template <class F>
int capture(AdjJob& j, cudaGraphExec_t* out, F body);
int launch_graph(AdjJob& j, cudaGraphExec_t g);

// The reverse sweep runs once for all seeds (adj_backward_step_seeds) when the
// seeds share every parameter and the device; otherwise per seed.
bool same_setup(const qlgpu_t* a, const qlgpu_t* b) {
    const qlgpu_params &p = a->p, &r = b->p;
    return a->device == b->device && p.model == r.model && p.integrator == r.integrator && p.nx == r.nx &&
           p.ny == r.ny && p.NZ == r.NZ && p.L[0] == r.L[0] && p.L[1] == r.L[1] && p.L[2] == r.L[2] && p.q == r.q &&
           p.omega == r.omega && p.nu == r.nu && p.eta == r.eta && p.B0z == r.B0z &&
           p.viscosity_order == r.viscosity_order && p.dt == r.dt && p.remap == r.remap &&
           p.quasilinear == r.quasilinear;
}

struct BatchGuard {
    qlgpu_batch_t* b = nullptr;
    ~BatchGuard() {
        if (b) qlgpu_batch_destroy(b);
    }
};

int run_jobs_persistent(std::vector<AdjJob>& jobs, double t0, const double* lin0, const double* mf0, const double* kx0,
                        double* J, double* const* grad_lin, double* const* grad_mf) {
    const int nj = (int)jobs.size();
    const int N = jobs[0].N, C = jobs[0].C, NC = jobs[0].NC;
    qlgpu_t* h0 = jobs[0].h;
    qlgpu_t* h = h0;  // for QA_CK
    std::vector<qlgpu_params> ps(nj);
    for (int q = 0; q < nj; ++q) ps[q] = jobs[q].h->p;
    BatchGuard g;
    int rc = qlgpu_batch_create(ps.data(), nj, h0->device, &g.b);
    if (rc) {
        char buf[256];
        qlgpu_batch_last_error(nullptr, buf, sizeof(buf));
        return afail(h0, rc, std::string("adjoint batch: ") + buf);
    }
    qlgpu_batch_t* b = g.b;
    cudaStream_t bs = qlgpu_batch_cuda_stream(b);
    const size_t nlin = jobs[0].nlin, nmfe = jobs[0].nmfe, nxy = jobs[0].nxy;
    // reverse windows as graphs (C even keeps the ping-pong buffers in place across
    // windows) only with QLGPU_ADJ_GRAPH=1: at 16 seeds x 496 modes they measured
    // slower (3.9 s) than direct launches (3.4 s) for 2000 steps
    const char* genv = getenv("QLGPU_ADJ_GRAPH");
    const bool graphs = (C % 2 == 0) && genv && genv[0] == '1';
    for (int q = 0; q < nj; ++q) {
        rc = qlgpu_batch_set_state(b, q, t0, lin0 + q * 2 * nlin, mf0 + q * 2 * nmfe, kx0 ? kx0 + q * nxy : nullptr);
        if (rc) return afail(h0, rc, "adjoint batch: set_state");
    }
    // ---- forward sweep: checkpoints, then one launch per window with a record every step
    std::vector<double> recs((size_t)nj * C * 15);
    std::vector<int> nd(nj);
    std::vector<double> Js(nj, 0.0);
    for (int w = 0; w < NC; ++w) {
        const int steps = std::min(N, w * C + C) - w * C;
        for (int q = 0; q < nj; ++q) {
            AdjJob& j = jobs[q];
            BatchCaseDev d;
            qlgpu_batch_case_dev(b, q, &d);
            QA_CK(cudaMemcpyAsync(j.ck_lin + w * nlin, d.lin, nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, bs));
            QA_CK(cudaMemcpyAsync(j.ck_mf + w * nmfe, d.mf, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, bs));
            QA_CK(cudaMemcpyAsync(j.ck_kx0 + w * nxy, d.kx0, nxy * sizeof(double), cudaMemcpyDeviceToDevice, bs));
            QA_CK(cudaMemcpyAsync(j.ck_clk + w, d.clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, bs));
        }
        rc = qlgpu_batch_step(b, steps, 1, recs.data(), C, nd.data());
        if (rc) {
            char buf[256];
            qlgpu_batch_last_error(b, buf, sizeof(buf));
            return afail(h0, rc, std::string("adjoint forward sweep: ") + buf);
        }
        for (int q = 0; q < nj; ++q) {
            if (nd[q] != steps) return afail(h0, QLGPU_ERR_STATUS, "forward run: missing diagnostic records");
            for (int n = 0; n < steps; ++n) Js[q] += recs[((size_t)q * C + n) * 15 + 8];  // AM_b
        }
    }
    for (int q = 0; q < nj; ++q) {
        AdjJob& j = jobs[q];
        j.J = Js[q] / N;
        BatchCaseDev d;
        qlgpu_batch_case_dev(b, q, &d);
        QA_CK(cudaMemcpyAsync(j.fin_lin, d.lin, nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, bs));
        QA_CK(cudaMemcpyAsync(j.fin_mf, d.mf, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, bs));
        QA_CK(cudaMemcpyAsync(j.fin_kx0, d.kx0, nxy * sizeof(double), cudaMemcpyDeviceToDevice, bs));
        QA_CK(cudaMemcpyAsync(j.fin_clk, d.clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, bs));
        j.fin_cur = 0;
        j.h->dp.tv_interval = 0.0;
        rc = adj_alloc_backward(j);
        if (rc) return rc;
    }
    // the reverse sweep: one launch per kernel for all seeds (default), or every seed on its
    // own stream (QLGPU_ADJ_REVERSE=streams, or seeds that differ in a parameter)
    const char* renv = getenv("QLGPU_ADJ_REVERSE");
    bool seeds_rev = !(renv && std::string(renv) == "streams");
    for (int q = 1; q < nj; ++q)
        if (!same_setup(jobs[q].h, h0)) seeds_rev = false;
    Pool tab;
    SeedReverse R;
    if (seeds_rev) {
        std::vector<AdjSeedBufs> hb(nj);
        for (int q = 0; q < nj; ++q) {
            const AdjJob& j = jobs[q];
            AdjSeedBufs& e = hb[q];
            e.cn_pre = adj_integ(j.h) == INTEG_CN ? j.cn_pre : nullptr;
            e.stU = j.stU;
            e.stB = j.stB;
            e.postU = j.postU;
            e.kx_pre = j.kx_pre;
            e.kx_post = j.kx_post;
            e.t_pre = j.t_pre;
            for (int i = 0; i < 2; ++i) {
                e.lamU[i] = j.lamU[i];
                e.lamB[i] = j.lamB[i];
                e.lamF[i] = j.lamF[i];
                e.lamG[i] = j.lamG[i];
            }
            e.prof = j.prof;
            e.bpart = j.bpart;
            e.bsum = j.bsum;
        }
        AdjSeedBufs* d = nullptr;
        QA_CK(tab.get(&d, (size_t)nj));
        QA_CK(cudaMemcpy(d, hb.data(), sizeof(AdjSeedBufs) * nj, cudaMemcpyHostToDevice));
        R.h = h0;
        R.ops = jobs[0].ops;
        R.d_seeds = d;
        R.nseeds = nj;
        R.nlin = nlin;
        R.nmfe = nmfe;
        R.nxy = nxy;
        R.weight = 1.0 / N;
    }
    // ---- reverse sweep, window by window
    cudaEvent_t ev_b = nullptr;
    std::vector<cudaEvent_t> ev_h(nj, nullptr);
    struct EvGuard {
        cudaEvent_t* e;
        std::vector<cudaEvent_t>* v;
        ~EvGuard() {
            if (*e) cudaEventDestroy(*e);
            for (cudaEvent_t x : *v)
                if (x) cudaEventDestroy(x);
        }
    } evg{&ev_b, &ev_h};
    QA_CK(cudaEventCreateWithFlags(&ev_b, cudaEventDisableTiming));
    for (int q = 0; q < nj; ++q) QA_CK(cudaEventCreateWithFlags(&ev_h[q], cudaEventDisableTiming));
    const int zero = 0;
    for (int w = NC - 1; w >= 0; --w) {
        const int steps = std::min(N, w * C + C) - w * C;
        // the previous window's reverse steps must be done with stU before the recompute rewrites it
        if (w != NC - 1 && !seeds_rev)
            for (int q = 0; q < nj; ++q) {
                QA_CK(cudaEventRecord(ev_h[q], jobs[q].h->stream));
                QA_CK(cudaStreamWaitEvent(bs, ev_h[q], 0));
            }
        for (int q = 0; q < nj; ++q) {
            AdjJob& j = jobs[q];
            BatchCaseDev d;
            qlgpu_batch_case_dev(b, q, &d);
            QA_CK(cudaMemcpyAsync(d.lin, j.ck_lin + w * nlin, nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, bs));
            QA_CK(cudaMemcpyAsync(d.mf, j.ck_mf + w * nmfe, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, bs));
            QA_CK(cudaMemcpyAsync(d.kx0, j.ck_kx0 + w * nxy, nxy * sizeof(double), cudaMemcpyDeviceToDevice, bs));
            QA_CK(cudaMemcpyAsync(d.clk, j.ck_clk + w, sizeof(DevClock), cudaMemcpyDeviceToDevice, bs));
            // the mean-field profile cache holds a later mean field: recompute it in the first stage
            QA_CK(cudaMemcpyAsync(&d.clk->mfr_valid, &zero, sizeof(int), cudaMemcpyHostToDevice, bs));
            qlgpu_batch_set_record(b, q, j.stU, j.stB, j.kx_pre, j.t_pre, j.cn_pre);
        }
        rc = qlgpu_batch_step(b, steps, 0, nullptr, 0, nullptr);
        if (rc) {
            char buf[256];
            qlgpu_batch_last_error(b, buf, sizeof(buf));
            return afail(h0, rc, std::string("adjoint recompute: ") + buf);
        }
        for (int q = 0; q < nj; ++q) {
            AdjJob& j = jobs[q];
            BatchCaseDev d;
            qlgpu_batch_case_dev(b, q, &d);  // the buffer parity after the launch
            QA_CK(cudaMemcpyAsync(j.postU, d.lin, nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, bs));
            QA_CK(cudaMemcpyAsync(j.kx_post, d.kx0, nxy * sizeof(double), cudaMemcpyDeviceToDevice, bs));
            QA_CK(cudaMemcpyAsync(j.t_pre + steps, &d.clk->t, sizeof(double), cudaMemcpyDeviceToDevice, bs));
        }
        if (seeds_rev) {
            for (int n = steps - 1; n >= 0; --n) {
                rc = adj_backward_step_seeds(R, bs, steps, n);
                if (rc) return rc;
            }
            continue;
        }
        QA_CK(cudaEventRecord(ev_b, bs));
        for (int q = 0; q < nj; ++q) {
            AdjJob& j = jobs[q];
            QA_CK(cudaStreamWaitEvent(j.h->stream, ev_b, 0));
            if (graphs && steps == C) {
                // a full window's reverse steps: 14 small kernels per step, one graph launch
                if (!j.g_bwd) {
                    rc = capture(j, &j.g_bwd, [&] {
                        for (int n = C - 1; n >= 0; --n) {
                            int r = adj_backward_step(j, C, n);
                            if (r) return r;
                        }
                        return (int)QLGPU_OK;
                    });
                    if (rc) return rc;
                }
                rc = launch_graph(j, j.g_bwd);
                if (rc) return rc;
                continue;
            }
            for (int n = steps - 1; n >= 0; --n) {
                rc = adj_backward_step(j, steps, n);
                if (rc) return rc;
            }
        }
    }
    if (seeds_rev) {
        // every seed's buffers in the state adj_backward_step would have left them
        QA_CK(cudaEventRecord(ev_b, bs));
        for (int q = 0; q < nj; ++q) {
            AdjJob& j = jobs[q];
            j.iu = j.ib = R.par;
            if (R.par) {
                std::swap(j.lamF[0], j.lamF[1]);
                std::swap(j.lamG[0], j.lamG[1]);
            }
            QA_CK(cudaStreamWaitEvent(j.h->stream, ev_b, 0));
        }
    }
    for (int q = 0; q < nj; ++q) qlgpu_batch_set_record(b, q, nullptr, nullptr, nullptr, nullptr);
    for (int q = 0; q < nj; ++q) {
        rc = adj_finish(jobs[q], grad_lin[q], grad_mf ? grad_mf[q] : nullptr);
        if (rc) return rc;
    }
    for (int q = 0; q < nj; ++q) {
        rc = sync_job(jobs[q]);
        if (rc) return rc;
    }
    QA_CK(cudaStreamSynchronize(bs));
    for (int q = 0; q < nj; ++q) J[q] = jobs[q].J;
    return QLGPU_OK;
}

// Capture `body` on the job's stream into an executable graph.
template <class F>
int capture(AdjJob& j, cudaGraphExec_t* out, F body) {
    qlgpu_t* h = j.h;
    QA_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    QA_CK(e);
    const cudaError_t e2 = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    QA_CK(e2);
    return QLGPU_OK;
}

int launch_graph(AdjJob& j, cudaGraphExec_t g) {
    qlgpu_t* h = j.h;
    QA_CK(cudaGraphLaunch(g, h->stream));
    return QLGPU_OK;
}

// All jobs phase by phase; every job's work goes to its own handle's stream.
// Optionally a window of C steps (forward, recompute, reverse) is one graph
// launch per job after its first capture: the buffers a window uses do not
// depend on the window, and with C even the adjoint's ping-pong buffers are
// back in the same order after every window, so the graphs replay unchanged.
int run_jobs(std::vector<AdjJob>& jobs, double* J, double* const* grad_lin, double* const* grad_mf) {
    const int nj = (int)jobs.size();
    const int N = jobs[0].N, C = jobs[0].C, NC = jobs[0].NC;
    // opt-in (QLGPU_ADJ_GRAPH=1): at 16 seeds x 496 modes the graphs measured slower
    // (5.4 s) than direct launches (3.5 s) for 2000 steps
    const char* env = getenv("QLGPU_ADJ_GRAPH");
    const bool graphs = (C % 2 == 0) && env && env[0] == '1';
#define QA_ALL(expr)                                    \
    for (int q_ = 0; q_ < nj; ++q_) {                   \
        AdjJob& jj = jobs[q_];                          \
        (void)jj;                                       \
        int rc_ = (expr);                               \
        if (rc_) return rc_;                            \
    }
    auto fwd_window = [&](AdjJob& j, int steps) -> int {
        for (int n = 0; n < steps; ++n) {
            int rc = adj_forward_step(j, n);
            if (rc) return rc;
        }
        return QLGPU_OK;
    };
    auto rec_window = [&](AdjJob& j, int w, int steps) -> int {
        for (int n = 0; n < steps; ++n) {
            int rc = adj_recompute_step(j, n);
            if (rc) return rc;
        }
        return adj_window_end(j, w);
    };
    auto bwd_window = [&](AdjJob& j, int steps) -> int {
        for (int n = steps - 1; n >= 0; --n) {
            int rc = adj_backward_step(j, steps, n);
            if (rc) return rc;
        }
        return QLGPU_OK;
    };
    for (int w = 0; w < NC; ++w) {
        const int steps = std::min(N, w * C + C) - w * C;
        QA_ALL(adj_checkpoint(jj, w));
        if (graphs && steps == C) {
            QA_ALL(jj.g_fwd ? QLGPU_OK : capture(jj, &jj.g_fwd, [&] { return fwd_window(jj, C); }));
            QA_ALL(launch_graph(jj, jj.g_fwd));
        } else {
            for (int n = 0; n < steps; ++n) QA_ALL(adj_forward_step(jj, n));
        }
    }
    QA_ALL(adj_forward_end(jj));
    QA_ALL(sync_job(jj));
    QA_ALL(adj_forward_finish(jj));
    for (int w = NC - 1; w >= 0; --w) {
        const int steps = std::min(N, w * C + C) - w * C;
        QA_ALL(adj_window_begin(jj, w));
        if (graphs && steps == C) {
            QA_ALL(jj.g_rec ? QLGPU_OK : capture(jj, &jj.g_rec, [&] { return rec_window(jj, w, C); }));
            QA_ALL(launch_graph(jj, jj.g_rec));
            QA_ALL(jj.g_bwd ? QLGPU_OK : capture(jj, &jj.g_bwd, [&] { return bwd_window(jj, C); }));
            QA_ALL(launch_graph(jj, jj.g_bwd));
        } else {
            for (int n = 0; n < steps; ++n) QA_ALL(adj_recompute_step(jj, n));
            QA_ALL(adj_window_end(jj, w));
            for (int n = steps - 1; n >= 0; --n) QA_ALL(adj_backward_step(jj, steps, n));
        }
    }
    for (int q = 0; q < nj; ++q) {
        int rc = adj_finish(jobs[q], grad_lin[q], grad_mf ? grad_mf[q] : nullptr);
        if (rc) return rc;
    }
    QA_ALL(sync_job(jj));
#undef QA_ALL
    for (int q = 0; q < nj; ++q) J[q] = jobs[q].J;
    return QLGPU_OK;
}

}  // namespace

extern "C" int qlgpu_adjoint_maxwell(qlgpu_t* h, double t0, const double* lin0, const double* mf0,
                                     const double* kx0, int nsteps, int checkpoint_every, double* J,
                                     double* grad_lin, double* grad_mf) {
    if (!h) return QLGPU_ERR_ARG;
    if (!J || !grad_lin) return afail(h, QLGPU_ERR_ARG, "null argument");
    std::vector<AdjJob> jobs(1);
    int rc = adj_begin(jobs[0], h, t0, lin0, mf0, kx0, nsteps, checkpoint_every);
    if (rc) return rc;
    double* gl[1] = {grad_lin};
    double* gm[1] = {grad_mf};
    rc = run_jobs(jobs, J, gl, grad_mf ? gm : nullptr);
    return rc ? rc : qlgpu_debug_verify(h);
}

extern "C" int qlgpu_adjoint_maxwell_batch(qlgpu_t* const* handles, int nseeds, double t0, const double* lin0,
                                           const double* mf0, const double* kx0, int nsteps, int checkpoint_every,
                                           double* J, double* grad_lin, double* grad_mf) {
    if (!handles || nseeds < 1 || !handles[0]) return QLGPU_ERR_ARG;
    qlgpu_t* h0 = handles[0];
    if (!lin0 || !mf0 || !J || !grad_lin) return afail(h0, QLGPU_ERR_ARG, "null argument");
    for (int q = 0; q < nseeds; ++q) {
        if (!handles[q]) return afail(h0, QLGPU_ERR_ARG, "null handle");
        for (int r = 0; r < q; ++r)
            if (handles[r] == handles[q]) return afail(h0, QLGPU_ERR_ARG, "each seed needs its own handle");
        if (handles[q]->nxy != h0->nxy || handles[q]->nz != h0->nz || handles[q]->nmf != h0->nmf)
            return afail(h0, QLGPU_ERR_ARG, "handles of a batch must have the same dimensions");
    }
    const size_t nlin = (size_t)h0->nxy * 4 * h0->nz, nmfe = (size_t)h0->nmf * h0->nz;
    std::vector<AdjJob> jobs(nseeds);
    std::vector<double*> gl(nseeds), gm(nseeds);
    for (int q = 0; q < nseeds; ++q) {
        int rc = adj_begin(jobs[q], handles[q], t0, lin0 + q * 2 * nlin, mf0 + q * 2 * nmfe,
                           kx0 ? kx0 + q * (size_t)h0->nxy : nullptr, nsteps, checkpoint_every);
        if (rc) {
            if (handles[q] != h0) h0->err = handles[q]->err;
            return rc;
        }
        gl[q] = grad_lin + q * 2 * nlin;
        gm[q] = grad_mf ? grad_mf + q * 2 * nmfe : nullptr;
    }
    // default: forward sweep and recompute of all seeds in the persistent batch kernel;
    // QLGPU_ADJ_BATCH=streams interleaves the single-case path of every seed on its stream
    // (results bit-identical to qlgpu_adjoint_maxwell) from one host thread (threads per
    // seed were slower: their launches contend in the driver)
    const char* mode = getenv("QLGPU_ADJ_BATCH");
    const bool streams = mode && std::string(mode) == "streams";
    int rc = streams ? run_jobs(jobs, J, gl.data(), grad_mf ? gm.data() : nullptr)
                     : run_jobs_persistent(jobs, t0, lin0, mf0, kx0, J, gl.data(), grad_mf ? gm.data() : nullptr);
    for (int q = 0; q < nseeds && !rc; ++q) rc = qlgpu_debug_verify(handles[q]);
    if (rc) {
        for (int q = 0; q < nseeds; ++q)
            if (!handles[q]->err.empty() && handles[q] != h0) h0->err = handles[q]->err;
    }
    return rc;
}
