// qlgpu_adjoint.cu -- gradient of the time-averaged Maxwell stress with
// respect to the initial fluctuation field: the forward MHD_BQlin /
// RK3CN_Elin run with checkpoints, then the discrete adjoint of every step in
// reverse, with the stages of each checkpoint window recomputed
// (qlgpu_adjoint_maxwell in include/qlgpu.h; kernels in qlgpu_adjoint.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qlgpu.h"
#include "qlgpu_adjoint.cuh"
#include "qlgpu_handle.h"

using namespace qlgpu;

namespace {

struct AdjOps {
    void (*mf_pre)(const AdjMfArgs&, const DevParams&, cudaStream_t);
    void (*modes)(const AdjStageArgs&, const DevParams&, int nxy, cudaStream_t);
    void (*mf_post)(const double*, const cplx*, const DevParams&, cplx*, cudaStream_t);
    void (*jgrad)(const cplx*, const double*, const double*, const int*, const double*, const DevParams&, double,
                  double, cplx*, cudaStream_t);
    const void* modes_kernel;
    size_t modes_smem;
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
               const DevParams& P, double t, double w, cplx* lam, cudaStream_t st) {
    adj_jgrad_kernel<NZ><<<148, 256, 0, st>>>(U, kx0, ky, kyi, il2, P, t, w, lam);
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

}  // namespace

extern "C" int qlgpu_adjoint_maxwell(qlgpu_t* h, double t0, const double* lin0, const double* mf0,
                                     const double* kx0, int nsteps, int checkpoint_every, double* J,
                                     double* grad_lin, double* grad_mf) {
    if (!h) return QLGPU_ERR_ARG;
    if (!lin0 || !mf0 || !J || !grad_lin || nsteps < 1 || checkpoint_every < 1)
        return afail(h, QLGPU_ERR_ARG, "null argument, nsteps < 1 or checkpoint_every < 1");
    if (h->p.model != QLGPU_MODEL_MHD_BQLIN || h->p.integrator != QLGPU_INTEG_RK3CN_ELIN)
        return afail(h, QLGPU_ERR_UNSUPPORTED, "the adjoint covers MHD_BQlin with RK3CN_Elin");
    AdjOps ops;
    if (!pick_ops(h->NZ, &ops)) return afail(h, QLGPU_ERR_UNSUPPORTED, "unsupported NZ");
    QA_CK(cudaSetDevice(h->device));
    QA_CK(ensure_smem_attr(ops.modes_kernel, ops.modes_smem));
    int rc = qlgpu_set_state(h, t0, lin0, mf0, kx0);
    if (rc) return rc;
    const int N = nsteps, C = std::min(checkpoint_every, nsteps);
    const int NC = (N + C - 1) / C;
    const size_t nlin = (size_t)h->nxy * 4 * h->nz, nmfe = (size_t)h->nmf * h->nz, nxy = (size_t)h->nxy;
    cudaStream_t st = h->stream;
    Pool pool;
    cplx *ck_lin, *ck_mf;
    double* ck_kx0;
    DevClock* ck_clk;
    QA_CK(pool.get(&ck_lin, (size_t)NC * nlin));
    QA_CK(pool.get(&ck_mf, (size_t)NC * nmfe));
    QA_CK(pool.get(&ck_kx0, (size_t)NC * nxy));
    QA_CK(pool.get(&ck_clk, (size_t)NC));
    cplx *fin_lin, *fin_mf;
    double* fin_kx0;
    DevClock* fin_clk;
    QA_CK(pool.get(&fin_lin, nlin));
    QA_CK(pool.get(&fin_mf, nmfe));
    QA_CK(pool.get(&fin_kx0, nxy));
    QA_CK(pool.get(&fin_clk, 1));
    // ---- forward sweep: checkpoints and the AM_b record of every step
    {
        if (h->diag_cap < N) {
            if (h->d_diag) cudaFree(h->d_diag);
            h->d_diag = nullptr;
            h->diag_cap = 0;
            QA_CK(cudaMalloc(&h->d_diag, sizeof(double) * 15 * (size_t)N));
            h->diag_cap = N;
        }
        const int zero = 0;
        QA_CK(cudaMemcpyAsync(&h->d_clk->ndiag, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
        h->dp.tv_interval = h->p.dt;
        for (int n = 0; n < N; ++n) {
            if (n % C == 0) {
                const int c = n / C;
                QA_CK(cudaMemcpyAsync(ck_lin + c * nlin, h->d_lin[h->cur], nlin * sizeof(cplx),
                                      cudaMemcpyDeviceToDevice, st));
                QA_CK(cudaMemcpyAsync(ck_mf + c * nmfe, h->d_mf, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
                QA_CK(cudaMemcpyAsync(ck_kx0 + c * nxy, h->d_kx0, nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
                QA_CK(cudaMemcpyAsync(ck_clk + c, h->d_clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, st));
            }
            qlgpu_enqueue_step(h, nullptr, nullptr);
        }
        QA_CK(cudaGetLastError());
        std::vector<double> rec((size_t)15 * N);
        QA_CK(cudaMemcpyAsync(rec.data(), h->d_diag, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        DevClock c;
        QA_CK(cudaMemcpyAsync(&c, h->d_clk, sizeof(DevClock), cudaMemcpyDeviceToHost, st));
        QA_CK(cudaStreamSynchronize(st));
        h->dp.tv_interval = 0.0;
        if (c.status & (QLGPU_STATUS_NONFINITE | QLGPU_STATUS_UNSTABLE))
            return afail(h, QLGPU_ERR_STATUS, "forward run: non-finite or unstable solution");
        if (c.ndiag != N) return afail(h, QLGPU_ERR_STATUS, "forward run: missing diagnostic records");
        double s = 0.0;
        for (int n = 0; n < N; ++n) s += rec[(size_t)15 * n + 8];  // AM_b (MHD_BQlin.cpp:459)
        *J = s / N;
        QA_CK(cudaMemcpyAsync(fin_lin, h->d_lin[h->cur], nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(fin_mf, h->d_mf, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(fin_kx0, h->d_kx0, nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(fin_clk, h->d_clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, st));
    }
    const int fin_cur = h->cur;
    // ---- backward sweep
    cplx *stU, *stB, *postU;
    double *kx_pre, *kx_post, *t_pre;
    QA_CK(pool.get(&stU, (size_t)C * 3 * nlin));
    QA_CK(pool.get(&stB, (size_t)C * 3 * nmfe));
    QA_CK(pool.get(&postU, nlin));
    QA_CK(pool.get(&kx_pre, (size_t)C * nxy));
    QA_CK(pool.get(&kx_post, nxy));
    QA_CK(pool.get(&t_pre, (size_t)C + 1));
    cplx *lamU[2], *lamB[2], *lamF[2], *lamG[2];
    for (int i = 0; i < 2; ++i) {
        QA_CK(pool.get(&lamU[i], nlin));
        QA_CK(pool.get(&lamB[i], nmfe));
        QA_CK(pool.get(&lamF[i], nlin));
        QA_CK(pool.get(&lamG[i], nmfe));
    }
    double *prof, *bpart, *bsum;
    QA_CK(pool.get(&prof, (size_t)5 * h->NZ));
    QA_CK(pool.get(&bpart, (size_t)3 * h->NZ * nxy));
    QA_CK(pool.get(&bsum, (size_t)3 * h->NZ));
    int iu = 0, ib = 0;
    std::vector<double> tp((size_t)C + 1);
    for (int w = NC - 1; w >= 0; --w) {
        const int n0 = w * C, steps = std::min(N, n0 + C) - n0;
        // restore the checkpoint and recompute the window, recording the stage inputs
        h->cur = 0;
        QA_CK(cudaMemcpyAsync(h->d_lin[0], ck_lin + w * nlin, nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(h->d_mf, ck_mf + w * nmfe, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(h->d_kx0, ck_kx0 + w * nxy, nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(h->d_clk, ck_clk + w, sizeof(DevClock), cudaMemcpyDeviceToDevice, st));
        {
            // the mean-field profile cache holds a later mean field: recompute it in the first stage
            const int zero = 0;
            QA_CK(cudaMemcpyAsync(&h->d_clk->mfr_valid, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
        }
        cudaError_t herr = cudaSuccess;
        for (int n = 0; n < steps; ++n) {
            QA_CK(cudaMemcpyAsync(kx_pre + n * nxy, h->d_kx0, nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
            QA_CK(cudaMemcpyAsync(t_pre + n, &h->d_clk->t, sizeof(double), cudaMemcpyDeviceToDevice, st));
            qlgpu_enqueue_step(h, nullptr, [&](int s) {
                const cudaError_t e1 = cudaMemcpyAsync(stU + ((size_t)n * 3 + s) * nlin, h->d_lin[h->cur],
                                                       nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
                const cudaError_t e2 = cudaMemcpyAsync(stB + ((size_t)n * 3 + s) * nmfe, h->d_mf,
                                                       nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
                if (herr == cudaSuccess) herr = e1 != cudaSuccess ? e1 : e2;
            });
        }
        QA_CK(herr);
        QA_CK(cudaMemcpyAsync(postU, h->d_lin[h->cur], nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(kx_post, h->d_kx0, nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(t_pre + steps, &h->d_clk->t, sizeof(double), cudaMemcpyDeviceToDevice, st));
        QA_CK(cudaMemcpyAsync(tp.data(), t_pre, sizeof(double) * (steps + 1), cudaMemcpyDeviceToHost, st));
        QA_CK(cudaStreamSynchronize(st));
        for (int n = steps - 1; n >= 0; --n) {
            const cplx* Upost = (n + 1 < steps) ? stU + (size_t)(n + 1) * 3 * nlin : postU;
            const double* kxa = (n + 1 < steps) ? kx_pre + (n + 1) * nxy : kx_post;
            // J = (1/N) sum AM_b(post-step state), recorded after the remap (main.cpp:122-130)
            ops.jgrad(Upost, kxa, h->d_ky, h->d_kyi, h->d_ilap2, h->dp, tp[n + 1], 1.0 / N, lamU[iu], st);
            adj_remap_kernel<<<148, 256, 0, st>>>(kx_pre + n * nxy, kxa, h->nxy, h->nz, lamU[iu]);
            for (int s = 2; s >= 0; --s) {
                const StageConst& S = h->sc[s];
                AdjMfArgs M;
                std::memset(&M, 0, sizeof(M));
                M.B = stB + ((size_t)n * 3 + s) * nmfe;
                M.lamB_out = lamB[ib];
                M.lamG_out = (s == 2) ? nullptr : lamG[0];
                M.lamB_in = lamB[ib ^ 1];
                M.lamGp = (s == 0) ? nullptr : lamG[1];
                M.prof = prof;
                M.tw = h->d_tw;
                M.sc = S;
                ops.mf_pre(M, h->dp, st);
                AdjStageArgs A;
                std::memset(&A, 0, sizeof(A));
                A.U = stU + ((size_t)n * 3 + s) * nlin;
                A.lamU_out = lamU[iu];
                A.lamF_out = (s == 2) ? nullptr : lamF[0];
                A.lamU_in = lamU[iu ^ 1];
                A.lamFp = (s == 0) ? nullptr : lamF[1];
                A.kx0 = kx_pre + n * nxy;
                A.ky = h->d_ky;
                A.kxi = h->d_kxi;
                A.kyi = h->d_kyi;
                A.ilap2 = h->d_ilap2;
                A.tw = h->d_tw;
                A.prof = prof;
                A.bpart = bpart;
                A.t_s = tp[n] + S.t_off;
                A.sc = S;
                ops.modes(A, h->dp, h->nxy, st);
                const int nout = 3 * h->NZ;
                adj_bsum_kernel<<<(nout + 7) / 8, 256, 0, st>>>(bpart, h->nxy, nout, bsum);
                ops.mf_post(bsum, h->d_tw, h->dp, lamB[ib ^ 1], st);
                iu ^= 1;
                ib ^= 1;
                std::swap(lamF[0], lamF[1]);
                std::swap(lamG[0], lamG[1]);
            }
        }
        QA_CK(cudaGetLastError());
    }
    QA_CK(cudaMemcpyAsync(grad_lin, lamU[iu], nlin * sizeof(cplx), cudaMemcpyDeviceToHost, st));
    if (grad_mf) QA_CK(cudaMemcpyAsync(grad_mf, lamB[ib], nmfe * sizeof(cplx), cudaMemcpyDeviceToHost, st));
    // leave the handle at the end of the forward run
    h->cur = fin_cur;
    QA_CK(cudaMemcpyAsync(h->d_lin[h->cur], fin_lin, nlin * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_mf, fin_mf, nmfe * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_kx0, fin_kx0, nxy * sizeof(double), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaMemcpyAsync(h->d_clk, fin_clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, st));
    QA_CK(cudaStreamSynchronize(st));
    return QLGPU_OK;
}
