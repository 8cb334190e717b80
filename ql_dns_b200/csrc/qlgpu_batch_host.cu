// qlgpu_batch_host.cu -- host side of the batched ensemble (qlgpu_batch_* in
// include/qlgpu.h): per-case device buffers in one arena, the case
// descriptors of the persistent kernel, the CTA mapping and its autotuner, and
// the CUDA-graph launch of the persistent kernel.
//
// Mapping model.  A CTA of w warps steps mpc = w*(32/T)/2 modes of a case at a
// time (one mode per pair of transform groups).  Giving case c k CTAs costs it
// rounds(c, k) = ceil(nxy_c / (k*mpc)) passes of its stage pipeline per stage.
// A CTA that owns several work items runs them one after the other, so its
// stage time is modelled as the sum over its items of
//     beta + rounds * r[NZ],
// and the launch time per stage as the largest CTA time plus a per-stage
// constant alpha (reduction, mean-field stage, release / wait).  The planner
// binary-searches the smallest per-CTA budget M for which every case's CTA
// count k_c(M) fits and first-fit-decreasing packs all items onto the launch's
// CTAs.  The autotuner measures the per-case finishing times of probe launches
// (%globaltimer stamps written by the kernel), fits alpha, beta and r[NZ] by
// least squares, re-plans, and keeps the fastest measured mapping over two CTA
// widths: the widest that fits the batch and half of it.
//
// Two engines step a batch.  The work-item engine above (qlgpu_batch.cuh) runs
// every model, integrator and NZ.  The chunk-queue engine (qlgpu_ens.cuh) runs
// MHD_BQlin batches with NZ <= 128: CTAs take chunks of a case's modes from a
// global ticket counter, so no CTA waits at a stage boundary of another case.
// Its tuning knob is the number of CTA passes per chunk of each NZ class; its
// autotuner times probe launches over those and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/qlgpu.h"
#include "qlgpu_batch_internal.h"
#include "qlgpu_ens_host.h"
#include "qlgpu_guard.h"
#include "qlgpu_host.h"
#include "qlgpu_kernel.cuh"

using namespace qlgpu;

namespace {

thread_local std::string g_batch_create_error;

constexpr int NCLASS = 5;  // NZ = 16, 32, 64, 128, 256
inline int nz_class(int NZ) {
    switch (NZ) {
        case 16: return 0;
        case 32: return 1;
        case 64: return 2;
        case 128: return 3;
        default: return 4;
    }
}

struct CaseHost {
    qlgpu_params p;
    DevParams dp;
    StageConst sc[3];
    int nxy = 0, nz = 0, NZ = 0, nmf = 0, T = 0, PL = 0, max_cta = 0;
    Variant var;  // single-case variant of the same NZ (initial diagnostics)
    // device pointers into the arena
    cplx* lin[2] = {nullptr, nullptr};
    cplx *F1 = nullptr, *F2 = nullptr, *mf = nullptr, *Fmf1 = nullptr, *Fmf2 = nullptr, *tw = nullptr;
    double *kx0 = nullptr, *ky = nullptr, *il2 = nullptr, *partials = nullptr, *gpartials = nullptr;
    double *mfr = nullptr, *ekz = nullptr, *kx_init = nullptr;
    int *kxi = nullptr, *kyi = nullptr;
    DevClock* clk = nullptr;
    double* diag = nullptr;
    int diag_cap = 0;
    std::vector<double> kx_tab;
    // stage-input record (qlgpu_batch_internal.h), null: off
    cplx *rec_lin = nullptr, *rec_mf = nullptr;
    double *rec_kx = nullptr, *rec_t = nullptr;
    CnRec* rec_cn = nullptr;
    bool noise_on = false;  // driving noise after every step (qlgpu_batch_set_noise)
};

// One work item of the planner: CTA number i of the k given to case c.
struct Item {
    int c, i, k;
    double cost;
};

struct CostModel {
    double alpha = 12.0;                              // us per stage, per launch
    double beta = 2.5;                                // us per work item per stage
    double r[NCLASS] = {4.0, 6.0, 14.0, 30.0, 70.0};  // us per pipeline pass, per NZ class
};

// Zeroes the launch control words, the case stage counters and the reduction
// counters (left non-zero only by a launch that gave up), and optionally the
// diagnostic record counts.
__global__ void batch_reset_kernel(const BatchCase* cases, int ncases, unsigned* epoch, BatchCtl* ctl,
                                   int reset_ndiag) {
    const int c = blockIdx.x;
    if (c == 0 && threadIdx.x == 0) {
        ctl->status = 0;
        ctl->abort = 0;
        ctl->fail_case = -1;
        ctl->fail_stage = -1;
        ctl->fail_where = 0;
        ctl->t_start = 0;
        ctl->next = 0u;
    }
    if (c >= ncases) return;
    DevClock* clk = cases[c].A[0].clk;
    if (threadIdx.x < 64) clk->cnt_group[threadIdx.x] = 0u;
    if (threadIdx.x == 0) {
        clk->cnt_top = 0u;
        epoch[(size_t)c * BATCH_EPOCH_STRIDE] = 0u;
        epoch[(size_t)c * BATCH_EPOCH_STRIDE + 1] = 0u;
        if (reset_ndiag) clk->ndiag = 0;
    }
}

// Gathers every case's status word and diagnostic record count, then the
// launch status and the case of a wait that gave up.
__global__ void batch_collect_kernel(const BatchCase* cases, int ncases, const BatchCtl* ctl,
                                     int* out /* [ncases][2], status, fail_case */) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncases; c += gridDim.x * blockDim.x) {
        const DevClock* clk = cases[c].A[0].clk;
        out[2 * c] = clk->status;
        out[2 * c + 1] = clk->ndiag;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        out[2 * ncases] = ctl->status;
        out[2 * ncases + 1] = ctl->fail_case;
    }
}

// set_states: case c's clock starts at t (reset_case_clock for every case at once).  One block
// per case.
__global__ void batch_set_clocks_kernel(const BatchCase* cases, int ncases, double t) {
    const int c = blockIdx.x;
    if (c >= ncases) return;
    DevClock* k = cases[c].A[0].clk;
    unsigned* w = reinterpret_cast<unsigned*>(k);
    for (int i = threadIdx.x; i < (int)(sizeof(DevClock) / sizeof(unsigned)); i += blockDim.x) w[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        k->t = t;
        k->old_init = 1;
    }
}

// The small per-case arrays of set_states / get_states travel as one block (one copy instead of
// two per case): case c's mean fields [2 nmf nz] and kx0 [nxy] at off[c], then one value per case
// at off[ncases] (set: 1 where kx0 is given, else the case takes its unsheared table; get: t).
__global__ void batch_scatter_small_kernel(const BatchCase* cases, int ncases, const double* src,
                                           const long long* off) {
    const int c = blockIdx.x;
    if (c >= ncases) return;
    const BatchCase& bc = cases[c];
    const int nmf2 = 2 * bc.P.nmf * bc.P.nz, nxy = bc.P.nxy;
    const double* sp = src + off[c];
    double* mf = reinterpret_cast<double*>(bc.A[0].mf);
    for (int i = threadIdx.x; i < nmf2; i += blockDim.x) mf[i] = sp[i];
    const double* kx = src[off[ncases] + c] != 0.0 ? sp + nmf2 : bc.kx_init;
    for (int i = threadIdx.x; i < nxy; i += blockDim.x) bc.A[0].kx0[i] = kx[i];
}
__global__ void batch_gather_small_kernel(const BatchCase* cases, int ncases, double* dst, const long long* off) {
    const int c = blockIdx.x;
    if (c >= ncases) return;
    const BatchCase& bc = cases[c];
    const int nmf2 = 2 * bc.P.nmf * bc.P.nz, nxy = bc.P.nxy;
    double* dp = dst + off[c];
    const double* mf = reinterpret_cast<const double*>(bc.A[0].mf);
    for (int i = threadIdx.x; i < nmf2; i += blockDim.x) dp[i] = mf[i];
    for (int i = threadIdx.x; i < nxy; i += blockDim.x) dp[nmf2 + i] = bc.A[0].kx0[i];
    if (threadIdx.x == 0) dst[off[ncases] + c] = bc.A[0].clk->t;
}

}  // namespace

struct qlgpu_batch {
    int device = 0, model = 0, integ = 0, ncases = 0;
    cudaStream_t stream = nullptr;
    std::vector<CaseHost> cs;
    unsigned char* arena = nullptr;
    size_t arena_bytes = 0;
    BatchCase* d_cases = nullptr;
    BatchCta* d_ctas = nullptr;
    unsigned* d_epoch = nullptr;
    BatchCtl* d_ctl = nullptr;
    unsigned long long* d_case_end = nullptr;
    int* d_collect = nullptr;
    double* d_out15 = nullptr;
    double* d_diag = nullptr;  // [ncases][diag_cap][15] diagnostic records of every case
    int diag_cap = 0;
    BatchKernel bk;
    int sms = 0;
    size_t smem_optin = 0;
    // current mapping
    int warps = 8, per_sm = 1, grid = 0;
    int wide_warps = 0;  // widest CTA that fits every NZ class of the batch
    size_t smem = 0;
    std::vector<BatchCta> ctas;
    std::vector<int> ncta;
    CostModel cost;
    int cur = 0;
    long long wait_ns = 2000000000LL;
    bool use_graph = true;
    std::map<std::tuple<int, int, int>, cudaGraphExec_t> graphs;  // (nsteps, parity, reset_ndiag)
    std::vector<double> tv_set;  // diagnostic interval in each case's uploaded descriptor
    bool descr_dirty = true;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::string err;
    // chunk-queue engine (qlgpu_ens.cuh)
    int engine = QLGPU_BATCH_ENGINE_ITEMS;
    bool queue_ok = false;               // MHD_BQlin and every NZ <= 128
    int qpasses[4] = {4, 4, 4, 4};       // CTA passes per chunk, NZ = 16, 32, 64, 128
    std::vector<ens::EnsCase> ec;
    std::vector<ens::RoundItem> round;
    ens::EnsCase* d_ec = nullptr;
    ens::RoundItem* d_round = nullptr;
    cplx* d_tw8 = nullptr;               // 8-point twiddles of NZ = 16, 32, 64, 128 (240 cplx)
    size_t qsmem = 0;
    int qgrid = 0;
    int drop_case = -1;                  // failure-detection aid: a chunk of this case is left out
    bool qdirty = true;
    unsigned long long* d_qtrace = nullptr;  // [grid][4] per-CTA time sums of the last queue launch (QLGPU_TRACE=1)
    // the small arrays of set_states / get_states in one block (batch_scatter_small_kernel)
    std::vector<long long> soff;             // [ncases + 1] offsets in doubles
    long long* d_soff = nullptr;
    double* d_small = nullptr;
    double* h_small = nullptr;               // pinned
    int* h_col = nullptr;                    // pinned copy of d_collect
    double* h_diag = nullptr;                // pinned copy of d_diag
    // asynchronous steps (qlgpu_batch_step_async): a ring of two slots, each with pinned copies of
    // the launch's statuses, control block and records, and an event after those copies
    struct AsyncSlot {
        int* col = nullptr;
        BatchCtl* ctl = nullptr;
        double* diag = nullptr;
        cudaEvent_t done = nullptr;
        int diag_every = 0, max_diag = 0;
    } aslot[2];
    int a_head = 0, a_count = 0;
    NoiseSpec* d_noise = nullptr;            // [ncases] driving-noise constants
    GuardList guards;                        // debug build: canary zones after the device buffers
};

namespace {

int bfail(qlgpu_batch_t* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    else g_batch_create_error = msg;
    return code;
}

#define QB_CK(call)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return bfail(b, QLGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
// one arena slot: the buffer and, in the debug build, its guard zone
size_t gslot(size_t x) { return al256(x + QLGPU_GUARD_BYTES); }

int modes_per_cta(int warps, int T) { return warps * (32 / T) / 2; }

int rounds_of(const CaseHost& c, int k, int warps) {
    const int m = modes_per_cta(warps, c.T) * k;
    return (c.nxy + m - 1) / m;
}

void drop_graphs(qlgpu_batch_t* b) {
    for (auto& kv : b->graphs)
        if (kv.second) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

// CTAs per SM and dynamic shared memory of a CTA width over the NZ classes present.
bool width_limits(qlgpu_batch_t* b, int warps, int* per_sm, size_t* smem) {
    size_t sm = 0;
    int tc = 0;
    for (const CaseHost& c : b->cs) {
        sm = std::max(sm, b->bk.smem(c.NZ, warps));
        tc = std::max(tc, b->bk.tmem(c.NZ, warps));
    }
    if (sm > b->smem_optin || tc > 512) return false;
    if (ensure_smem_attr(b->bk.kernel(), sm) != cudaSuccess)
        return false;
    cudaFuncSetAttribute(b->bk.kernel(), cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, b->bk.kernel(), 32 * warps, sm) != cudaSuccess) return false;
    if (tc > 0) occ = std::min(occ, 512 / tc);  // TMEM columns per SM: an allocation beyond them would wait
    if (occ < 1) return false;
    *per_sm = occ;
    *smem = sm;
    return true;
}

// Plan: CTAs per case and the packing of work items onto at most G CTAs.
// fixed_k (optional) pins the CTA count of every case.
bool plan(const qlgpu_batch_t* b, int warps, int G, const CostModel& cm, const int* fixed_k, std::vector<int>& k_out,
          std::vector<std::vector<Item>>& bins_out, double* makespan) {
    const int nc = b->ncases;
    auto item_cost = [&](int c, int k) {
        const CaseHost& h = b->cs[c];
        return cm.beta + rounds_of(h, k, warps) * cm.r[nz_class(h.NZ)];
    };
    auto try_budget = [&](double M, std::vector<int>& k, std::vector<std::vector<Item>>& bins) -> bool {
        k.assign(nc, 1);
        std::vector<Item> items;
        for (int c = 0; c < nc; ++c) {
            const CaseHost& h = b->cs[c];
            if (fixed_k) {
                k[c] = fixed_k[c];
            } else {
                const int kmax = std::min(h.max_cta, G);
                int kk = 1;
                while (kk < kmax && item_cost(c, kk) > M) {
                    // next CTA count that lowers the number of passes
                    const int r = rounds_of(h, kk, warps);
                    const int m = modes_per_cta(warps, h.T);
                    int nk = r > 1 ? (h.nxy + m * (r - 1) - 1) / (m * (r - 1)) : kk + 1;
                    if (nk <= kk) nk = kk + 1;
                    kk = std::min(nk, kmax);
                }
                if (item_cost(c, kk) > M) return false;
                k[c] = kk;
            }
            for (int i = 0; i < k[c]; ++i) items.push_back(Item{c, i, k[c], item_cost(c, k[c])});
        }
        std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) { return x.cost > y.cost; });
        bins.clear();
        std::vector<double> load;
        for (const Item& it : items) {
            int best = -1;
            for (size_t j = 0; j < bins.size(); ++j)
                if ((int)bins[j].size() < BATCH_MAX_SLOTS && load[j] + it.cost <= M) {
                    best = (int)j;
                    break;
                }
            if (best < 0) {
                if ((int)bins.size() >= G) return false;
                bins.emplace_back();
                load.push_back(0.0);
                best = (int)bins.size() - 1;
            }
            bins[best].push_back(it);
            load[best] += it.cost;
        }
        return true;
    };
    double lo = 0.0, hi = 0.0;
    for (int c = 0; c < nc; ++c) {
        const int kmin = fixed_k ? fixed_k[c] : 1;
        const int kbest = fixed_k ? fixed_k[c] : std::min(b->cs[c].max_cta, G);
        lo = std::max(lo, item_cost(c, kbest));
        hi += item_cost(c, kmin) * kmin;
    }
    hi = std::max(hi, lo) * 1.0001 + 1.0;
    std::vector<int> kb;
    std::vector<std::vector<Item>> bb;
    if (!try_budget(hi, kb, bb)) return false;  // more items than CTA slots
    for (int it = 0; it < 60 && hi - lo > 1e-3 * hi; ++it) {
        const double mid = 0.5 * (lo + hi);
        std::vector<int> k;
        std::vector<std::vector<Item>> bins;
        if (try_budget(mid, k, bins)) {
            hi = mid;
            kb.swap(k);
            bb.swap(bins);
        } else {
            lo = mid;
        }
    }
    k_out = kb;
    bins_out = bb;
    if (makespan) *makespan = hi;
    return true;
}

// Device descriptors of every case.
int upload_descriptors(qlgpu_batch_t* b) {
    std::vector<BatchCase> hc(b->ncases);
    for (int c = 0; c < b->ncases; ++c) {
        CaseHost& h = b->cs[c];
        BatchCase& d = hc[c];
        std::memset(&d, 0, sizeof(d));
        d.P = h.dp;
        d.P.tv_interval = b->tv_set[c];
        cplx* Fbuf[3] = {h.F1, h.F2, nullptr};
        const cplx* Fprev[3] = {nullptr, h.F1, h.F2};
        cplx* Fmf[3] = {h.Fmf1, h.Fmf2, nullptr};
        const cplx* Fmfp[3] = {nullptr, h.Fmf1, h.Fmf2};
        for (int s = 0; s < 3; ++s) {
            StageArgs& A = d.A[s];
            A.lin_in = h.lin[s & 1];
            A.lin_out = h.lin[(s & 1) ^ 1];
            A.Fprev = Fprev[s];
            A.Fout = Fbuf[s];
            A.mf = h.mf;
            A.Fmf_prev = Fmfp[s];
            A.Fmf_out = Fmf[s];
            A.kx0 = h.kx0;
            A.ky = h.ky;
            A.kxi = h.kxi;
            A.kyi = h.kyi;
            A.tw = h.tw;
            A.ilap2 = h.il2;
            A.partials = h.partials;
            A.gpartials = h.gpartials;
            A.clk = h.clk;
            A.diag_ring = h.diag;
            A.diag_cap = h.diag_cap;
            A.mfr_cache = h.mfr;
            A.ekz_tab = h.ekz + (size_t)s * 2 * h.nz;
            A.noise = (s == 2 && h.noise_on) ? b->d_noise + c : nullptr;
            A.sc = h.sc[s];
        }
        d.kx_init = h.kx_init;
        d.rec_lin = h.rec_lin;
        d.rec_mf = h.rec_mf;
        d.rec_kx = h.rec_kx;
        d.rec_t = h.rec_t;
        d.rec_cn = h.rec_cn;
    }
    QB_CK(cudaMemcpyAsync(b->d_cases, hc.data(), sizeof(BatchCase) * hc.size(), cudaMemcpyHostToDevice, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    b->descr_dirty = false;
    return QLGPU_OK;
}

// Install a mapping (CTA width + packed work items).
int apply_mapping(qlgpu_batch_t* b, int warps, int per_sm, size_t smem, const std::vector<int>& k,
                  const std::vector<std::vector<Item>>& bins) {
    std::vector<BatchCta> ctas(bins.size());
    for (size_t j = 0; j < bins.size(); ++j) {
        BatchCta& m = ctas[j];
        std::memset(&m, 0, sizeof(m));
        m.nslots = (int)bins[j].size();
        int tc = 0;
        for (int i = 0; i < m.nslots; ++i) {
            const Item& it = bins[j][i];
            m.slot[i].c = it.c;
            m.slot[i].cta = it.i;
            m.slot[i].ncta = it.k;
            m.slot[i].NZ = b->cs[it.c].NZ;
            tc = std::max(tc, b->bk.tmem(b->cs[it.c].NZ, warps));
        }
        m.tcols = tc;
    }
    if (ensure_smem_attr(b->bk.kernel(), smem) != cudaSuccess)
        return bfail(b, QLGPU_ERR_CUDA, "batch kernel: shared memory request too large");
    QB_CK(cudaMemcpyAsync(b->d_ctas, ctas.data(), sizeof(BatchCta) * ctas.size(), cudaMemcpyHostToDevice, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    b->ctas = ctas;
    b->ncta = k;
    b->warps = warps;
    b->per_sm = per_sm;
    b->smem = smem;
    b->grid = (int)ctas.size();
    drop_graphs(b);
    return QLGPU_OK;
}

int plan_and_apply(qlgpu_batch_t* b, int warps, const int* fixed_k) {
    int per_sm = 0;
    size_t smem = 0;
    if (!width_limits(b, warps, &per_sm, &smem))
        return bfail(b, QLGPU_ERR_UNSUPPORTED, "batch: CTA width does not fit (shared memory / TMEM)");
    const int G = std::min(b->sms * per_sm, b->sms * 2);
    std::vector<int> k;
    std::vector<std::vector<Item>> bins;
    if (fixed_k)
        for (int c = 0; c < b->ncases; ++c)
            if (fixed_k[c] < 1 || fixed_k[c] > b->cs[c].max_cta)
                return bfail(b, QLGPU_ERR_ARG, "batch mapping: CTAs per case out of range");
    if (!plan(b, warps, G, b->cost, fixed_k, k, bins, nullptr))
        return bfail(b, QLGPU_ERR_UNSUPPORTED,
                     "batch: the cases do not fit one launch (at most 8 work items on each co-resident CTA)");
    return apply_mapping(b, warps, per_sm, smem, k, bins);
}

// ---------------------------------------------------------------------------
// Chunk-queue engine
// ---------------------------------------------------------------------------
constexpr int QTRACE_MAX_CTAS_PER_SM = 4;  // bound of the queue grid: at most this many CTAs per SM

int ens_class(int NZ) { return NZ == 16 ? 0 : NZ == 32 ? 1 : NZ == 64 ? 2 : 3; }
size_t tw8_offset(int NZ) { return NZ == 16 ? 0 : NZ == 32 ? 16 : NZ == 64 ? 48 : 112; }  // cplx

// Default CTA passes per chunk of each NZ class, before any tuning.  Four passes
// keep the fixed cost of a chunk small (about 12 us against about 25 us per pass,
// the same at every NZ by the choice of modes per pass; measured on B200).  When
// four passes leave CTAs without a chunk (a small batch), the combination of
// {1, 2, 3, 4} that minimises whole waves of chunks times the mean chunk time is
// taken instead.
void default_passes(qlgpu_batch_t* b) {
    constexpr double PASS_US = 25.0, CHUNK_US = 12.0;
    const int grid = b->sms;
    std::vector<int> need(b->ncases), cls(b->ncases);
    bool present[4] = {false, false, false, false};
    for (int c = 0; c < b->ncases; ++c) {
        const CaseHost& h = b->cs[c];
        const int mpp = ens::modes_per_pass(h.NZ);
        need[c] = (h.nxy + mpp - 1) / mpp;
        cls[c] = ens_class(h.NZ);
        present[cls[c]] = true;
    }
    auto chunks_and_work = [&](const int (&p)[4], double* work) {
        long C = 0;
        double W = 0.0;
        for (int c = 0; c < b->ncases; ++c) {
            const int pc = p[cls[c]];
            const long n = (need[c] + pc - 1) / pc;
            C += n;
            W += (double)n * (pc * PASS_US + CHUNK_US);
        }
        *work = W;
        return C;
    };
    int best[4] = {4, 4, 4, 4};
    double W4 = 0.0;
    if (chunks_and_work(best, &W4) >= grid) {
        std::copy(best, best + 4, b->qpasses);
        return;
    }
    double best_est = 1e300;
    for (int code = 0; code < 256; ++code) {
        int p[4];
        bool skip = false;
        for (int k = 0; k < 4; ++k) {
            p[k] = 1 + ((code >> (2 * k)) & 3);
            if (!present[k] && p[k] != 4) skip = true;
        }
        if (skip) continue;
        double W = 0.0;
        const long C = chunks_and_work(p, &W);
        const double est = (double)((C + grid - 1) / grid) * (W / (double)C);
        if (est < best_est - 1e-9) {
            best_est = est;
            std::copy(p, p + 4, best);
        }
    }
    std::copy(best, best + 4, b->qpasses);
}

bool queue_usable(const qlgpu_batch_t* b) { return b->queue_ok && b->engine == QLGPU_BATCH_ENGINE_QUEUE; }

// Some case records its stage inputs: the queue engine's recording build runs.
bool queue_rec(const qlgpu_batch_t* b) {
    for (const CaseHost& h : b->cs)
        if (h.rec_lin) return true;
    return false;
}

// Chunks per stage of every case (passes per chunk of its NZ class, raised until
// the case's partial-sum slots hold every chunk) and the order of one round:
// cases with the longest chunks first, each case's chunks consecutive.
int queue_plan(qlgpu_batch_t* b) {
    const int nc = b->ncases;
    b->ec.assign(nc, ens::EnsCase());
    std::vector<double> len(nc);
    size_t smem = 0;
    for (int c = 0; c < nc; ++c) {
        const CaseHost& h = b->cs[c];
        const int mpp = ens::modes_per_pass(h.NZ);
        int passes = std::max(1, b->qpasses[ens_class(h.NZ)]);
        int nch = 0, mpc = 0;
        for (;;) {
            mpc = passes * mpp;
            nch = (h.nxy + mpc - 1) / mpc;
            if (nch <= h.max_cta) break;
            ++passes;
        }
        ens::EnsCase& e = b->ec[c];
        std::memset(&e, 0, sizeof(e));
        e.NZ = h.NZ;
        e.nch = nch;
        e.mpc = mpc;
        e.tw8 = b->d_tw8 + tw8_offset(h.NZ);
        len[c] = (double)passes * h.NZ;
        smem = std::max(smem, ens::smem_bytes(h.NZ));
    }
    std::vector<int> ord(nc);
    for (int c = 0; c < nc; ++c) ord[c] = c;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return len[x] > len[y]; });
    b->round.clear();
    for (int c : ord)
        for (int j = 0; j < b->ec[c].nch; ++j) {
            if (c == b->drop_case && j == b->ec[c].nch - 1) continue;
            b->round.push_back(ens::RoundItem{c, j});
        }
    if (b->d_round) cudaFree(b->d_round);
    b->d_round = nullptr;
    QB_CK(cudaMalloc(&b->d_round, sizeof(ens::RoundItem) * std::max<size_t>(1, b->round.size())));
    QB_CK(cudaMemcpyAsync(b->d_round, b->round.data(), sizeof(ens::RoundItem) * b->round.size(),
                          cudaMemcpyHostToDevice, b->stream));
    QB_CK(cudaMemcpyAsync(b->d_ec, b->ec.data(), sizeof(ens::EnsCase) * nc, cudaMemcpyHostToDevice, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    const void* k = ens::kernel(b->integ, queue_rec(b));
    if (smem > b->smem_optin) return bfail(b, QLGPU_ERR_UNSUPPORTED, "queue engine: shared memory request too large");
    QB_CK(ensure_smem_attr(k, smem));
    int occ = 0;
    QB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, ens::threads(), smem));
    if (occ < 1) return bfail(b, QLGPU_ERR_UNSUPPORTED, "queue engine: the CTA does not fit an SM");
    b->qsmem = smem;
    if (occ > QTRACE_MAX_CTAS_PER_SM) occ = QTRACE_MAX_CTAS_PER_SM;
    b->qgrid = b->sms * occ;  // every resident CTA (a cooperative launch)
    b->qdirty = false;
    drop_graphs(b);
    return QLGPU_OK;
}

cudaError_t enqueue_queue(qlgpu_batch_t* b, int nsteps, int reset_ndiag) {
    batch_reset_kernel<<<b->ncases, 64, 0, b->stream>>>(b->d_cases, b->ncases, b->d_epoch, b->d_ctl, reset_ndiag);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ens::EnsLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.cases = b->d_cases;
    L.ec = b->d_ec;
    L.round = b->d_round;
    L.epoch = b->d_epoch;
    L.ctl = b->d_ctl;
    L.next = &b->d_ctl->next;
    L.case_end = b->d_case_end;
    L.R = (int)b->round.size();
    L.nrounds = 3 * nsteps;
    L.parity = b->cur;
    L.ncases = b->ncases;
    L.wait_ns = b->wait_ns;
    L.trace = b->d_qtrace;
    if (b->d_qtrace) {
        e = cudaMemsetAsync(b->d_qtrace, 0, sizeof(unsigned long long) * 4 * b->qgrid, b->stream);
        if (e != cudaSuccess) return e;
    }
    return ens::launch(b->integ, queue_rec(b), L, b->qgrid, b->qsmem, b->stream);
}

BatchLaunch launch_args(qlgpu_batch_t* b, int nsteps) {
    BatchLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.cases = b->d_cases;
    L.ctas = b->d_ctas;
    L.epoch = b->d_epoch;
    L.ctl = b->d_ctl;
    L.case_end = b->d_case_end;
    L.nsteps = nsteps;
    L.parity = b->cur;
    L.wait_ns = b->wait_ns;
    L.ncases = b->ncases;
    return L;
}

// Enqueue the reset kernel and the persistent launch on the batch stream.
cudaError_t enqueue_launch(qlgpu_batch_t* b, int nsteps, int reset_ndiag) {
    batch_reset_kernel<<<b->ncases, 64, 0, b->stream>>>(b->d_cases, b->ncases, b->d_epoch, b->d_ctl, reset_ndiag);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return b->bk.launch(launch_args(b, nsteps), b->grid, 32 * b->warps, b->smem, b->stream);
}

// Prepares the launch of nsteps steps (descriptors, queue plan, the CUDA graph for this
// step count), then records ev_before (if any) on the batch stream and launches: a timing
// bracket around the launch holds only device work.
int run_launch(qlgpu_batch_t* b, int nsteps, int reset_ndiag, cudaEvent_t ev_before = nullptr) {
    if (b->descr_dirty) {
        int rc = upload_descriptors(b);
        if (rc) return rc;
    }
    if (nsteps == 0) return QLGPU_OK;
    const bool q = queue_usable(b);
    if (q && b->qdirty) {
        int rc = queue_plan(b);
        if (rc) return rc;
    }
    // the dynamic shared memory attribute belongs to the kernel, not to this batch
    if (q) QB_CK(ensure_smem_attr(ens::kernel(b->integ, queue_rec(b)), b->qsmem));
    else QB_CK(ensure_smem_attr(b->bk.kernel(), b->smem));
    auto enqueue = [&]() { return q ? enqueue_queue(b, nsteps, reset_ndiag) : enqueue_launch(b, nsteps, reset_ndiag); };
    if (b->use_graph) {
        const auto key = std::make_tuple(nsteps, b->cur + (q ? 2 : 0) + (q && queue_rec(b) ? 4 : 0), reset_ndiag);
        auto itg = b->graphs.find(key);
        if (itg == b->graphs.end()) {
            if (b->graphs.size() >= 8) drop_graphs(b);
            cudaGraph_t g = nullptr;
            QB_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            const cudaError_t le = enqueue();
            const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
            if (le != cudaSuccess || ce != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                return bfail(b, QLGPU_ERR_CUDA,
                             std::string("batch graph capture: ") + cudaGetErrorString(le != cudaSuccess ? le : ce));
            }
            cudaGraphExec_t ex = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return bfail(b, QLGPU_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(ie));
            itg = b->graphs.emplace(key, ex).first;
            // upload the new graph before the first timed launch (instantiation work stays outside
            // the timing bracket)
            QB_CK(cudaGraphUpload(ex, b->stream));
        }
        if (ev_before) QB_CK(cudaEventRecord(ev_before, b->stream));
        QB_CK(cudaGraphLaunch(itg->second, b->stream));
    } else {
        if (ev_before) QB_CK(cudaEventRecord(ev_before, b->stream));
        QB_CK(enqueue());
    }
    b->cur = (b->cur + nsteps) & 1;
    return QLGPU_OK;
}

// Debug build: after a launch, the index checks' bit in the launch status and in every case's
// status word, and the guard zones after every buffer.  A release build returns at once.
int debug_verify(qlgpu_batch_t* b) {
#ifdef QLGPU_DEBUG
    const int nc = b->ncases;
    std::vector<int> col(2 * (size_t)nc + 2);
    batch_collect_kernel<<<(nc + 127) / 128, 128, 0, b->stream>>>(b->d_cases, nc, b->d_ctl, b->d_collect);
    QB_CK(cudaGetLastError());
    QB_CK(cudaMemcpyAsync(col.data(), b->d_collect, col.size() * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    int g = 0;
    QB_CK(guard_check(b->guards, b->stream, &g));
    int st = g | (col[2 * nc] & QLGPU_STATUS_BOUNDS);
    for (int c = 0; c < nc; ++c) st |= col[2 * c] & QLGPU_STATUS_BOUNDS;
    if (st) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "debug build: device status 0x%x (%s)", st,
                      (st & QLGPU_STATUS_BOUNDS) ? "an index check failed" : "a guard zone was overwritten");
        return bfail(b, QLGPU_ERR_STATUS, buf);
    }
#else
    (void)b;
#endif
    return QLGPU_OK;
}

int launch_timeout(qlgpu_batch_t* b, const BatchCtl& ctl) {
    char buf[200];
    std::snprintf(buf, sizeof(buf),
                  "batch: a CTA gave up waiting %s case %d at stage %d (wait bound %.3g s); the state of the "
                  "batch is undefined",
                  ctl.fail_where == 1 ? "for a staged copy of" : "for", ctl.fail_case, ctl.fail_stage,
                  b->wait_ns * 1e-9);
    return bfail(b, QLGPU_ERR_STATUS, buf);
}

int check_launch_status(qlgpu_batch_t* b) {
    BatchCtl ctl;
    QB_CK(cudaMemcpyAsync(&ctl, b->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    if (ctl.status & QLGPU_STATUS_TIMEOUT) return launch_timeout(b, ctl);
    return debug_verify(b);
}

// One block for every case's records, laid out as the callers' diag_out: [case][max_diag][15].
int alloc_records(qlgpu_batch_t* b, int max_diag) {
    if (b->d_diag) cudaFree(b->d_diag);
    if (b->h_diag) cudaFreeHost(b->h_diag);
    b->d_diag = nullptr;
    b->h_diag = nullptr;
    b->diag_cap = 0;
    QB_CK(cudaMalloc(&b->d_diag, sizeof(double) * 15 * (size_t)max_diag * b->ncases));
    QB_CK(cudaHostAlloc(&b->h_diag, sizeof(double) * 15 * (size_t)max_diag * b->ncases, cudaHostAllocDefault));
    b->diag_cap = max_diag;
    for (int c = 0; c < b->ncases; ++c) {
        b->cs[c].diag = b->d_diag + (size_t)c * max_diag * 15;
        b->cs[c].diag_cap = max_diag;
    }
    b->descr_dirty = true;
    return QLGPU_OK;
}

// Record counts and case statuses of a finished step launch (col = batch_collect_kernel's output).
int step_records(qlgpu_batch_t* b, const int* col, int diag_every, int max_diag, int* ndiag) {
    const int nc = b->ncases;
    int bad = -1;
    for (int c = 0; c < nc; ++c) {
        if (diag_every > 0) ndiag[c] = std::min(col[2 * c + 1], max_diag);
        if (bad < 0 && (col[2 * c] & (QLGPU_STATUS_NONFINITE | QLGPU_STATUS_UNSTABLE | QLGPU_STATUS_DIAG_FULL)))
            bad = c;
    }
    if (bad >= 0) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "case %d: device status 0x%x (non-finite, unstable or records dropped)", bad,
                      col[2 * bad]);
        return bfail(b, QLGPU_ERR_STATUS, buf);
    }
    return QLGPU_OK;
}

int reset_case_clock(qlgpu_batch_t* b, int c, double t) {
    DevClock k;
    std::memset(&k, 0, sizeof(k));
    k.t = t;
    k.old_init = 1;
    QB_CK(cudaMemcpyAsync(b->cs[c].clk, &k, sizeof(k), cudaMemcpyHostToDevice, b->stream));
    return QLGPU_OK;
}

}  // namespace

extern "C" {

int qlgpu_batch_last_error(const qlgpu_batch_t* b, char* buf, int buflen) {
    const std::string& s = b ? b->err : g_batch_create_error;
    if (buf && buflen > 0) std::snprintf(buf, (size_t)buflen, "%s", s.c_str());
    return (int)s.size();
}

int qlgpu_batch_destroy(qlgpu_batch_t* b) {
    if (!b) return QLGPU_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    void* bufs[] = {b->arena,   b->d_cases, b->d_ctas, b->d_epoch, b->d_ctl, b->d_case_end, b->d_collect,
                    b->d_out15, b->d_diag,  b->d_ec,   b->d_round, b->d_tw8, b->d_qtrace, b->d_noise, b->d_soff,
                    b->d_small};
    for (void* p : bufs)
        if (p) cudaFree(p);
    if (b->h_small) cudaFreeHost(b->h_small);
    if (b->h_col) cudaFreeHost(b->h_col);
    if (b->h_diag) cudaFreeHost(b->h_diag);
    for (auto& a : b->aslot) {
        if (a.col) cudaFreeHost(a.col);
        if (a.ctl) cudaFreeHost(a.ctl);
        if (a.diag) cudaFreeHost(a.diag);
        if (a.done) cudaEventDestroy(a.done);
    }
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    guard_release(b->guards);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return QLGPU_OK;
}

int qlgpu_batch_create(const qlgpu_params* cases, int ncases, int device, qlgpu_batch_t** out) {
    qlgpu_batch_t* b = nullptr;
    if (!cases || !out || ncases < 1) return bfail(nullptr, QLGPU_ERR_ARG, "null argument or ncases < 1");
    *out = nullptr;
    for (int c = 0; c < ncases; ++c) {
        std::string msg;
        const int rc = check_params(cases[c], &msg);
        if (rc) return bfail(nullptr, rc, "case " + std::to_string(c) + ": " + msg);
        if (cases[c].model != cases[0].model || cases[c].integrator != cases[0].integrator)
            return bfail(nullptr, QLGPU_ERR_UNSUPPORTED, "all cases of a batch share the model and the integrator");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bfail(nullptr, QLGPU_ERR_NODEVICE, "no CUDA device");
    b = new (std::nothrow) qlgpu_batch();
    if (!b) return bfail(nullptr, QLGPU_ERR_ARG, "out of host memory");
    auto bail = [&](int code) {
        g_batch_create_error = b->err;
        qlgpu_batch_destroy(b);
        return code;
    };
    if (device < 0) cudaGetDevice(&device);
    b->device = device;
    b->model = cases[0].model;
    b->integ = cases[0].integrator;
    b->ncases = ncases;
    if (cudaSetDevice(device) != cudaSuccess) {
        b->err = "cudaSetDevice failed";
        return bail(QLGPU_ERR_NODEVICE);
    }
    int max_nz = 0;
    for (int c = 0; c < ncases; ++c) max_nz = std::max(max_nz, cases[c].NZ);
    if (!pick_batch_kernel(b->model, b->integ, max_nz > 64, &b->bk)) {
        b->err = "no batch kernel for this model / integrator";
        return bail(QLGPU_ERR_UNSUPPORTED);
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        b->err = "cudaGetDeviceProperties failed";
        return bail(QLGPU_ERR_CUDA);
    }
    if (!prop.cooperativeLaunch) {
        b->err = "device does not support cooperative launches";
        return bail(QLGPU_ERR_UNSUPPORTED);
    }
    b->sms = prop.multiProcessorCount;
    b->smem_optin = prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        b->err = "stream create failed";
        return bail(QLGPU_ERR_CUDA);
    }
    {
        const char* g = std::getenv("QLGPU_BATCH_GRAPH");
        b->use_graph = !(g && g[0] == '0');
    }
    // Per-case sizes and the arena layout
    b->cs.resize(ncases);
    b->tv_set.assign(ncases, 0.0);
    const int max_grid = 2 * b->sms;  // widest launch: two CTAs per SM
    std::vector<size_t> off(ncases);
    size_t o = 0;
    for (int c = 0; c < ncases; ++c) {
        CaseHost& h = b->cs[c];
        h.p = cases[c];
        h.dp = make_devparams(h.p);
        for (int s = 0; s < 3; ++s) h.sc[s] = stage_const(h.p, s);
        h.nxy = h.dp.nxy;
        h.nz = h.dp.nz;
        h.NZ = h.p.NZ;
        h.nmf = h.dp.nmf;
        h.T = group_threads(h.NZ);
        h.PL = (h.nmf == 2 ? 2 : 4) * h.NZ + 8;
        h.max_cta = std::min(max_grid, (h.nxy + modes_per_cta(4, h.T) - 1) / modes_per_cta(4, h.T));
        h.max_cta = std::min(h.max_cta, 64 * RED_GROUP);
        if (!pick_variant(h.NZ, b->model, b->integ, true, &h.var)) {
            b->err = "unsupported NZ";
            return bail(QLGPU_ERR_UNSUPPORTED);
        }
        const size_t nlin = (size_t)h.nxy * 4 * h.nz, nmfe = (size_t)h.nmf * h.nz;
        off[c] = o;
        o += 4 * gslot(nlin * sizeof(cplx));                       // lin[2], F1, F2
        o += 3 * gslot(nmfe * sizeof(cplx));                       // mf, Fmf1, Fmf2
        o += 3 * gslot(h.nxy * sizeof(double));                    // kx0, ky, kx_init
        o += 2 * gslot(h.nxy * sizeof(int));                       // kxi, kyi
        o += gslot(h.NZ * sizeof(cplx));                           // twiddles
        o += gslot((size_t)(h.p.ny / 2) * h.nz * sizeof(double));  // 1/lap2
        o += gslot((size_t)h.max_cta * h.PL * sizeof(double));     // partials
        o += gslot((size_t)((h.max_cta + RED_GROUP - 1) / RED_GROUP) * h.PL * sizeof(double));
        o += gslot(sizeof(DevClock));
        o += gslot((size_t)8 * h.NZ * sizeof(double));  // mean-field profile cache
        o += gslot((size_t)6 * h.nz * sizeof(double));  // integrating-factor tables
    }
    b->arena_bytes = o;
    if (cudaMalloc(&b->arena, o) != cudaSuccess) {
        b->err = "cudaMalloc of the batch arena failed (" + std::to_string(o >> 20) + " MiB)";
        return bail(QLGPU_ERR_CUDA);
    }
    cudaMemsetAsync(b->arena, 0, o, b->stream);
    for (int c = 0; c < ncases; ++c) {
        CaseHost& h = b->cs[c];
        unsigned char* p = b->arena + off[c];
        const size_t nlin = (size_t)h.nxy * 4 * h.nz, nmfe = (size_t)h.nmf * h.nz;
        auto take = [&](size_t bytes) {
            unsigned char* r = p;
            p += gslot(bytes);
            guard_add(b->guards, r, bytes);
            return r;
        };
        h.lin[0] = reinterpret_cast<cplx*>(take(nlin * sizeof(cplx)));
        h.lin[1] = reinterpret_cast<cplx*>(take(nlin * sizeof(cplx)));
        h.F1 = reinterpret_cast<cplx*>(take(nlin * sizeof(cplx)));
        h.F2 = reinterpret_cast<cplx*>(take(nlin * sizeof(cplx)));
        h.mf = reinterpret_cast<cplx*>(take(nmfe * sizeof(cplx)));
        h.Fmf1 = reinterpret_cast<cplx*>(take(nmfe * sizeof(cplx)));
        h.Fmf2 = reinterpret_cast<cplx*>(take(nmfe * sizeof(cplx)));
        h.kx0 = reinterpret_cast<double*>(take(h.nxy * sizeof(double)));
        h.kx_init = reinterpret_cast<double*>(take(h.nxy * sizeof(double)));
        h.ky = reinterpret_cast<double*>(take(h.nxy * sizeof(double)));
        h.kxi = reinterpret_cast<int*>(take(h.nxy * sizeof(int)));
        h.kyi = reinterpret_cast<int*>(take(h.nxy * sizeof(int)));
        h.tw = reinterpret_cast<cplx*>(take(h.NZ * sizeof(cplx)));
        h.il2 = reinterpret_cast<double*>(take((size_t)(h.p.ny / 2) * h.nz * sizeof(double)));
        h.partials = reinterpret_cast<double*>(take((size_t)h.max_cta * h.PL * sizeof(double)));
        h.gpartials = reinterpret_cast<double*>(
            take((size_t)((h.max_cta + RED_GROUP - 1) / RED_GROUP) * h.PL * sizeof(double)));
        h.clk = reinterpret_cast<DevClock*>(take(sizeof(DevClock)));
        h.mfr = reinterpret_cast<double*>(take((size_t)8 * h.NZ * sizeof(double)));
        h.ekz = reinterpret_cast<double*>(take((size_t)6 * h.nz * sizeof(double)));
        // tables (Kdata.cpp:24-46,100-119; twiddles; exp(linC nu kz2) per stage)
        std::vector<double> ky;
        std::vector<int> kxi, kyi;
        ktables(h.p, h.kx_tab, ky, kxi, kyi);
        const std::vector<double> tw = twiddles(h.NZ, h.T);
        const std::vector<double> il2 = ilap2_table(h.p, h.nz);
        const std::vector<double> ekz = ekz_table(h.p, h.dp);
        cudaMemcpyAsync(h.kx0, h.kx_tab.data(), h.nxy * sizeof(double), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(h.kx_init, h.kx_tab.data(), h.nxy * sizeof(double), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(h.ky, ky.data(), h.nxy * sizeof(double), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(h.kxi, kxi.data(), h.nxy * sizeof(int), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(h.kyi, kyi.data(), h.nxy * sizeof(int), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(h.tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(h.il2, il2.data(), il2.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(h.ekz, ekz.data(), ekz.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream);
        if (reset_case_clock(b, c, 0.0)) return bail(QLGPU_ERR_CUDA);
        // the host vectors above die at the end of this iteration: finish the copies first
        if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
            b->err = "table upload failed";
            return bail(QLGPU_ERR_CUDA);
        }
    }
#define QB_ALLOC(ptr, bytes)                                              \
    if (cudaMalloc(&(ptr), (bytes) + QLGPU_GUARD_BYTES) != cudaSuccess) { \
        b->err = "cudaMalloc failed for " #ptr;                           \
        return bail(QLGPU_ERR_CUDA);                                      \
    }                                                                     \
    guard_add(b->guards, (ptr), (bytes));                                 \
    cudaMemsetAsync((ptr), 0, (bytes), b->stream);
    QB_ALLOC(b->d_cases, sizeof(BatchCase) * ncases);
    QB_ALLOC(b->d_ctas, sizeof(BatchCta) * (size_t)max_grid);
    QB_ALLOC(b->d_epoch, sizeof(unsigned) * BATCH_EPOCH_STRIDE * (size_t)ncases);
    QB_ALLOC(b->d_ctl, sizeof(BatchCtl));
    QB_ALLOC(b->d_case_end, sizeof(unsigned long long) * ncases);
    QB_ALLOC(b->d_collect, sizeof(int) * (2 * ncases + 2));
    QB_ALLOC(b->d_out15, sizeof(double) * 15);
    QB_ALLOC(b->d_ec, sizeof(ens::EnsCase) * ncases);
    QB_ALLOC(b->d_noise, sizeof(NoiseSpec) * ncases);
    QB_ALLOC(b->d_tw8, sizeof(cplx) * 240);
    b->soff.assign(ncases + 1, 0);
    for (int c = 0; c < ncases; ++c)
        b->soff[c + 1] = b->soff[c] + 2LL * b->cs[c].nmf * b->cs[c].nz + b->cs[c].nxy;
    const size_t small_bytes = sizeof(double) * ((size_t)b->soff[ncases] + ncases);
    QB_ALLOC(b->d_soff, sizeof(long long) * (ncases + 1));
    QB_ALLOC(b->d_small, small_bytes);
#undef QB_ALLOC
    if (cudaHostAlloc(&b->h_small, small_bytes, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc(&b->h_col, sizeof(int) * (2 * ncases + 2), cudaHostAllocDefault) != cudaSuccess ||
        cudaMemcpyAsync(b->d_soff, b->soff.data(), sizeof(long long) * (ncases + 1), cudaMemcpyHostToDevice,
                        b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess) {
        b->err = "staging buffers";
        return bail(QLGPU_ERR_CUDA);
    }
    if (guard_arm(b->guards, b->stream) != cudaSuccess) {
        b->err = "guard zones";
        return bail(QLGPU_ERR_CUDA);
    }
    {
        // 8-point twiddles of the queue engine, tw[q T + t] = exp(2 pi i q t / NZ), T = NZ / 8
        std::vector<double> tw8(480, 0.0);
        for (int NZ : {16, 32, 64, 128}) {
            const std::vector<double> t = twiddles(NZ, NZ / 8);
            std::copy(t.begin(), t.end(), tw8.begin() + 2 * tw8_offset(NZ));
        }
        if (cudaMemcpyAsync(b->d_tw8, tw8.data(), sizeof(double) * 480, cudaMemcpyHostToDevice, b->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(b->stream) != cudaSuccess) {
            b->err = "twiddle upload failed";
            return bail(QLGPU_ERR_CUDA);
        }
        b->queue_ok = b->model == MODEL_BQLIN;
        for (int c = 0; c < ncases; ++c)
            if (cases[c].NZ > 128) b->queue_ok = false;
        if (b->queue_ok) default_passes(b);
        const char* tr = std::getenv("QLGPU_TRACE");
        if (tr && tr[0] == '1' &&
            cudaMalloc(&b->d_qtrace, sizeof(unsigned long long) * 4 * QTRACE_MAX_CTAS_PER_SM * (size_t)b->sms) !=
                cudaSuccess) {
            b->err = "trace buffer";
            return bail(QLGPU_ERR_CUDA);
        }
        const char* e = std::getenv("QLGPU_BATCH_ENGINE");
        const bool force_items = e && std::string(e) == "items";
        b->engine = (b->queue_ok && !force_items) ? QLGPU_BATCH_ENGINE_QUEUE : QLGPU_BATCH_ENGINE_ITEMS;
    }
    if (cudaEventCreate(&b->ev[0]) != cudaSuccess || cudaEventCreate(&b->ev[1]) != cudaSuccess) {
        b->err = "event create failed";
        return bail(QLGPU_ERR_CUDA);
    }
    // initial mapping from the cost model: the widest CTA that fits
    b->wide_warps = 0;
    for (int w = b->bk.max_warps; w >= 1 && !b->wide_warps; --w) {
        int ps = 0;
        size_t sm = 0;
        if (width_limits(b, w, &ps, &sm)) b->wide_warps = w;
    }
    if (!b->wide_warps) {
        b->err = "batch: no CTA width fits (shared memory / TMEM)";
        return bail(QLGPU_ERR_UNSUPPORTED);
    }
    int rc = plan_and_apply(b, b->wide_warps, nullptr);
    if (rc) return bail(rc);
    rc = upload_descriptors(b);
    if (rc) return bail(rc);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
        b->err = "initialisation failed";
        return bail(QLGPU_ERR_CUDA);
    }
    *out = b;
    return QLGPU_OK;
}

int qlgpu_batch_dims(const qlgpu_batch_t* b, int c, int* nxy, int* nz, int* nmf) {
    if (!b || c < 0 || c >= b->ncases) return QLGPU_ERR_ARG;
    if (nxy) *nxy = b->cs[c].nxy;
    if (nz) *nz = b->cs[c].nz;
    if (nmf) *nmf = b->cs[c].nmf;
    return QLGPU_OK;
}

int qlgpu_batch_set_state(qlgpu_batch_t* b, int c, double t, const double* lin, const double* mf, const double* kx0) {
    if (!b) return QLGPU_ERR_ARG;
    if (b->a_count) return bfail(b, QLGPU_ERR_ARG, "asynchronous steps outstanding: collect them first");
    if (c < 0 || c >= b->ncases || !lin || !mf) return bfail(b, QLGPU_ERR_ARG, "bad case index or null state");
    QB_CK(cudaSetDevice(b->device));
    CaseHost& h = b->cs[c];
    const size_t nlin = (size_t)h.nxy * 4 * h.nz, nmfe = (size_t)h.nmf * h.nz;
    QB_CK(cudaMemcpyAsync(h.lin[b->cur], lin, nlin * sizeof(cplx), cudaMemcpyHostToDevice, b->stream));
    QB_CK(cudaMemcpyAsync(h.mf, mf, nmfe * sizeof(cplx), cudaMemcpyHostToDevice, b->stream));
    QB_CK(cudaMemcpyAsync(h.kx0, kx0 ? kx0 : h.kx_tab.data(), h.nxy * sizeof(double), cudaMemcpyHostToDevice,
                          b->stream));
    int rc = reset_case_clock(b, c, t);
    if (rc) return rc;
    QB_CK(cudaStreamSynchronize(b->stream));
    return QLGPU_OK;
}

int qlgpu_batch_get_state(qlgpu_batch_t* b, int c, double* t, double* lin, double* mf, double* kx0) {
    if (!b) return QLGPU_ERR_ARG;
    if (b->a_count) return bfail(b, QLGPU_ERR_ARG, "asynchronous steps outstanding: collect them first");
    if (c < 0 || c >= b->ncases) return bfail(b, QLGPU_ERR_ARG, "bad case index");
    QB_CK(cudaSetDevice(b->device));
    CaseHost& h = b->cs[c];
    const size_t nlin = (size_t)h.nxy * 4 * h.nz, nmfe = (size_t)h.nmf * h.nz;
    if (lin) QB_CK(cudaMemcpyAsync(lin, h.lin[b->cur], nlin * sizeof(cplx), cudaMemcpyDeviceToHost, b->stream));
    if (mf) QB_CK(cudaMemcpyAsync(mf, h.mf, nmfe * sizeof(cplx), cudaMemcpyDeviceToHost, b->stream));
    if (kx0) QB_CK(cudaMemcpyAsync(kx0, h.kx0, h.nxy * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    double tt = 0;
    QB_CK(cudaMemcpyAsync(&tt, &h.clk->t, sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    if (t) *t = tt;
    return QLGPU_OK;
}

int qlgpu_batch_set_states(qlgpu_batch_t* b, double t, const double* const* lin, const double* const* mf,
                           const double* const* kx0) {
    if (!b || !lin || !mf) return QLGPU_ERR_ARG;
    for (int c = 0; c < b->ncases; ++c)
        if (!lin[c] || !mf[c]) return bfail(b, QLGPU_ERR_ARG, "null state of case " + std::to_string(c));
    if (b->a_count) return bfail(b, QLGPU_ERR_ARG, "asynchronous steps outstanding: collect them first");
    QB_CK(cudaSetDevice(b->device));
    if (b->descr_dirty) {
        int rc = upload_descriptors(b);
        if (rc) return rc;
    }
    const int nc = b->ncases;
    double* flag = b->h_small + b->soff[nc];
    for (int c = 0; c < nc; ++c) {
        CaseHost& h = b->cs[c];
        const size_t nlin = (size_t)h.nxy * 4 * h.nz, nmfe = (size_t)h.nmf * h.nz;
        QB_CK(cudaMemcpyAsync(h.lin[b->cur], lin[c], nlin * sizeof(cplx), cudaMemcpyHostToDevice, b->stream));
        // the mean fields and kx0 go through the staging block (one copy for every case)
        double* sp = b->h_small + b->soff[c];
        std::memcpy(sp, mf[c], nmfe * sizeof(cplx));
        flag[c] = (kx0 && kx0[c]) ? 1.0 : 0.0;
        if (kx0 && kx0[c]) std::memcpy(sp + 2 * nmfe, kx0[c], h.nxy * sizeof(double));
    }
    QB_CK(cudaMemcpyAsync(b->d_small, b->h_small, sizeof(double) * ((size_t)b->soff[nc] + nc), cudaMemcpyHostToDevice,
                          b->stream));
    batch_scatter_small_kernel<<<nc, 128, 0, b->stream>>>(b->d_cases, nc, b->d_small, b->d_soff);
    QB_CK(cudaGetLastError());
    // the clocks of every case in one launch, after the copies above
    batch_set_clocks_kernel<<<nc, 128, 0, b->stream>>>(b->d_cases, nc, t);
    QB_CK(cudaGetLastError());
    QB_CK(cudaStreamSynchronize(b->stream));
    return QLGPU_OK;
}

int qlgpu_batch_get_states(qlgpu_batch_t* b, double* t, double* const* lin, double* const* mf, double* const* kx0) {
    if (!b) return QLGPU_ERR_ARG;
    if (b->a_count) return bfail(b, QLGPU_ERR_ARG, "asynchronous steps outstanding: collect them first");
    QB_CK(cudaSetDevice(b->device));
    if (b->descr_dirty) {
        int rc = upload_descriptors(b);
        if (rc) return rc;
    }
    const int nc = b->ncases;
    for (int c = 0; c < nc; ++c) {
        CaseHost& h = b->cs[c];
        const size_t nlin = (size_t)h.nxy * 4 * h.nz;
        if (lin && lin[c])
            QB_CK(cudaMemcpyAsync(lin[c], h.lin[b->cur], nlin * sizeof(cplx), cudaMemcpyDeviceToHost, b->stream));
    }
    // the mean fields, kx0 and clocks of every case through the staging block: one copy
    batch_gather_small_kernel<<<nc, 128, 0, b->stream>>>(b->d_cases, nc, b->d_small, b->d_soff);
    QB_CK(cudaGetLastError());
    QB_CK(cudaMemcpyAsync(b->h_small, b->d_small, sizeof(double) * ((size_t)b->soff[nc] + nc), cudaMemcpyDeviceToHost,
                          b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    for (int c = 0; c < nc; ++c) {
        const CaseHost& h = b->cs[c];
        const size_t nmfe = (size_t)h.nmf * h.nz;
        const double* sp = b->h_small + b->soff[c];
        if (mf && mf[c]) std::memcpy(mf[c], sp, nmfe * sizeof(cplx));
        if (kx0 && kx0[c]) std::memcpy(kx0[c], sp + 2 * nmfe, h.nxy * sizeof(double));
        if (t) t[c] = b->h_small[b->soff[nc] + c];
    }
    return QLGPU_OK;
}

int qlgpu_batch_diagnostics(qlgpu_batch_t* b, int c, double* out15) {
    if (!b || !out15) return QLGPU_ERR_ARG;
    if (c < 0 || c >= b->ncases) return bfail(b, QLGPU_ERR_ARG, "bad case index");
    QB_CK(cudaSetDevice(b->device));
    CaseHost& h = b->cs[c];
    double t = 0;
    QB_CK(cudaMemcpyAsync(&t, &h.clk->t, sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    h.var.diag(h.lin[b->cur], h.mf, h.kx0, h.ky, h.kxi, h.kyi, h.dp, t, b->d_out15, b->stream);
    QB_CK(cudaGetLastError());
    QB_CK(cudaMemcpyAsync(out15, b->d_out15, 15 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    return QLGPU_OK;
}

int qlgpu_batch_step(qlgpu_batch_t* b, int nsteps, int diag_every, double* diag_out, int max_diag, int* ndiag) {
    if (!b) return QLGPU_ERR_ARG;
    if (b->a_count) return bfail(b, QLGPU_ERR_ARG, "asynchronous steps outstanding: collect them first");
    if (nsteps < 0) return bfail(b, QLGPU_ERR_ARG, "nsteps < 0");
    if (diag_every > 0 && (!diag_out || !ndiag || max_diag < 1))
        return bfail(b, QLGPU_ERR_ARG, "diag_out, ndiag and max_diag >= 1 required");
    QB_CK(cudaSetDevice(b->device));
    if (diag_every > 0 && b->diag_cap != max_diag) {
        int rc = alloc_records(b, max_diag);
        if (rc) return rc;
    }
    for (int c = 0; c < b->ncases; ++c) {
        const double tv = diag_every > 0 ? diag_every * b->cs[c].p.dt : 0.0;
        if (tv != b->tv_set[c]) {
            b->tv_set[c] = tv;
            b->descr_dirty = true;
        }
    }
    int rc = run_launch(b, nsteps, diag_every > 0 ? 1 : 0);
    if (rc) return rc;
    const int nc = b->ncases;
    // the statuses and records come back through pinned buffers (asynchronous copies)
    batch_collect_kernel<<<(nc + 127) / 128, 128, 0, b->stream>>>(b->d_cases, nc, b->d_ctl, b->d_collect);
    QB_CK(cudaGetLastError());
    QB_CK(cudaMemcpyAsync(b->h_col, b->d_collect, sizeof(int) * (2 * (size_t)nc + 2), cudaMemcpyDeviceToHost,
                          b->stream));
    const size_t rec_bytes = sizeof(double) * 15 * (size_t)max_diag * nc;
    if (diag_every > 0) QB_CK(cudaMemcpyAsync(b->h_diag, b->d_diag, rec_bytes, cudaMemcpyDeviceToHost, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    if (diag_every > 0) std::memcpy(diag_out, b->h_diag, rec_bytes);
    if (b->h_col[2 * nc] & QLGPU_STATUS_TIMEOUT) return check_launch_status(b);
    int rc2 = step_records(b, b->h_col, diag_every, max_diag, ndiag);
    if (rc2) return rc2;
    return debug_verify(b);
}

int qlgpu_batch_step_async(qlgpu_batch_t* b, int nsteps, int diag_every, int max_diag) {
    if (!b) return QLGPU_ERR_ARG;
    if (nsteps < 1) return bfail(b, QLGPU_ERR_ARG, "nsteps < 1");
    if (diag_every > 0 && max_diag < 1) return bfail(b, QLGPU_ERR_ARG, "max_diag >= 1 required");
    if (b->a_count == 2) return bfail(b, QLGPU_ERR_ARG, "two asynchronous steps outstanding: collect one first");
    QB_CK(cudaSetDevice(b->device));
    const int nc = b->ncases;
    if (diag_every > 0 && b->diag_cap != max_diag) {
        if (b->a_count) return bfail(b, QLGPU_ERR_ARG, "max_diag differs from the outstanding step's");
        int rc = alloc_records(b, max_diag);
        if (rc) return rc;
    }
    for (int c = 0; c < nc; ++c) {
        const double tv = diag_every > 0 ? diag_every * b->cs[c].p.dt : 0.0;
        if (tv != b->tv_set[c]) {
            b->tv_set[c] = tv;
            b->descr_dirty = true;
        }
    }
    // new descriptors must not be written under a running launch
    if (b->descr_dirty && b->a_count) QB_CK(cudaStreamSynchronize(b->stream));
    const int slot = (b->a_head + b->a_count) & 1;
    qlgpu_batch::AsyncSlot& a = b->aslot[slot];
    if (!a.col) {
        QB_CK(cudaHostAlloc(&a.col, sizeof(int) * (2 * (size_t)nc + 2), cudaHostAllocDefault));
        QB_CK(cudaHostAlloc(&a.ctl, sizeof(BatchCtl), cudaHostAllocDefault));
        QB_CK(cudaEventCreateWithFlags(&a.done, cudaEventDisableTiming));
    }
    const size_t rec_bytes = sizeof(double) * 15 * (size_t)std::max(max_diag, 1) * nc;
    if (diag_every > 0 && a.max_diag != max_diag) {
        if (a.diag) cudaFreeHost(a.diag);
        a.diag = nullptr;
        a.max_diag = 0;
        QB_CK(cudaHostAlloc(&a.diag, rec_bytes, cudaHostAllocDefault));
        a.max_diag = max_diag;
    }
    int rc = run_launch(b, nsteps, diag_every > 0 ? 1 : 0);
    if (rc) return rc;
    // the copies are queued behind the launch and ahead of the next one, which reuses the buffers
    batch_collect_kernel<<<(nc + 127) / 128, 128, 0, b->stream>>>(b->d_cases, nc, b->d_ctl, b->d_collect);
    QB_CK(cudaGetLastError());
    QB_CK(cudaMemcpyAsync(a.col, b->d_collect, sizeof(int) * (2 * (size_t)nc + 2), cudaMemcpyDeviceToHost, b->stream));
    QB_CK(cudaMemcpyAsync(a.ctl, b->d_ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, b->stream));
    if (diag_every > 0) QB_CK(cudaMemcpyAsync(a.diag, b->d_diag, rec_bytes, cudaMemcpyDeviceToHost, b->stream));
    QB_CK(cudaEventRecord(a.done, b->stream));
    a.diag_every = diag_every;
    b->a_count += 1;
    return QLGPU_OK;
}

int qlgpu_batch_step_collect(qlgpu_batch_t* b, double* diag_out, int max_diag, int* ndiag) {
    if (!b) return QLGPU_ERR_ARG;
    if (b->a_count == 0) return bfail(b, QLGPU_ERR_ARG, "no asynchronous step outstanding");
    qlgpu_batch::AsyncSlot& a = b->aslot[b->a_head];
    if (a.diag_every > 0 && (!diag_out || !ndiag || max_diag != a.max_diag))
        return bfail(b, QLGPU_ERR_ARG, "diag_out, ndiag and the step's max_diag required");
    QB_CK(cudaSetDevice(b->device));
    QB_CK(cudaEventSynchronize(a.done));
    b->a_head ^= 1;
    b->a_count -= 1;
    const int nc = b->ncases;
    if (a.diag_every > 0) std::memcpy(diag_out, a.diag, sizeof(double) * 15 * (size_t)max_diag * nc);
    if (a.col[2 * nc] & QLGPU_STATUS_TIMEOUT) return launch_timeout(b, *a.ctl);
    return step_records(b, a.col, a.diag_every, max_diag, ndiag);
}

int qlgpu_batch_step_timed(qlgpu_batch_t* b, int nsteps, float* ms) {
    if (!b || !ms || nsteps < 1) return QLGPU_ERR_ARG;
    if (b->a_count) return bfail(b, QLGPU_ERR_ARG, "asynchronous steps outstanding: collect them first");
    QB_CK(cudaSetDevice(b->device));
    for (int c = 0; c < b->ncases; ++c)
        if (b->tv_set[c] != 0.0) {
            b->tv_set[c] = 0.0;
            b->descr_dirty = true;
        }
    if (b->descr_dirty) {
        int rc = upload_descriptors(b);
        if (rc) return rc;
    }
    int rc = run_launch(b, nsteps, 0, b->ev[0]);
    if (rc) return rc;
    QB_CK(cudaEventRecord(b->ev[1], b->stream));
    QB_CK(cudaEventSynchronize(b->ev[1]));
    QB_CK(cudaEventElapsedTime(ms, b->ev[0], b->ev[1]));
    return check_launch_status(b);
}

int qlgpu_batch_tune(qlgpu_batch_t* b, int probe_steps, double* best_ms) {
    if (!b || probe_steps < 1) return QLGPU_ERR_ARG;
    if (b->a_count) return bfail(b, QLGPU_ERR_ARG, "asynchronous steps outstanding: collect them first");
    QB_CK(cudaSetDevice(b->device));
    // probes run on the batch's own buffers; a copy of the whole arena is restored afterwards
    unsigned char* backup = nullptr;
    QB_CK(cudaMalloc(&backup, b->arena_bytes));
    struct Restore {
        qlgpu_batch_t* b;
        unsigned char* p;
        int cur;
        ~Restore() {
            cudaMemcpyAsync(b->arena, p, b->arena_bytes, cudaMemcpyDeviceToDevice, b->stream);
            cudaStreamSynchronize(b->stream);
            cudaFree(p);
            b->cur = cur;
        }
    } restore{b, backup, b->cur};
    QB_CK(cudaMemcpyAsync(backup, b->arena, b->arena_bytes, cudaMemcpyDeviceToDevice, b->stream));
    for (int c = 0; c < b->ncases; ++c)
        if (b->tv_set[c] != 0.0) {
            b->tv_set[c] = 0.0;
            b->descr_dirty = true;
        }
    if (b->descr_dirty) {
        int rc = upload_descriptors(b);
        if (rc) return rc;
    }
    if (queue_usable(b)) {
        // queue engine: coordinate search over the CTA passes per chunk of each NZ class present
        if (b->qdirty) {
            int rc = queue_plan(b);
            if (rc) return rc;
        }
        // a probe: the best of three launches of at least 6 steps after a warm-up launch (one
        // short launch per candidate let launch-to-launch noise pick the passes)
        const int qsteps = std::max(probe_steps, 6);
        auto qprobe = [&](double* ms) -> int {
            QB_CK(ensure_smem_attr(ens::kernel(b->integ, queue_rec(b)), b->qsmem));
            double best_of = 1e300;
            for (int rep = 0; rep < 4; ++rep) {  // the first launch of a plan is a warm-up
                QB_CK(cudaEventRecord(b->ev[0], b->stream));
                QB_CK(enqueue_queue(b, qsteps, 0));
                QB_CK(cudaEventRecord(b->ev[1], b->stream));
                QB_CK(cudaEventSynchronize(b->ev[1]));
                float f = 0;
                QB_CK(cudaEventElapsedTime(&f, b->ev[0], b->ev[1]));
                b->cur = (b->cur + qsteps) & 1;
                int rc = check_launch_status(b);
                if (rc) return rc;
                if (rep > 0) best_of = std::min(best_of, (double)f);
            }
            *ms = best_of;
            return QLGPU_OK;
        };
        bool present[4] = {false, false, false, false};
        for (const CaseHost& h : b->cs) present[ens_class(h.NZ)] = true;
        double best = 0;
        int rc = qprobe(&best);
        if (rc) return rc;
        // two sweeps: the best passes of a class depend on the other classes' chunks
        for (int sweep = 0; sweep < 2; ++sweep)
            for (int cls = 3; cls >= 0; --cls) {
                if (!present[cls]) continue;
                const int keep = b->qpasses[cls];
                int bestp = keep;
                for (int pp : {1, 2, 3, 4, 6, 8}) {
                    if (pp == keep) continue;
                    b->qpasses[cls] = pp;
                    rc = queue_plan(b);
                    if (rc) return rc;
                    double ms = 0;
                    rc = qprobe(&ms);
                    if (rc) return rc;
                    if (ms < best) {
                        best = ms;
                        bestp = pp;
                    }
                }
                b->qpasses[cls] = bestp;
            }
        rc = queue_plan(b);
        if (rc) return rc;
        if (best_ms) *best_ms = best;
        return QLGPU_OK;
    }
    struct Best {
        double ms = 1e300;
        int warps = 0, per_sm = 0;
        size_t smem = 0;
        std::vector<int> k;
        std::vector<std::vector<Item>> bins;
        CostModel cm;
    } best;
    std::vector<unsigned long long> ends(b->ncases);
    // one probe of the current mapping: launch time and per-case stage times (us per stage)
    auto probe = [&](double* ms, std::vector<double>* ystage) -> int {
        QB_CK(ensure_smem_attr(b->bk.kernel(), b->smem));
        QB_CK(cudaEventRecord(b->ev[0], b->stream));
        QB_CK(enqueue_launch(b, probe_steps, 0));
        QB_CK(cudaEventRecord(b->ev[1], b->stream));
        QB_CK(cudaEventSynchronize(b->ev[1]));
        float f = 0;
        QB_CK(cudaEventElapsedTime(&f, b->ev[0], b->ev[1]));
        b->cur = (b->cur + probe_steps) & 1;
        int rc = check_launch_status(b);
        if (rc) return rc;
        BatchCtl ctl;
        QB_CK(cudaMemcpy(&ctl, b->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
        QB_CK(cudaMemcpy(ends.data(), b->d_case_end, sizeof(unsigned long long) * b->ncases, cudaMemcpyDeviceToHost));
        *ms = f;
        if (ystage) {
            ystage->resize(b->ncases);
            for (int c = 0; c < b->ncases; ++c)
                (*ystage)[c] = (double)(long long)(ends[c] - ctl.t_start) * 1e-3 / (3.0 * probe_steps);
        }
        return QLGPU_OK;
    };
    // least-squares fit of alpha, beta, r[NZ] to the per-case stage times, ridge towards the prior
    auto fit = [&](const std::vector<double>& y, CostModel& cm) {
        const int nu = 2 + NCLASS;
        // the CTA that finished a case last is modelled as the most loaded CTA holding one of its items
        std::vector<double> load(b->ctas.size(), 0.0);
        for (size_t j = 0; j < b->ctas.size(); ++j)
            for (int i = 0; i < b->ctas[j].nslots; ++i) {
                const BatchSlot& s = b->ctas[j].slot[i];
                load[j] += cm.beta + rounds_of(b->cs[s.c], s.ncta, b->warps) * cm.r[nz_class(s.NZ)];
            }
        std::vector<int> crit(b->ncases, -1);
        for (size_t j = 0; j < b->ctas.size(); ++j)
            for (int i = 0; i < b->ctas[j].nslots; ++i) {
                const int c = b->ctas[j].slot[i].c;
                if (crit[c] < 0 || load[j] > load[crit[c]]) crit[c] = (int)j;
            }
        std::vector<std::vector<double>> rows(b->ncases, std::vector<double>(nu, 0.0));
        for (int c = 0; c < b->ncases; ++c) {
            std::vector<double>& r = rows[c];
            r[0] = 1.0;
            if (crit[c] < 0) continue;
            const BatchCta& m = b->ctas[crit[c]];
            for (int i = 0; i < m.nslots; ++i) {
                const BatchSlot& s = m.slot[i];
                r[1] += 1.0;
                r[2 + nz_class(s.NZ)] += rounds_of(b->cs[s.c], s.ncta, b->warps);
            }
        }
        double prior[2 + NCLASS];
        prior[0] = cm.alpha;
        prior[1] = cm.beta;
        for (int j = 0; j < NCLASS; ++j) prior[2 + j] = cm.r[j];
        std::vector<double> M((size_t)nu * nu, 0.0), v(nu, 0.0);
        const double lam = 1e-3;
        for (int c = 0; c < b->ncases; ++c)
            for (int i = 0; i < nu; ++i) {
                v[i] += rows[c][i] * y[c];
                for (int j = 0; j < nu; ++j) M[i * nu + j] += rows[c][i] * rows[c][j];
            }
        for (int i = 0; i < nu; ++i) {
            const double w = lam * (1.0 + M[i * nu + i]);
            M[i * nu + i] += w;
            v[i] += w * prior[i];
        }
        // Gaussian elimination with partial pivoting
        std::vector<double> x(nu, 0.0);
        for (int col = 0; col < nu; ++col) {
            int piv = col;
            for (int r = col + 1; r < nu; ++r)
                if (std::fabs(M[r * nu + col]) > std::fabs(M[piv * nu + col])) piv = r;
            for (int j = 0; j < nu; ++j) std::swap(M[col * nu + j], M[piv * nu + j]);
            std::swap(v[col], v[piv]);
            const double d = M[col * nu + col];
            if (std::fabs(d) < 1e-300) return;
            for (int r = col + 1; r < nu; ++r) {
                const double f = M[r * nu + col] / d;
                for (int j = col; j < nu; ++j) M[r * nu + j] -= f * M[col * nu + j];
                v[r] -= f * v[col];
            }
        }
        for (int i = nu - 1; i >= 0; --i) {
            double s = v[i];
            for (int j = i + 1; j < nu; ++j) s -= M[i * nu + j] * x[j];
            x[i] = s / M[i * nu + i];
        }
        cm.alpha = std::max(0.0, x[0]);
        cm.beta = std::max(0.0, x[1]);
        for (int j = 0; j < NCLASS; ++j)
            if (x[2 + j] > 0) cm.r[j] = x[2 + j];
    };
    int rc = QLGPU_OK;
    for (int warps : {b->wide_warps, std::max(1, b->wide_warps / 2)}) {
        int per_sm = 0;
        size_t smem = 0;
        if (!width_limits(b, warps, &per_sm, &smem)) continue;
        const int G = std::min(b->sms * per_sm, b->sms * 2);
        CostModel cm = b->cost;
        for (int pass = 0; pass < 3; ++pass) {
            std::vector<int> k;
            std::vector<std::vector<Item>> bins;
            if (!plan(b, warps, G, cm, nullptr, k, bins, nullptr)) break;
            rc = apply_mapping(b, warps, per_sm, smem, k, bins);
            if (rc) return rc;
            double ms = 0;
            std::vector<double> y;
            rc = probe(&ms, nullptr);  // warm-up of this mapping
            if (rc) return rc;
            rc = probe(&ms, &y);
            if (rc) return rc;
            if (ms < best.ms) {
                best.ms = ms;
                best.warps = warps;
                best.per_sm = per_sm;
                best.smem = smem;
                best.k = k;
                best.bins = bins;
                best.cm = cm;
            }
            fit(y, cm);
        }
    }
    if (best.warps == 0) return bfail(b, QLGPU_ERR_UNSUPPORTED, "batch tune: no CTA width fits");
    b->cost = best.cm;
    rc = apply_mapping(b, best.warps, best.per_sm, best.smem, best.k, best.bins);
    if (rc) return rc;
    if (best_ms) *best_ms = best.ms;
    return QLGPU_OK;
}

int qlgpu_batch_cost_model(const qlgpu_batch_t* b, double* out7) {
    if (!b || !out7) return QLGPU_ERR_ARG;
    out7[0] = b->cost.alpha;
    out7[1] = b->cost.beta;
    for (int i = 0; i < NCLASS; ++i) out7[2 + i] = b->cost.r[i];
    return QLGPU_OK;
}

int qlgpu_batch_mapping(const qlgpu_batch_t* b, int* info4, int* ncta) {
    if (!b) return QLGPU_ERR_ARG;
    if (queue_usable(b)) {
        if (b->qdirty) {
            int rc = queue_plan(const_cast<qlgpu_batch_t*>(b));
            if (rc) return rc;
        }
        if (info4) {
            info4[0] = ens::threads() / 32;
            info4[1] = b->qgrid;
            info4[2] = 1;
            info4[3] = (int)b->qsmem;
        }
        if (ncta)
            for (int c = 0; c < b->ncases; ++c) ncta[c] = b->ec[c].nch;
        return QLGPU_OK;
    }
    if (info4) {
        info4[0] = b->warps;
        info4[1] = b->grid;
        info4[2] = b->per_sm;
        info4[3] = (int)b->smem;
    }
    if (ncta)
        for (int c = 0; c < b->ncases; ++c) ncta[c] = b->ncta[c];
    return QLGPU_OK;
}

int qlgpu_batch_set_mapping(qlgpu_batch_t* b, int warps, const int* ncta) {
    if (!b || !ncta) return QLGPU_ERR_ARG;
    if (warps < 1 || warps > b->wide_warps)
        return bfail(b, QLGPU_ERR_ARG, "warps per CTA must be 1 ... " + std::to_string(b->wide_warps) + " for this batch");
    QB_CK(cudaSetDevice(b->device));
    b->engine = QLGPU_BATCH_ENGINE_ITEMS;  // an explicit CTA mapping is a work-item mapping
    drop_graphs(b);
    return plan_and_apply(b, warps, ncta);
}

int qlgpu_batch_status(qlgpu_batch_t* b, int* case_status, int* launch_status) {
    if (!b) return QLGPU_ERR_ARG;
    QB_CK(cudaSetDevice(b->device));
    if (case_status) {
        std::vector<int> col(2 * (size_t)b->ncases + 2);
        batch_collect_kernel<<<(b->ncases + 127) / 128, 128, 0, b->stream>>>(b->d_cases, b->ncases, b->d_ctl,
                                                                              b->d_collect);
        QB_CK(cudaGetLastError());
        QB_CK(cudaMemcpyAsync(col.data(), b->d_collect, col.size() * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
        QB_CK(cudaStreamSynchronize(b->stream));
        for (int c = 0; c < b->ncases; ++c) case_status[c] = col[2 * c];
    }
    if (launch_status) {
        BatchCtl ctl;
        QB_CK(cudaMemcpyAsync(&ctl, b->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, b->stream));
        QB_CK(cudaStreamSynchronize(b->stream));
        *launch_status = ctl.status;
    }
    return QLGPU_OK;
}

int qlgpu_batch_set_wait(qlgpu_batch_t* b, double seconds) {
    if (!b || !(seconds > 0) || seconds > 60) return QLGPU_ERR_ARG;
    b->wait_ns = (long long)(seconds * 1e9);
    drop_graphs(b);
    return QLGPU_OK;
}

int qlgpu_batch_debug_drop_item(qlgpu_batch_t* b, int c) {
    if (!b) return QLGPU_ERR_ARG;
    if (queue_usable(b)) {
        QB_CK(cudaSetDevice(b->device));
        if (b->qdirty) {
            int rc = queue_plan(b);
            if (rc) return rc;
        }
        if (c < 0 || c >= b->ncases || b->ec[c].nch < 2)
            return bfail(b, QLGPU_ERR_ARG, "drop item: the case needs two or more chunks");
        b->drop_case = c;
        return queue_plan(b);
    }
    if (c < 0 || c >= b->ncases || b->ncta[c] < 2)
        return bfail(b, QLGPU_ERR_ARG, "drop item: the case needs two or more CTAs");
    QB_CK(cudaSetDevice(b->device));
    std::vector<BatchCta> ctas = b->ctas;
    bool done = false;
    for (size_t j = 0; j < ctas.size() && !done; ++j)
        for (int i = 0; i < ctas[j].nslots; ++i)
            if (ctas[j].slot[i].c == c && ctas[j].slot[i].cta == b->ncta[c] - 1) {
                for (int m = i + 1; m < ctas[j].nslots; ++m) ctas[j].slot[m - 1] = ctas[j].slot[m];
                ctas[j].nslots -= 1;
                done = true;
                break;
            }
    if (!done) return bfail(b, QLGPU_ERR_ARG, "drop item: item not found");
    QB_CK(cudaMemcpyAsync(b->d_ctas, ctas.data(), sizeof(BatchCta) * ctas.size(), cudaMemcpyHostToDevice, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    b->ctas = ctas;
    drop_graphs(b);
    return QLGPU_OK;
}

int qlgpu_batch_set_engine(qlgpu_batch_t* b, int engine) {
    if (!b) return QLGPU_ERR_ARG;
    if (engine == QLGPU_BATCH_ENGINE_AUTO) engine = b->queue_ok ? QLGPU_BATCH_ENGINE_QUEUE : QLGPU_BATCH_ENGINE_ITEMS;
    if (engine != QLGPU_BATCH_ENGINE_ITEMS && engine != QLGPU_BATCH_ENGINE_QUEUE)
        return bfail(b, QLGPU_ERR_ARG, "unknown batch engine");
    if (engine == QLGPU_BATCH_ENGINE_QUEUE && !b->queue_ok)
        return bfail(b, QLGPU_ERR_UNSUPPORTED, "queue engine: MHD_BQlin batches with every NZ <= 128 only");
    QB_CK(cudaSetDevice(b->device));
    b->engine = engine;
    b->drop_case = -1;
    b->qdirty = true;
    drop_graphs(b);
    if (engine == QLGPU_BATCH_ENGINE_ITEMS) {
        // a mapping that a dropped work item changed is replaced by the cost model's
        return plan_and_apply(b, b->warps, nullptr);
    }
    return QLGPU_OK;
}

int qlgpu_batch_engine(const qlgpu_batch_t* b, int* engine) {
    if (!b || !engine) return QLGPU_ERR_ARG;
    *engine = queue_usable(b) ? QLGPU_BATCH_ENGINE_QUEUE : QLGPU_BATCH_ENGINE_ITEMS;
    return QLGPU_OK;
}

int qlgpu_batch_set_chunks(qlgpu_batch_t* b, const int* passes4) {
    if (!b || !passes4) return QLGPU_ERR_ARG;
    for (int i = 0; i < 4; ++i)
        if (passes4[i] < 1 || passes4[i] > 256) return bfail(b, QLGPU_ERR_ARG, "passes per chunk must be 1 ... 256");
    if (!b->queue_ok) return bfail(b, QLGPU_ERR_UNSUPPORTED, "queue engine: MHD_BQlin batches with every NZ <= 128 only");
    QB_CK(cudaSetDevice(b->device));
    for (int i = 0; i < 4; ++i) b->qpasses[i] = passes4[i];
    b->engine = QLGPU_BATCH_ENGINE_QUEUE;
    b->drop_case = -1;
    b->qdirty = true;
    drop_graphs(b);
    return queue_plan(b);
}

int qlgpu_batch_chunks(const qlgpu_batch_t* b, int* passes4) {
    if (!b || !passes4) return QLGPU_ERR_ARG;
    for (int i = 0; i < 4; ++i) passes4[i] = b->qpasses[i];
    return QLGPU_OK;
}

int qlgpu_batch_queue_trace(qlgpu_batch_t* b, double* out4) {
    if (!b || !out4) return QLGPU_ERR_ARG;
    if (!b->d_qtrace) return bfail(b, QLGPU_ERR_UNSUPPORTED, "queue trace: set QLGPU_TRACE=1 before qlgpu_batch_create");
    QB_CK(cudaSetDevice(b->device));
    std::vector<unsigned long long> t(4 * (size_t)b->qgrid);
    QB_CK(cudaMemcpy(t.data(), b->d_qtrace, sizeof(unsigned long long) * t.size(), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 4; ++k) out4[k] = 0.0;
    for (int g = 0; g < b->qgrid; ++g)
        for (int k = 0; k < 4; ++k) out4[k] += (double)t[4 * (size_t)g + k];
    for (int k = 0; k < 3; ++k) out4[k] *= 1e-3 / b->qgrid;  // us per CTA
    out4[3] /= b->qgrid;                                     // chunks per CTA
    return QLGPU_OK;
}

int qlgpu_batch_stream(qlgpu_batch_t* b, void** stream) {
    if (!b || !stream) return QLGPU_ERR_ARG;
    *stream = (void*)b->stream;
    return QLGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Internal entry points for the adjoint (qlgpu_batch_internal.h)
// ---------------------------------------------------------------------------
int qlgpu_batch_case_dev(qlgpu_batch_t* b, int c, BatchCaseDev* out) {
    if (!b || c < 0 || c >= b->ncases || !out) return QLGPU_ERR_ARG;
    CaseHost& h = b->cs[c];
    out->lin = h.lin[b->cur];
    out->mf = h.mf;
    out->kx0 = h.kx0;
    out->clk = h.clk;
    out->nlin = (size_t)h.nxy * 4 * h.nz;
    out->nmfe = (size_t)h.nmf * h.nz;
    out->nxy = h.nxy;
    return QLGPU_OK;
}

int qlgpu_batch_set_record(qlgpu_batch_t* b, int c, cplx* rec_lin, cplx* rec_mf, double* rec_kx, double* rec_t,
                           CnRec* rec_cn) {
    if (!b || c < 0 || c >= b->ncases) return QLGPU_ERR_ARG;
    CaseHost& h = b->cs[c];
    h.rec_lin = rec_lin;
    h.rec_mf = rec_lin ? rec_mf : nullptr;
    h.rec_kx = rec_lin ? rec_kx : nullptr;
    h.rec_t = rec_lin ? rec_t : nullptr;
    h.rec_cn = rec_lin ? rec_cn : nullptr;
    b->descr_dirty = true;
    return QLGPU_OK;
}

cudaStream_t qlgpu_batch_cuda_stream(qlgpu_batch_t* b) { return b ? b->stream : nullptr; }

int qlgpu_batch_debug_guard_poke(qlgpu_batch_t* b, int zone) {
    if (!b) return QLGPU_ERR_ARG;
    if (!QLGPU_DEBUG_BUILD) return bfail(b, QLGPU_ERR_UNSUPPORTED, "guard zones exist in the debug build only");
    if (zone < 0 || zone >= (int)b->guards.zones.size()) return bfail(b, QLGPU_ERR_ARG, "no such guard zone");
    QB_CK(cudaSetDevice(b->device));
    QB_CK(guard_poke(b->guards, zone, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    return QLGPU_OK;
}

int qlgpu_batch_set_noise(qlgpu_batch_t* b, int c, double f_noise, double k_low, double k_high,
                          unsigned long long seed, int drive_only_velocity, int drive_only_magnetic) {
    if (!b) return QLGPU_ERR_ARG;
    if (c < 0 || c >= b->ncases) return bfail(b, QLGPU_ERR_ARG, "case index out of range");
    if (!std::isfinite(f_noise) || !(k_low >= 0) || !(k_high >= k_low))
        return bfail(b, QLGPU_ERR_ARG, "noise: finite f_noise, 0 <= k_low <= k_high");
    CaseHost& h = b->cs[c];
    if ((drive_only_velocity || drive_only_magnetic) && h.p.model != QLGPU_MODEL_MHD_FULLQLIN)
        return bfail(b, QLGPU_ERR_UNSUPPORTED, "drive_only_velocity / drive_only_magnetic are MHD_FullQlin inputs");
    QB_CK(cudaSetDevice(b->device));
    const NoiseSpec ns = noise_spec(h.p, h.NZ, h.p.dt, f_noise, k_low, k_high, seed, drive_only_velocity != 0,
                                    drive_only_magnetic != 0);
    QB_CK(cudaMemcpyAsync(b->d_noise + c, &ns, sizeof(ns), cudaMemcpyHostToDevice, b->stream));
    QB_CK(cudaStreamSynchronize(b->stream));
    const bool on = f_noise != 0.0;
    if (on != h.noise_on) {
        h.noise_on = on;
        b->descr_dirty = true;
    }
    return QLGPU_OK;
}
