// qlgpu_types.h -- device-side parameter and argument blocks shared by the
// host code (qlgpu.cu) and the stage kernels (qlgpu_stage.cuh).
#pragma once

namespace qlgpu {

struct cplx;

enum { MODEL_BQLIN = 0, MODEL_FULLQLIN = 1 };
enum { INTEG_EXP = 0, INTEG_CN = 1 };

// Run constants, fixed for a handle.
struct DevParams {
    int nxy, nz, NZ, nmf;
    double q;       // shear
    double Omega;   // rotation: 2q/3 for MHD_BQlin (MHD_BQlin.cpp:19), input omega for FullQlin
    double nu, eta, etanu;  // etanu = eta/nu (MHD_BQlin.cpp:251)
    double cb;              // L_b = cb * lap: (eta/nu) nu for MHD_BQlin, eta for MHD_FullQlin
    int factored;           // the integrating factor exp(linC L) factors as exp(linC c h) exp(linC c kz2)
    double B0z;
    int visc_half;  // viscosity_order/2 (integer division, MHD_FullQlin.cpp:372)
    int ql;         // QuasiLinear?
    int remap;      // Remap?
    double kzL;     // 2 pi / Lz
    double fac;     // 1/NZ (fftwPlans.cpp:30)
    double rs_fac;  // 1/(Ny Nx)^2 (MHD_BQlin.cpp:56)
    double divfac;  // Lz/(Nx Ny NZ)^2 (MHD_BQlin.cpp:420)
    double divMF;   // Lz/NZ^2 (MHD_BQlin.cpp:434)
    double remap_thresh;  // (Nx-1)/2.0 * kxLfac (MHD_BQlin.cpp:322)
    double remap_shift;   // (Nx-1) * kxLfac     (MHD_BQlin.cpp:324)
    double dt;
    double tv_interval;   // diagnostic interval (<= 0: none)
    double kzmax;         // 2 pi/Lz * (NZ/3) for etaK (MHD_BQlin.cpp:476)
};

// Mutable per-handle clock and reduction state, in device memory.
struct DevClock {
    double t;          // current time (t += dt after each step, main.cpp:116)
    double timevar;    // SP.timevar_t accumulator (main.cpp:117,127-130)
    double t_old;      // CN: time at which the previous stage's operator was evaluated
    double dtlin_old;  // CN: dt_lin of the previous stage
    int old_init;      // CN: 1 -> the old operator is linearOPs_Init(t0) (RK3CN.cpp:57)
    int ndiag;         // diagnostic records written
    int since;         // steps since the last diagnostic record
    int status;        // error bits (QLGPU_STATUS_*)
    unsigned cnt_top;
    int mfr_valid;     // mean-field profiles cache holds the current mean field
    unsigned cnt_group[64];
    unsigned long long nstep;  // steps since the clock was set: the noise counter of the next step
};

// Driving noise of one case (Model::DrivingNoise, MHD_BQlin.cpp:558-618 and
// MHD_FullQlin.cpp:786-1045), added to every mode after its last-stage update.
struct NoiseSpec {
    double lo2, hi2;     // noise_range_ bounds squared (MHD_FullQlin.cpp:51-52)
    double multfac;      // dt (Nx Ny NZ)^2 mult_noise_fac_ (MHD_FullQlin.cpp:63-66,804)
    double sd;           // f_noise/sqrt(2), the standard deviation of each part (:45)
    unsigned long long seed;
    int pair_ky0;        // MHD_FullQlin: ky = 0 modes driven in conjugate pairs (dont_drive_ky0_modes_ = 0)
    int drive_u, drive_b;  // (u, zeta) / (b, eta) driven: !drive_only_magnetic / !drive_only_velocity (:21-22)
    int nxh, nyh;        // Nx/2, Ny/2: the Kdata layout that locates a kx > 0 mode's kx < 0 partner
    int pad;
};

// The Crank-Nicolson old-operator fields of a DevClock at a stage's start (the
// record the adjoint of RK3CN reads): the same byte layout as DevClock from t_old.
struct CnRec {
    double t_old, dtlin_old;
    int old_init, pad;
};

// Coefficients of one stage (RK3CN_Elin.cpp:89-91,122-125,155-158;
// RK3CN.cpp:92-94,...).
struct StageConst {
    double t_off;     // stage time = t + t_off (dt*{0, p1, p2})
    double dt_lin;    // operators evaluated at t_s + dt_lin
    double linC;      // dt*(a+b) (exp) or dt/2*(a+b) (CN)
    double n1, n2;    // a*dt, b*dt
    int has_prev;     // stage uses F of the previous stage
    int last;         // last stage of the step: advance time, remap, diagnostics
    int abs_time;     // Model::rhs mode: stage time is t_off itself
    int pad;
};

struct StageArgs {
    const cplx* lin_in;
    cplx* lin_out;
    const cplx* Fprev;
    cplx* Fout;
    cplx* mf;               // mean fields, updated in place by the top CTA
    const cplx* Fmf_prev;
    cplx* Fmf_out;
    double* kx0;            // unsheared kx per mode (Kdata::kx), updated by remap
    const double* ky;
    const int* kxi;
    const int* kyi;
    const cplx* tw;         // twiddles exp(2 pi i n2 t/NZ), [P][T]
    const double* ilap2;    // [Ny/2][nz] 1/lap2 table (Kdata.cpp:100-119)
    double* partials;       // [grid][PL]
    double* gpartials;      // [ngroups][PL]
    DevClock* clk;
    double* diag_ring;      // [diag_cap][15]
    int diag_cap;
    int rhs_only;           // Model::rhs: write F (and linop) only, no update
    double* linop_out;      // rhs_only: [nxy][4][nz]
    unsigned long long* trace;  // optional %globaltimer trace (null: off), see qlgpu_kernel.cuh
    double* mfr_cache;      // [NMFR][NZ] real-space mean-field profiles written by the top CTA
    const double* ekz_tab;  // [2][nz] exp(linC nu kz2), exp(linC eta kz2) for this stage (null: compute)
    // optional record of the stage input (null: off): the fields [nxy][4][nz], the mean
    // fields [nmf][nz] and, in the first stage of a step, kx0 [nxy] and the clock t
    cplx* rec_lin;
    cplx* rec_mf;
    double* rec_kx;
    double* rec_t;
    CnRec* rec_cn;          // the CN old-operator fields at the stage start (null: off)
    const NoiseSpec* noise;  // last stage of a driven batch case: noise after each mode's update (null: off)
    StageConst sc;
};

// ---------------------------------------------------------------------------
// Batched ensemble (persistent kernel, qlgpu_batch.cuh)
// ---------------------------------------------------------------------------
constexpr int BATCH_MAX_SLOTS = 8;      // work items (case, CTA index) per CTA
constexpr int BATCH_EPOCH_STRIDE = 32;  // words between the per-case stage counters (one 128-byte line each)

// One case of a batch in device memory: its run constants and the arguments of
// its three stages for a step that starts from lin buffer 0 (the kernel swaps
// lin_in / lin_out on steps that start from buffer 1).
struct BatchCase {
    DevParams P;
    StageArgs A[3];
    const double* kx_init;  // the unsheared wavenumber table (Kdata::kx) on the device
    // optional record of every stage input of a launch (null: off): step n, stage s at
    // rec_lin + (3 n + s) nxy 4 nz, rec_mf + (3 n + s) nmf nz, rec_kx + n nxy, rec_t + n
    cplx* rec_lin;
    cplx* rec_mf;
    double* rec_kx;
    double* rec_t;
    CnRec* rec_cn;   // [3 n + s]
};

// One work item: CTA number `cta` of the `ncta` CTAs that step case `c`.
struct BatchSlot {
    int c, cta, ncta, NZ;
};

// The work list of one CTA of the persistent launch.
struct BatchCta {
    int nslots;
    int tcols;  // TMEM columns the CTA allocates (the largest of its slots' needs)
    int pad[2];
    BatchSlot slot[BATCH_MAX_SLOTS];
};

// Launch-wide control words (zeroed before every launch).
struct BatchCtl {
    int status;      // QLGPU_STATUS_TIMEOUT when a wait gave up
    int abort;       // set with the timeout: every waiting CTA leaves
    int fail_case;   // case and stage of the first wait that gave up
    int fail_stage;
    unsigned long long t_start;  // %globaltimer at the start of CTA 0
    unsigned next;               // chunk-queue engine: next ticket
    int fail_where;              // 0 a wait for other CTAs of the case, 1 a wait for a staged copy
};

struct BatchLaunch {
    const BatchCase* cases;
    const BatchCta* ctas;
    unsigned* epoch;               // [ncases * BATCH_EPOCH_STRIDE] stages completed in this launch
    BatchCtl* ctl;
    unsigned long long* case_end;  // [ncases] %globaltimer when the case finished its last stage
    int nsteps;
    int parity;                    // 1: the first step starts from lin buffer 1
    long long wait_ns;             // bound on one wait for the other CTAs of a case
    int ncases;
    int pad;
};

// ---------------------------------------------------------------------------
// Chunk-queue engine of the batch (qlgpu_ens.cuh)
// ---------------------------------------------------------------------------
namespace ens {

// One entry of a round: chunk j of case c.
struct RoundItem {
    int c, j;
};

// Per-case constants of the queue engine.
struct EnsCase {
    int NZ, nch, mpc, pad;  // NZ class, chunks per stage, modes per chunk
    const cplx* tw8;        // [8][NZ/8] twiddles of the 8-point layout
};

struct EnsLaunch {
    const BatchCase* cases;
    const EnsCase* ec;
    const RoundItem* round;  // [R] one stage of every case
    unsigned* epoch;         // [ncases * BATCH_EPOCH_STRIDE]: +0 stages released, +1 chunks done
    BatchCtl* ctl;
    unsigned* next;          // ticket counter
    unsigned long long* case_end;
    int R;                   // items per round
    int nrounds;             // 3 K
    int parity;
    int ncases;
    long long wait_ns;
    unsigned long long* trace;  // optional [grid][4] %globaltimer sums: stage waits, chunks, mean-field stages, count
};

}  // namespace ens

}  // namespace qlgpu

#define QLGPU_STATUS_NONFINITE 1   // solution::Check_Solution NaN/Inf (solution.cpp:194)
#define QLGPU_STATUS_UNSTABLE 2    // |mean field| > 1e20 (solution.cpp:184)
#define QLGPU_STATUS_DIAG_FULL 4   // diagnostic ring overflowed (records dropped)
#define QLGPU_STATUS_TIMEOUT 8     // batch: a CTA gave up waiting for the other CTAs of its case
#define QLGPU_STATUS_BOUNDS 16     // debug build: a device index check failed (the access was redirected)
#define QLGPU_STATUS_CANARY 32     // debug build: a guard zone after a device buffer was overwritten
