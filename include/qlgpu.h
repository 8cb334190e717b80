/*
 * qlgpu.h -- C ABI of the B200 (sm_100a) quasi-linear shearing-box time step.
 *
 * A drop-in for the time step of Cxb1993/ql_dns: the Model / Integrator /
 * solution C++ API of the reference (QL_DNS/Models/Model.h:24-112,
 * QL_DNS/Integrators/Integrator.h:20-28, QL_DNS/solution.h:23-49) maps onto
 * these entry points.  Plain pointers and sizes only; every function returns
 * a status code (QLGPU_OK = 0) where the reference calls ABORT / MPI_Abort
 * (QL_DNS/General_Definitions.h:68-72).
 *
 * Data layout (host and device alike, interleaved re/im doubles):
 *   lin[nxy][4][nz]   fluctuations (u, zeta, b, eta) = (u_x, w_x, b_x, j_x),
 *                     kz in dealiased order 0..(nz-1)/2, -(nz-1)/2..-1
 *                     (QL_DNS/solution.cpp:17-25; solution::pLin(i, V))
 *   mf[nmf][nz]       mean fields (Bx, By[, Ux, Uy]) (solution.cpp:27-31;
 *                     solution::pMF(i))
 *   kx0[nxy]          unsheared kx of every mode (Kdata::kx imaginary part,
 *                     QL_DNS/Auxiliary/Kdata.cpp:30-46), shifted by remaps
 * nz = 1 + 2*floor(NZ/3), nxy = (nx-1)*(ny/2) (QL_DNS/Models/Model.h:34-36).
 *
 * Threading: one host thread per handle at a time.  Each handle owns its
 * device memory and one CUDA stream; host buffers are read or written only
 * during the call.
 */
#ifndef QLGPU_H_
#define QLGPU_H_

#ifdef __cplusplus
extern "C" {
#endif

#define QLGPU_OK 0
#define QLGPU_ERR_ARG 1         /* invalid parameter or size */
#define QLGPU_ERR_UNSUPPORTED 2 /* valid for the reference but not built here */
#define QLGPU_ERR_CUDA 3        /* CUDA runtime error (message via qlgpu_last_error) */
#define QLGPU_ERR_STATUS 4      /* device status word set: non-finite / unstable solution */
#define QLGPU_ERR_NODEVICE 5    /* no CUDA device / extension unusable */

#define QLGPU_MODEL_MHD_BQLIN 0    /* QL_DNS/Models/MHD_BQlin.cpp */
#define QLGPU_MODEL_MHD_FULLQLIN 1 /* QL_DNS/Models/MHD_FullQlin.cpp */
#define QLGPU_INTEG_RK3CN_ELIN 0   /* QL_DNS/Integrators/RK3CN_Elin.cpp (what main.cpp:95 uses) */
#define QLGPU_INTEG_RK3CN 1        /* QL_DNS/Integrators/RK3CN.cpp */

/* Parameters: the Inputs fields the step reads
 * (QL_DNS/Auxiliary/Input_parameters.cpp:68-138). */
typedef struct qlgpu_params {
    int model;           /* QLGPU_MODEL_* (equations_to_use_) */
    int integrator;      /* QLGPU_INTEG_* */
    int nx, ny, NZ;      /* nx_, ny_, nz_ (NZ: power of two, 16..256) */
    double L[3];         /* lx_, ly_, lz_ */
    double q, omega;     /* q_, omega_ (MHD_BQlin uses 2q/3, MHD_BQlin.cpp:19) */
    double nu, eta, B0z; /* nu_, eta_, B0z_ */
    int viscosity_order; /* viscosity_order_ (MHD_FullQlin) */
    double dt;           /* dt_ (> 0; variable CFL dt is not supported) */
    int remap;           /* Remap? */
    int quasilinear;     /* QuasiLinear? */
} qlgpu_params;

typedef struct qlgpu_handle qlgpu_t;

/* Model + Integrator construction: replaces `new MHD_BQlin(SP, mpi, fft)` /
 * `new MHD_FullQlin(...)` (QL_DNS/main.cpp:58-61) and `new RK3CN_Elin(t, SP,
 * model)` (main.cpp:95).  device < 0 picks the current device.  The state
 * starts at zero with t = 0 and kx0 from the wavenumber tables. */
int qlgpu_create(const qlgpu_params* p, int device, qlgpu_t** out);
int qlgpu_destroy(qlgpu_t* h);

/* Model::Dimxy(), num_Lin(), NZ() (dealiased), num_MFs() (Model.h:53-58). */
int qlgpu_dims(const qlgpu_t* h, int* nxy, int* nlin, int* nz, int* nmf);

/* solution contents <-> host buffers (solution::pLin / pMF, Kdata::kx).
 * set_state also resets the integrator as its constructor does
 * (RK3CN.cpp:57: linear operators taken at t) and the diagnostic clock.
 * kx0 may be NULL (set: wavenumber tables; get: not returned). */
int qlgpu_set_state(qlgpu_t* h, double t, const double* lin, const double* mf, const double* kx0);
int qlgpu_get_state(qlgpu_t* h, double* t, double* lin, double* mf, double* kx0);

/* Same, with device pointers (already resident in this device's memory). */
int qlgpu_set_state_device(qlgpu_t* h, double t, const void* lin, const void* mf, const void* kx0);
int qlgpu_get_state_device(qlgpu_t* h, double* t, void* lin, void* mf, void* kx0);

/* The main-loop body of QL_DNS/main.cpp:108-133 repeated nsteps times:
 * Integrator::Step, t += dt, ShearingBox_Remap(q t) if remap, and
 * Calc_Energy_AM_Diss whenever the time-variable accumulator reaches
 * diag_every*dt (main.cpp:127-130; diag_every <= 0: never).  Each diagnostic
 * record is 15 doubles: t, energy[MU, MB, u, b], AM[MU, MB, u, b],
 * diss[MU, MB, u, b], etaK_times_kmax[2] (MHD_BQlin.cpp:449-477).  Records go
 * to diag_out (max_diag of them; extra records set QLGPU_ERR_STATUS); *ndiag
 * receives the count.  diag_out may be NULL when diag_every <= 0. */
int qlgpu_step(qlgpu_t* h, int nsteps, int diag_every, double* diag_out, int max_diag, int* ndiag);

/* One step (as qlgpu_step with diag_every = 0) with a CUDA event pair around
 * each of its three stage launches on the handle's stream; stage_ms[3]
 * receives the device time of each stage kernel.  Profiling aid standing in
 * for the reference's clock() accumulators (QL_DNS/Auxiliary/TimeVariables.h:51-54). */
int qlgpu_step_timed(qlgpu_t* h, float* stage_ms);

/* Calc_Energy_AM_Diss at the current time without stepping (15 doubles as
 * above): the initial record of main.cpp:98-103. */
int qlgpu_diagnostics(qlgpu_t* h, double* out15);

/* Model::rhs(t, dt_lin, SolIn, SolOut, linOp) (Model.h:46-47) on host
 * buffers: rhs of the fluctuations and mean fields and the linear operator
 * at t + dt_lin.  Uses the handle's kx0; does not touch its state.
 * linop (nxy*4*nz doubles) may be NULL. */
int qlgpu_rhs(qlgpu_t* h, double t, double dt_lin, const double* lin_in, const double* mf_in, double* lin_rhs,
              double* mf_rhs, double* linop);

/* Model::rhs on caller-owned DEVICE buffers that allocates no device memory.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc while the step runs (a pre-sized device memory pool or arena, a
 * host framework that owns every device buffer, latency-critical loops where
 * an allocation or the synchronisation of cudaFree is not acceptable).
 * Inputs lin_in[nxy][4][nz], mf_in[nmf][nz] and kx0[nxy] (may be NULL: the
 * unsheared wavenumber table), outputs lin_rhs, mf_rhs and linop (nxy*4*nz
 * doubles, may be NULL); all pointers are device pointers on the current
 * device; the work is queued on `stream` (a cudaStream_t, NULL = legacy
 * default stream) and the call returns without synchronising.
 * Scratch: one fixed 4 MiB device array in the library, held by every GPU that
 * loads the library until the process exits.  Limits: at most 8192 (kx,ky)
 * modes and ny <= 256 (larger cases return QLGPU_ERR_ARG; use qlgpu_rhs).
 * The first call on each device looks up the scratch address
 * (cudaGetSymbolAddress) and the device's SM count and shared-memory limit;
 * make that first call before any stream capture.  These are kept for the
 * life of the process: they do not survive cudaDeviceReset (call no
 * qlgpu_rhs_noalloc after a reset).
 * All calls share the scratch: calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller.  Errors are
 * reported through qlgpu_last_error(NULL, ...). */
int qlgpu_rhs_noalloc(const qlgpu_params* p, double t, double dt_lin, const void* lin_in, const void* mf_in,
                      const void* kx0, void* lin_rhs, void* mf_rhs, void* linop, void* stream);

/* Device status word (solution::Check_Solution, QL_DNS/solution.cpp:169-203):
 * bit 1 non-finite mean field, bit 2 |mean field| > 1e20, bit 4 diagnostic
 * records dropped.  Reading does not clear it; set_state clears it. */
int qlgpu_status(qlgpu_t* h, int* status);

/* Profiling aid: with QLGPU_TRACE=1 in the environment at qlgpu_create, each
 * stage kernel records %globaltimer stamps (ns) of its phases; out96 receives
 * 3 stages x 32 slots of the most recent step (slot meanings are listed in
 * ql_dns_b200/csrc/qlgpu_kernel.cuh).  Returns QLGPU_ERR_UNSUPPORTED when off. */
int qlgpu_trace(qlgpu_t* h, unsigned long long* out96);

/* Launch geometry of the stage kernel: info8 = {grid, block, dynamic shared
 * bytes, CTAs per SM, TMEM columns per CTA, threads per transform, modes, warps
 * per CTA}. */
int qlgpu_launch_info(const qlgpu_t* h, int* info8);

/* Compiled attributes of the stage kernel: attrs8 = {registers per thread,
 * static shared bytes, local bytes per thread, max threads per block,
 * CTAs per SM without / with the dynamic shared memory, max dynamic shared
 * bytes, preferred carveout}. */
int qlgpu_kernel_attrs(const qlgpu_t* h, int* attrs8);

/* Current simulation time and the CUDA stream (cudaStream_t) of the handle. */
int qlgpu_time(qlgpu_t* h, double* t);
int qlgpu_stream(qlgpu_t* h, void** stream);

/* Message of the last error on this handle (or of the last failed create
 * when h is NULL).  Returns the message length. */
int qlgpu_last_error(const qlgpu_t* h, char* buf, int buflen);

/* 1 in the debug build (libqlgpu_debug.so, compiled with -DQLGPU_DEBUG: device
 * index checks and canary guard zones after every device buffer, checked after
 * each call that launches kernels), else 0. */
int qlgpu_debug_build(void);

/* Debug build: overwrites the first byte of guard zone `zone` of the handle's
 * buffers from the host, so that the next call that launches kernels returns
 * QLGPU_ERR_STATUS with QLGPU_STATUS_CANARY (the test of the check itself).
 * QLGPU_ERR_UNSUPPORTED in a release build; QLGPU_ERR_ARG for a bad zone. */
int qlgpu_debug_guard_poke(qlgpu_t* h, int zone);

/* Library version string. */
const char* qlgpu_version(void);

/* Driving noise after every step (Model::DrivingNoise, QL_DNS/Models/
 * MHD_BQlin.cpp:558-618 and MHD_FullQlin.cpp:786-1045, called by
 * main.cpp:112-113 when f_noise != 0): modes with k_low < |k| < k_high get
 * complex normal increments of standard deviation f_noise/sqrt(2) per part,
 * scaled as the reference.  MHD_BQlin drives ky != 0 modes only; MHD_FullQlin
 * also drives ky = 0, kz != 0 in conjugate pairs, so that the field stays real
 * (kx < 0 draws, its kx > 0 partner adds the conjugate at -kz).  The
 * reference's clock-seeded mt19937 (MHD_BQlin.cpp:22) is replaced by one
 * Philox4x32-10 counter per (step since set_state, mode, kz, field) under
 * `seed`.  f_noise = 0 turns it off. */
int qlgpu_set_noise(qlgpu_t* h, double f_noise, double k_low, double k_high, unsigned long long seed);

/* MHD_FullQlin's drive_only_velocityQ / drive_only_magneticQ inputs
 * (MHD_FullQlin.cpp:21-22): nonzero drive_only_velocity leaves b and eta
 * undriven, nonzero drive_only_magnetic leaves u and zeta undriven.  Both 0 by
 * default; MHD_BQlin has no such switches (QLGPU_ERR_UNSUPPORTED when set). */
int qlgpu_set_noise_fields(qlgpu_t* h, int drive_only_velocity, int drive_only_magnetic);

/* Variable time step (RK3CN_Elin.cpp:76-80; RK3CN.cpp alike): cfl > 0 makes
 * every step dt = cfl / Calculate_CFL (MHD_BQlin.cpp:540-552,
 * MHD_FullQlin.cpp:769-780), capped at dt_max (the reference's -dt input).
 * With noise or cfl set, qlgpu_step writes a record after every diag_every-th
 * step.  cfl = 0 restores the fixed dt of the parameters. */
int qlgpu_set_cfl(qlgpu_t* h, double cfl, double dt_max);

/* Integrator::mean_time_step(): mean dt of the steps since set_state. */
int qlgpu_mean_time_step(qlgpu_t* h, double* dt_mean);

/* Measured FP64 FMA throughput of a device (TFLOP/s, best of 5 timed launches
 * of independent FMA chains): the denominator of the FP64 roofline of the 3-D
 * DNS transforms (include/qlgpu_dns.h).  device < 0: the current device. */
int qlgpu_fp64_peak(int device, double* tflops);

/* Discrete adjoint (no counterpart in the reference).  For MHD_BQlin with
 * RK3CN_Elin: J = (1/N) sum_{n=1..N} AM_b(t0 + n dt), the fluctuation Maxwell
 * stress of the diagnostic records (MHD_BQlin.cpp:392,424, column 8 of a
 * record) averaged over N = nsteps steps.  Runs the N steps from (t0, lin0,
 * mf0, kx0) (kx0 may be NULL) keeping a checkpoint every checkpoint_every
 * steps, then the adjoint of every stage in reverse, recomputing the stages of
 * one checkpoint window at a time.  Returns J, grad_lin = dJ/d lin0 (complex
 * [nxy][4][nz]: dJ = Re sum conj(grad_lin) d lin0, i.e. the derivatives with
 * respect to the real and imaginary parts) and, when grad_mf is not NULL,
 * dJ/d mf0 likewise.  The handle is left at the end of the forward run. */
int qlgpu_adjoint_maxwell(qlgpu_t* h, double t0, const double* lin0, const double* mf0, const double* kx0,
                          int nsteps, int checkpoint_every, double* J, double* grad_lin, double* grad_mf);

/* The same for nseeds initial states at once, one handle per seed (handles of
 * equal dimensions).  The forward sweep and every window recompute of all
 * seeds run in the persistent batch kernel (one launch per window); the
 * reverse sweep launches each of its kernels once for all seeds when the
 * seeds share every parameter, else per seed on the seed's stream.
 * lin0 [nseeds][nxy][4][nz], mf0 [nseeds][nmf][nz], kx0 [nseeds][nxy] or
 * NULL; J [nseeds], grad_lin / grad_mf like lin0 / mf0.  Each seed's results
 * equal those of qlgpu_adjoint_maxwell on its handle to round-off (the batch
 * kernel sums in another order); with the environment variable
 * QLGPU_ADJ_BATCH=streams every seed runs the single-case path, bit for bit. */
int qlgpu_adjoint_maxwell_batch(qlgpu_t* const* handles, int nseeds, double t0, const double* lin0,
                                const double* mf0, const double* kx0, int nsteps, int checkpoint_every, double* J,
                                double* grad_lin, double* grad_mf);

/* ------------------------------------------------------------------------
 * Batched ensemble.  No counterpart in the reference, which runs one case per
 * MPI job (QL_DNS/main.cpp:23-180): here many independent cases, each with
 * its own qlgpu_params (mode grid, NZ, nu, eta, q, dt, ...), step together in
 * ONE persistent cooperative kernel launch per call.  All cases share the
 * model and the integrator.  Per case the step is the same fused RK3 step as
 * qlgpu_step (the same stage code); only the order of the floating-point sums
 * over CTAs depends on how many CTAs a case gets.  Every wait inside the
 * kernel is bounded (a status bit, never a hang).
 * ------------------------------------------------------------------------ */
typedef struct qlgpu_batch qlgpu_batch_t;

#define QLGPU_STATUS_BATCH_TIMEOUT 8 /* a CTA gave up waiting for the others of its case */
/* Debug build only (libqlgpu_debug.so, -DQLGPU_DEBUG): a device index check
 * failed (the access was redirected in bounds), or a guard zone after a device
 * buffer was overwritten.  Either makes the call return QLGPU_ERR_STATUS. */
#define QLGPU_STATUS_BOUNDS 16
#define QLGPU_STATUS_CANARY 32

/* Creates the batch (device memory, wavenumber tables, an initial CTA
 * mapping from the cost model).  All cases zero; t = 0. */
int qlgpu_batch_create(const qlgpu_params* cases, int ncases, int device, qlgpu_batch_t** out);
int qlgpu_batch_destroy(qlgpu_batch_t* b);
int qlgpu_batch_dims(const qlgpu_batch_t* b, int c, int* nxy, int* nz, int* nmf);

/* State of case c, as qlgpu_set_state / qlgpu_get_state (host buffers; kx0 may be NULL). */
int qlgpu_batch_set_state(qlgpu_batch_t* b, int c, double t, const double* lin, const double* mf, const double* kx0);
int qlgpu_batch_get_state(qlgpu_batch_t* b, int c, double* t, double* lin, double* mf, double* kx0);

/* Every case at once, one synchronisation: lin[c], mf[c] (and kx0[c], which
 * may be NULL, as may kx0 itself) are case c's host buffers, pinned for
 * asynchronous copies; get: t[ncases] (may be NULL) and any non-NULL buffer. */
int qlgpu_batch_set_states(qlgpu_batch_t* b, double t, const double* const* lin, const double* const* mf,
                           const double* const* kx0);
int qlgpu_batch_get_states(qlgpu_batch_t* b, double* t, double* const* lin, double* const* mf, double* const* kx0);

/* Driving noise of case c after every step, as qlgpu_set_noise and
 * qlgpu_set_noise_fields of a single handle with the case's fixed dt: the
 * Philox counter's step word counts the steps since the case's state was set.
 * f_noise = 0 turns it off (the default). */
int qlgpu_batch_set_noise(qlgpu_batch_t* b, int c, double f_noise, double k_low, double k_high,
                          unsigned long long seed, int drive_only_velocity, int drive_only_magnetic);

/* Debug build: as qlgpu_debug_guard_poke for the batch's buffers. */
int qlgpu_batch_debug_guard_poke(qlgpu_batch_t* b, int zone);

/* Initial diagnostic record of case c (15 doubles, as qlgpu_diagnostics). */
int qlgpu_batch_diagnostics(qlgpu_batch_t* b, int c, double* out15);

/* nsteps steps of every case in one launch (replayed from a CUDA graph).
 * diag_every > 0: case c writes a record every diag_every steps to
 * diag_out + c*max_diag*15 and its count to ndiag[c]. */
int qlgpu_batch_step(qlgpu_batch_t* b, int nsteps, int diag_every, double* diag_out, int max_diag, int* ndiag);

/* Asynchronous stepping, for a caller that reads every step's records while the
 * next steps run: qlgpu_batch_step_async queues nsteps steps of every case (one
 * launch) and the copy of their records and statuses into pinned memory, and
 * returns without waiting.  At most two calls are outstanding.
 * qlgpu_batch_step_collect waits for the oldest and returns its records and
 * status as qlgpu_batch_step does (max_diag as given to its step_async).  The
 * other batch calls that step, tune or move state refuse while a step is
 * outstanding (QLGPU_ERR_ARG). */
int qlgpu_batch_step_async(qlgpu_batch_t* b, int nsteps, int diag_every, int max_diag);
int qlgpu_batch_step_collect(qlgpu_batch_t* b, double* diag_out, int max_diag, int* ndiag);

/* As qlgpu_batch_step without diagnostics; *ms = device time of the launch
 * (CUDA events on the batch stream). */
int qlgpu_batch_step_timed(qlgpu_batch_t* b, int nsteps, float* ms);

/* Autotuner: times probe_steps-step launches of candidate mappings (CTA
 * width, CTAs per case, cases per CTA) on a copy of the state, fits the cost
 * model to the per-case times and keeps the fastest mapping.  Queue engine: a
 * coordinate search, two sweeps, over the passes per chunk of each NZ class,
 * each candidate timed as the best of three launches of max(probe_steps, 6)
 * steps.  The state is unchanged.  *best_ms (may be NULL) = time of the kept
 * mapping's probe. */
int qlgpu_batch_tune(qlgpu_batch_t* b, int probe_steps, double* best_ms);

/* The planner's cost model (after qlgpu_batch_tune: fitted to the measured
 * per-case stage times): out7 = {alpha (us per stage per launch), beta (us per
 * work item per stage), r[NZ = 16, 32, 64, 128, 256] (us per pipeline pass)}. */
int qlgpu_batch_cost_model(const qlgpu_batch_t* b, double* out7);

/* Current mapping: info4 = {warps per CTA, CTAs launched, CTAs per SM,
 * dynamic shared bytes}; ncta[c] = CTAs that step case c (may be NULL);
 * queue engine: ncta[c] = chunks of case c per stage. */
int qlgpu_batch_mapping(const qlgpu_batch_t* b, int* info4, int* ncta);

/* Fixed mapping: ncta[c] CTAs for case c at `warps` warps per CTA (1 up to
 * the widest CTA that fits the batch's NZ classes); cases are packed onto the
 * launch's CTAs by the cost model. */
int qlgpu_batch_set_mapping(qlgpu_batch_t* b, int warps, const int* ncta);

/* Per-case device status words (bits as qlgpu_status) and the launch status
 * of the most recent step (QLGPU_STATUS_BATCH_TIMEOUT). */
int qlgpu_batch_status(qlgpu_batch_t* b, int* case_status, int* launch_status);

/* Bound on one in-kernel wait (default 2 s). */
int qlgpu_batch_set_wait(qlgpu_batch_t* b, double seconds);

/* Failure-detection test aid: removes the last work item of case c (a case
 * with two or more CTAs) from the current mapping (queue engine: one chunk
 * of case c, which needs two or more chunks, from every stage), so that the
 * case's other CTAs wait for a stage that never completes.  The next step call must return
 * QLGPU_ERR_STATUS with QLGPU_STATUS_BATCH_TIMEOUT after the wait bound; the
 * batch stays usable after qlgpu_batch_set_mapping / qlgpu_batch_tune and
 * qlgpu_batch_set_state. */
int qlgpu_batch_debug_drop_item(qlgpu_batch_t* b, int c);

/* Engines.  QLGPU_BATCH_ENGINE_ITEMS: the work-item engine above (every model,
 * integrator and NZ; CTAs own fixed work items and wait for their cases at
 * each stage).  QLGPU_BATCH_ENGINE_QUEUE: MHD_BQlin batches with every NZ <=
 * 128 -- CTAs take chunks of consecutive modes of one case and one stage from
 * a global ticket counter; the CTA that completes a case's stage runs its
 * mean-field stage, so no CTA waits at another case's stage boundary.  Chunk
 * partial sums go to fixed slots summed in slot order: results do not depend
 * on which CTA ran which chunk.  QLGPU_BATCH_ENGINE_AUTO picks the queue
 * engine where it applies (the default at creation).  The per-case
 * arithmetic of the two engines agrees to round-off (1e-12 relative), not
 * bit for bit.  qlgpu_batch_set_mapping selects the work-item engine. */
#define QLGPU_BATCH_ENGINE_AUTO 0
#define QLGPU_BATCH_ENGINE_ITEMS 1
#define QLGPU_BATCH_ENGINE_QUEUE 2
int qlgpu_batch_set_engine(qlgpu_batch_t* b, int engine);
int qlgpu_batch_engine(const qlgpu_batch_t* b, int* engine);

/* Queue engine: CTA passes per chunk for the NZ classes 16, 32, 64, 128
 * (passes4[i] >= 1; a pass steps 12 warps x 32/(NZ/4) modes).  Selects the
 * queue engine.  qlgpu_batch_tune searches these when the queue engine is
 * active. */
int qlgpu_batch_set_chunks(qlgpu_batch_t* b, const int* passes4);
/* The current passes per chunk of the four NZ classes: after qlgpu_batch_tune the
 * tuned ones; before, 4 per class, or fewer where 4 would leave SMs without a chunk
 * (a small batch). */
int qlgpu_batch_chunks(const qlgpu_batch_t* b, int* passes4);

/* Profiling aid of the queue engine (QLGPU_TRACE=1 in the environment at
 * qlgpu_batch_create): per CTA of the last launch, averaged over CTAs, out4 =
 * {us waiting for tickets and stages, us in chunks, us of that in mean-field
 * stages, chunks}.  QLGPU_ERR_UNSUPPORTED when off. */
int qlgpu_batch_queue_trace(qlgpu_batch_t* b, double* out4);

int qlgpu_batch_stream(qlgpu_batch_t* b, void** stream);
int qlgpu_batch_last_error(const qlgpu_batch_t* b, char* buf, int buflen);

#ifdef __cplusplus
}
#endif
#endif /* QLGPU_H_ */
