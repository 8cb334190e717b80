/*
 * qlgpu_dns.h -- C ABI of the B200 (sm_100a) full 3-D shearing-box MHD DNS.
 *
 * The reference has no 3-D model: its Model interface (QL_DNS/Models/
 * Model.h:24-112) is the plug-in point a DNS model would fill, and its only
 * transforms are 1-D z plans (QL_DNS/Auxiliary/fftwPlans.cpp:48-51).  This
 * handle is the full nonlinear extension of MHD_FullQlin
 * (QL_DNS/Models/MHD_FullQlin.cpp:171-456): same box, shear, rotation, B0z,
 * dissipation (order viscosity_order), integrators (RK3CN_Elin, RK3CN) and
 * remap rule, with every product of u and b taken on the Mx x My x NZ grid
 * (2/3 dealiased in x, y and z) instead of the mean x fluctuation products only.
 *
 * Data layout (host and device alike, interleaved re/im doubles):
 *   lin[nxy][6][nz]  (u_x, u_y, u_z, b_x, b_y, b_z) per (kx, ky) mode column
 *                    in the Kdata order of the QL models
 *                    (QL_DNS/Auxiliary/Kdata.cpp:30-46) with nx = 2 floor(Mx/3)+2
 *                    and ny = 2 floor(My/3)+2 modes; kz in dealiased order
 *                    0..(nz-1)/2, -(nz-1)/2..-1, nz = 1 + 2 floor(NZ/3).
 *                    Column 0 (kx = ky = 0) holds the mean fields
 *                    (Ux, Uy, 0, Bx, By, 0).  Values are physical Fourier
 *                    amplitudes times Mx*My*NZ.
 *   kx0[nxy]         unsheared kx of every column, shifted by remaps.
 * Every function returns a status code of include/qlgpu.h (QLGPU_OK = 0).
 * One host thread per handle at a time; each handle owns its device memory
 * and one CUDA stream.
 */
#ifndef QLGPU_DNS_H_
#define QLGPU_DNS_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qlgpu_dns_params {
    int integrator;      /* QLGPU_INTEG_RK3CN_ELIN (0) or QLGPU_INTEG_RK3CN (1) */
    int Mx, My, NZ;      /* grid: Mx, NZ in {16, 32, 64}, My in {16, 32, 64, 128, 256} */
    double L[3];         /* lx_, ly_, lz_ */
    double q, omega;     /* shear rate and rotation (MHD_FullQlin.cpp:15) */
    double nu, eta, B0z; /* dissipation coefficients, uniform vertical field */
    int viscosity_order; /* dissipation -nu |k|^(2*(viscosity_order/2)) (MHD_FullQlin.cpp:372) */
    double dt;           /* fixed time step */
    int remap;           /* shearing-box remap of whole columns (MHD_FullQlin.cpp:464-481) */
    int dealias_xy;      /* zero columns with |kx(t)| > Mx/3 (2 pi/Lx) at every stage */
} qlgpu_dns_params;

typedef struct qlgpu_dns qlgpu_dns_t;

/* Model + Integrator construction for the DNS (the role of main.cpp:58-74,95
 * for the QL models).  device < 0 picks the current device.  The state starts
 * at zero with t = 0 and kx0 from the wavenumber tables. */
int qlgpu_dns_create(const qlgpu_dns_params* p, int device, qlgpu_dns_t** out);
int qlgpu_dns_destroy(qlgpu_dns_t* h);

/* Mode columns nxy, stored kz length nz, and the QL mode counts nx, ny. */
int qlgpu_dns_dims(const qlgpu_dns_t* h, int* nxy, int* nz, int* nx, int* ny);

/* State <-> host buffers.  set_state resets the integrator (CN operator at t)
 * and the diagnostic count; kx0 may be NULL (set: wavenumber tables; get: not
 * returned). */
int qlgpu_dns_set_state(qlgpu_dns_t* h, double t, const double* lin, const double* kx0);
int qlgpu_dns_get_state(qlgpu_dns_t* h, double* t, double* lin, double* kx0);

/* nsteps RK3 steps (Integrator::Step then the remap, main.cpp:111-123).  With
 * diag_every > 0 a 15-double record (t, energy[MU,MB,u,b]/2, AM[MU,MB,u,b],
 * diss[MU,MB,u,b], etaK[u,b]: the layout of MHD_FullQlin::Calc_Energy_AM_Diss,
 * MHD_FullQlin.cpp:487-717) is written after every diag_every-th step into
 * diag_out (room for max_diag records); *ndiag gets the count. */
int qlgpu_dns_step(qlgpu_dns_t* h, int nsteps, int diag_every, double* diag_out, int max_diag, int* ndiag);

/* The diagnostic record of the current state. */
int qlgpu_dns_diagnostics(qlgpu_dns_t* h, double* out15);

/* One right-hand-side evaluation at time t of the current state (no update):
 * F[nxy][6][nz] as the stage kernels compute it. */
int qlgpu_dns_rhs(qlgpu_dns_t* h, double t, double* F);

/* Device status bits (1 = non-finite state) and the last error message. */
int qlgpu_dns_status(qlgpu_dns_t* h, int* status);
int qlgpu_dns_last_error(const qlgpu_dns_t* h, char* buf, int buflen);

/* One step timed with CUDA events on the handle's stream (ms); the stream. */
int qlgpu_dns_step_timed(qlgpu_dns_t* h, int nsteps, float* ms);
void* qlgpu_dns_stream(qlgpu_dns_t* h);

#ifdef __cplusplus
}
#endif
#endif /* QLGPU_DNS_H_ */
