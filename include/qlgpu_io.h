/*
 * qlgpu_io.h -- host-side output and restart files of the quasi-linear step,
 * in the reference's layouts.  No GPU is needed; these functions read and
 * write host buffers in the layout of qlgpu.h (lin[nxy][4][nz], mf[nmf][nz]
 * complex doubles, kx0[nxy]) and of the diagnostic records of qlgpu_step
 * (15 doubles: t, energy[4], AM[4], diss[4], etaK[2]).
 */
#ifndef QLGPU_IO_H_
#define QLGPU_IO_H_

#include "qlgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- TimeVariables (QL_DNS/Auxiliary/TimeVariables.cpp:25-228) -------------
 * The binary .dat files the reference's MATLAB readers consume, in `dir`
 * (a path prefix as SP.simulation_dir, normally ending in '/'):
 *   energy.dat, angular_momentum.dat, dissipation.dat  4 doubles per save
 *   reynolds_stress.dat                                num_reynolds doubles per save
 *   time_vec.dat                                       1 double per save
 *   mean_fields.dat                                    nmf x NZ doubles per mean-field save
 * append = 0 truncates the files (TimeVariables.cpp:62-68 without
 * start_from_saved_Q), 1 appends.  num_reynolds is the model's
 * num_reynolds_saves() (MHD_BQlin.h:41: 5; MHD_FullQlin: 4); the reference
 * leaves these values unset for MHD_BQlin and writes the stress-drive
 * projections for MHD_FullQlin (MHD_FullQlin.cpp:632-660), which the GPU step
 * does not keep: zeros are written. */
typedef struct qlgpu_timevars qlgpu_timevars_t;
int qlgpu_timevars_open(const char* dir, int nmf, int NZ, int num_reynolds, int append, qlgpu_timevars_t** out);
/* TimeVariables::Save_Data(t) for one diagnostic record (15 doubles). */
int qlgpu_timevars_save_data(qlgpu_timevars_t* tv, const double* rec15);
/* TimeVariables::Save_Mean_Fields: the real part of the inverse transform of
 * every mean field (padded nz -> NZ, times 1/NZ, fftwPlans.cpp:29-34). */
int qlgpu_timevars_save_mean_fields(qlgpu_timevars_t* tv, const double* mf, int nz);
int qlgpu_timevars_close(qlgpu_timevars_t* tv);

/* ---- FullSave_Load (QL_DNS/Auxiliary/FullSave_Load.cpp:176-329) -----------
 * The reference writes an HDF5 file; HDF5 is not available to this build, so
 * the same content goes into a raw binary container with the same groups and
 * dataset names, in save order:
 *   file   : "QLFSAVE1" (8 bytes), int32 nlin, nz, nmf, nxy
 *   group  : uint32 len, name "/t=<t with %.15g>", double t, uint32 ndatasets
 *   dataset: uint32 len, name, uint32 type (0 complex float32 pairs, 1 float32),
 *            uint64 count, count values
 * with, per group, datasets "Ind j: kx <kx index> ky <ky index>" (complex
 * float32 [4*nz], field after field, FullSave_Load.cpp:190-211), "Mean"
 * (complex float32 [nmf*nz], :216-224) and "kx" (float32 [nxy], the sheared
 * kx0 + q t ky, :229-239). */
/* SaveSolution(t, sol): appends a group (creates the file when missing). */
int qlgpu_fullsave_write(const char* path, const qlgpu_params* p, double t, const double* lin, const double* mf,
                         const double* kx0);
/* LoadSolution_forRestart: the group with the largest t; kx0 = kx - q t ky
 * (FullSave_Load.cpp:317-320).  Any output pointer may be NULL. */
int qlgpu_fullsave_read_latest(const char* path, const qlgpu_params* p, double* t, double* lin, double* mf,
                               double* kx0);
/* Number of groups and their times (times may be NULL; at most max_times written). */
int qlgpu_fullsave_times(const char* path, double* times, int max_times, int* ngroups);

/* Message of the last I/O error of this thread. */
int qlgpu_io_last_error(char* buf, int buflen);

#ifdef __cplusplus
}
#endif
#endif /* QLGPU_IO_H_ */
