// qlgpu.hpp -- header-only C++ mirror of the reference's Model / Integrator /
// solution objects (QL_DNS/Models/Model.h:24-112, QL_DNS/Integrators/Integrator.h:20-28,
// QL_DNS/solution.h:23-49) on top of the C ABI in qlgpu.h.
//
// A driver written like QL_DNS/main.cpp keeps its shape:
//     qlgpu::Inputs SP = ...;                      // Inputs fields the step reads
//     qlgpu::MHD_BQlin model(SP);                   // new MHD_BQlin(SP, mpi, fft)
//     qlgpu::solution sol(&model);                  // new solution(model)
//     ... fill sol.pLin(i, V), sol.pMF(i) ...
//     qlgpu::RK3CN_Elin integ(t, SP, &model);       // new RK3CN_Elin(t, SP, model)
//     while (t < SP.t_final) { dt = integ.Step(t, &sol); t += dt; ... }
// The state lives on the GPU between Step calls; solution::pLin / pMF pull it
// back to the host lazily (sync()) so host reads always see the current step.
// Errors throw qlgpu::Error (the reference calls ABORT, General_Definitions.h:68-72).
#ifndef QLGPU_HPP_
#define QLGPU_HPP_

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "qlgpu.h"

namespace qlgpu {

typedef std::complex<double> dcmplx;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const qlgpu_t* h) {
    if (rc != QLGPU_OK) {
        char buf[512];
        qlgpu_last_error(h, buf, sizeof(buf));
        throw Error(rc, buf);
    }
}

// The Inputs fields of QL_DNS/Auxiliary/Input_parameters.cpp:68-138 that the step reads.
struct Inputs {
    std::string equations_to_use = "MHD_BQlin";
    int NXY[2] = {16, 16};
    int NZ = 16;
    double L[3] = {2 * 3.14159265358979323846, 2 * 3.14159265358979323846, 2 * 3.14159265358979323846};
    double dt = 0.33333333333333;
    double t_final = 10.0;
    double nu = 0.01, eta = 0.01;
    int viscosity_order = 2;
    double q = 1.5, omega = 1.0, B0z = 0.0;
    bool remapQ = true, QuasiLinearQ = true;
    // dt < 0: variable dt = CFL / Calculate_CFL capped at -dt (RK3CN_Elin.cpp:22-27)
    double CFL = 1.0;
    // driving noise (Input_parameters.cpp:107-109); the generator's seed replaces the clock
    double f_noise = 0.0, noise_range_low = 0.0, noise_range_high = 1e16;
    unsigned long long noise_seed = 0;
    // MHD_FullQlin only (Input_parameters.cpp:110-111, MHD_FullQlin.cpp:21-22)
    bool drive_only_velocityQ = false, drive_only_magneticQ = false;
};

class Model;

// solution (QL_DNS/solution.h:23-49): host copy of the state, kx0 of the modes.
class solution {
public:
    explicit solution(Model* m);
    dcmplx* pLin(int i, int V);  // nz contiguous values, kz order 0..(nz-1)/2, -(nz-1)/2..-1
    dcmplx* pMF(int i);
    std::vector<dcmplx> lin, mf;
    std::vector<double> kx0;
    Model* model;
    bool host_stale = false;  // the GPU holds a newer state
    void sync();              // pull the GPU state into lin / mf / kx0
};

// Model (QL_DNS/Models/Model.h:24-112)
class Model {
public:
    explicit Model(const Inputs& sp, int model_id) : sp_(sp) {
        p_.model = model_id;
        p_.integrator = QLGPU_INTEG_RK3CN_ELIN;
        p_.nx = sp.NXY[0];
        p_.ny = sp.NXY[1];
        p_.NZ = sp.NZ;
        for (int i = 0; i < 3; ++i) p_.L[i] = sp.L[i];
        p_.q = sp.q;
        p_.omega = sp.omega;
        p_.nu = sp.nu;
        p_.eta = sp.eta;
        p_.B0z = sp.B0z;
        p_.viscosity_order = sp.viscosity_order;
        p_.dt = sp.dt;
        p_.remap = sp.remapQ ? 1 : 0;
        p_.quasilinear = sp.QuasiLinearQ ? 1 : 0;
        nz_ = 1 + 2 * int(sp.NZ / 3.0);
        nxy_ = (sp.NXY[0] - 1) * (sp.NXY[1] / 2);
        nmf_ = model_id == QLGPU_MODEL_MHD_BQLIN ? 2 : 4;
    }
    virtual ~Model() {
        if (h_) qlgpu_destroy(h_);
    }
    int Dimxy() const { return nxy_; }
    int Dimxy_full() const { return nxy_; }
    int NZ() const { return nz_; }
    int NZfull() const { return p_.NZ; }
    int num_MFs() const { return nmf_; }
    int num_Lin() const { return 4; }
    double L(int i) const { return p_.L[i]; }

    // Model::rhs (Model.h:46-47): rhs of SolIn into SolOut and the linear
    // operator at t + dt_lin into linOp (nxy*4*nz doubles, may be null).
    void rhs(double t, double dt_lin, solution* in, solution* out, double* linOp) {
        handle();
        in->sync();
        check(qlgpu_rhs(h_, t, dt_lin, reinterpret_cast<const double*>(in->lin.data()),
                        reinterpret_cast<const double*>(in->mf.data()), reinterpret_cast<double*>(out->lin.data()),
                        reinterpret_cast<double*>(out->mf.data()), linOp),
              h_);
    }
    // Calc_Energy_AM_Diss (Model.h:95): 15 doubles t, energy[4], AM[4], diss[4], etaK[2]
    std::vector<double> Calc_Energy_AM_Diss(double t, solution* sol) {
        handle();
        sol->sync();
        check(qlgpu_set_state(h_, t, reinterpret_cast<const double*>(sol->lin.data()),
                              reinterpret_cast<const double*>(sol->mf.data()), sol->kx0.data()),
              h_);
        std::vector<double> out(15);
        check(qlgpu_diagnostics(h_, out.data()), h_);
        return out;
    }
    // Model::DrivingNoise (Model.h:85): the integrator's handle adds the noise after every
    // step when Inputs::f_noise != 0 (qlgpu_set_noise), so the call of main.cpp:112-113
    // has nothing left to do.
    void DrivingNoise(double, double, solution*) {}
    qlgpu_params params() const { return p_; }

protected:
    qlgpu_t* handle() {
        if (!h_) check(qlgpu_create(&p_, -1, &h_), nullptr);
        return h_;
    }
    Inputs sp_;
    qlgpu_params p_;
    int nz_, nxy_, nmf_;
    qlgpu_t* h_ = nullptr;
};

class MHD_BQlin : public Model {
public:
    explicit MHD_BQlin(const Inputs& sp) : Model(sp, QLGPU_MODEL_MHD_BQLIN) {}
};
class MHD_FullQlin : public Model {
public:
    explicit MHD_FullQlin(const Inputs& sp) : Model(sp, QLGPU_MODEL_MHD_FULLQLIN) {}
};

inline solution::solution(Model* m) : model(m) {
    lin.assign((size_t)m->Dimxy() * 4 * m->NZ(), dcmplx(0, 0));
    mf.assign((size_t)m->num_MFs() * m->NZ(), dcmplx(0, 0));
    // Kdata::kx (Kdata.cpp:30-46): i*2pi/Lx for i < Nx/2, then -(Nx/2-1)..-1
    const int nx = m->params().nx / 2, ny = m->params().ny / 2;
    const double kxL = 2 * 3.14159265358979323846 / m->L(0);
    kx0.assign(m->Dimxy(), 0.0);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) kx0[j + ny * i] = i * kxL;
    for (int i = nx + 1; i < 2 * nx; ++i)
        for (int j = 0; j < ny; ++j) kx0[j + ny * (i - 1)] = (-2 * nx + i) * kxL;
}

// Integrator (QL_DNS/Integrators/Integrator.h:20-28).  Step runs the fused
// GPU step of the main-loop body (main.cpp:111-123: step, t += dt, remap).
class Integrator {
public:
    Integrator(double t0, const Inputs& sp, Model* mod, int integ_id) : t0_(t0), model_(mod) {
        p_ = mod->params();
        p_.integrator = integ_id;
        p_.dt = sp.dt < 0 ? -sp.dt : sp.dt;
        check(qlgpu_create(&p_, -1, &h_), nullptr);
        variable_dt_ = sp.dt < 0;
        if (variable_dt_) check(qlgpu_set_cfl(h_, sp.CFL, -sp.dt), h_);
        if (sp.f_noise != 0.0) {
            check(qlgpu_set_noise(h_, sp.f_noise, sp.noise_range_low, sp.noise_range_high, sp.noise_seed), h_);
            if (sp.drive_only_velocityQ || sp.drive_only_magneticQ)
                check(qlgpu_set_noise_fields(h_, sp.drive_only_velocityQ, sp.drive_only_magneticQ), h_);
        }
    }
    virtual ~Integrator() {
        if (h_) qlgpu_destroy(h_);
    }
    double Step(double t, solution* sol) {
        if (bound_ != sol || sol->host_stale == false) {
            check(qlgpu_set_state(h_, t, reinterpret_cast<const double*>(sol->lin.data()),
                                  reinterpret_cast<const double*>(sol->mf.data()), sol->kx0.data()),
                  h_);
            bound_ = sol;
        }
        double t0 = 0, t1 = 0;
        if (variable_dt_) check(qlgpu_time(h_, &t0), h_);
        check(qlgpu_step(h_, 1, 0, nullptr, 0, nullptr), h_);
        sol->host_stale = true;
        sol->model = model_;
        last_handle_ = h_;
        ++steps_;
        if (!variable_dt_) return p_.dt;
        check(qlgpu_time(h_, &t1), h_);
        return t1 - t0;  // the step's dt (CFL)
    }
    // main-loop form: n steps with a diagnostic record every diag_every steps
    std::vector<double> Run(double t, solution* sol, int n, int diag_every) {
        check(qlgpu_set_state(h_, t, reinterpret_cast<const double*>(sol->lin.data()),
                              reinterpret_cast<const double*>(sol->mf.data()), sol->kx0.data()),
              h_);
        std::vector<double> d(15 * (size_t)(n + 1));
        d.resize(15);
        check(qlgpu_diagnostics(h_, d.data()), h_);
        int nd = 0;
        if (diag_every > 0) {
            d.resize(15 * (size_t)(n / diag_every + 2));
            check(qlgpu_step(h_, n, diag_every, d.data() + 15, n / diag_every + 1, &nd), h_);
        } else {
            check(qlgpu_step(h_, n, 0, nullptr, 0, nullptr), h_);
        }
        d.resize(15 * (size_t)(nd + 1));
        pull(sol);
        bound_ = nullptr;
        return d;
    }
    void pull(solution* sol) {
        double t;
        check(qlgpu_get_state(h_, &t, reinterpret_cast<double*>(sol->lin.data()),
                              reinterpret_cast<double*>(sol->mf.data()), sol->kx0.data()),
              h_);
        sol->host_stale = false;
    }
    double mean_time_step() const {
        double m = p_.dt;
        qlgpu_mean_time_step(h_, &m);
        return m;
    }
    qlgpu_t* handle() const { return h_; }
    static qlgpu_t* last_handle_;

protected:
    double t0_;
    Model* model_;
    qlgpu_params p_;
    qlgpu_t* h_ = nullptr;
    solution* bound_ = nullptr;
    long steps_ = 0;
    bool variable_dt_ = false;
};
inline qlgpu_t* Integrator::last_handle_ = nullptr;

inline void solution::sync() {
    if (!host_stale || !Integrator::last_handle_) return;
    double t;
    check(qlgpu_get_state(Integrator::last_handle_, &t, reinterpret_cast<double*>(lin.data()),
                          reinterpret_cast<double*>(mf.data()), kx0.data()),
          Integrator::last_handle_);
    host_stale = false;
}
inline dcmplx* solution::pLin(int i, int V) {
    sync();
    return &lin[((size_t)i * 4 + V) * model->NZ()];
}
inline dcmplx* solution::pMF(int i) {
    sync();
    return &mf[(size_t)i * model->NZ()];
}

class RK3CN_Elin : public Integrator {
public:
    RK3CN_Elin(double t0, const Inputs& sp, Model* mod) : Integrator(t0, sp, mod, QLGPU_INTEG_RK3CN_ELIN) {}
};
class RK3CN : public Integrator {
public:
    RK3CN(double t0, const Inputs& sp, Model* mod) : Integrator(t0, sp, mod, QLGPU_INTEG_RK3CN) {}
};

}  // namespace qlgpu

#endif  // QLGPU_HPP_
