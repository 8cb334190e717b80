// ql_main.cpp -- a QL_DNS/main.cpp-shaped driver on the B200 step.
//
//   ql_main <input.DSSinput> <state_in.bin> <nsteps> <state_out.bin> <diag_out.bin> [output_dir]
//
// Reads the reference's .DSSinput keys (QL_DNS/Auxiliary/Input_parameters.cpp:68-138,
// found by substring then '=' like Read_From_Input_File_, :178-209), an initial
// state (t, lin[nxy][4][nz], mf[nmf][nz], kx0[nxy] as raw doubles), runs the
// main-loop body nsteps times with a diagnostic record every tv_save_/dt steps
// (main.cpp:108-133) and writes the final state and the diagnostic records.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "qlgpu.hpp"
#include "qlgpu_io.h"

template <class T>
static T read_key(const std::string& file, const std::string& key, T dflt) {
    size_t pos = file.find(key);
    if (pos == std::string::npos) return dflt;
    pos = file.find_first_of('=', pos);
    std::istringstream ss(file.substr(pos + 1, 100));
    T out;
    ss >> out;
    return out;
}

int main(int argc, char** argv) {
    if (argc != 6 && argc != 7) {
        std::fprintf(stderr, "usage: %s input.DSSinput state_in.bin nsteps state_out.bin diag_out.bin [output_dir]\n",
                     argv[0]);
        return 2;
    }
    std::ifstream fin(argv[1]);
    std::string full((std::istreambuf_iterator<char>(fin)), std::istreambuf_iterator<char>());
    qlgpu::Inputs SP;
    const double PI = 3.14159265358979323846;
    SP.NXY[0] = read_key<int>(full, "nx_", 16);
    SP.NXY[1] = read_key<int>(full, "ny_", 16);
    SP.NZ = read_key<int>(full, "nz_", 16);
    SP.L[0] = read_key<double>(full, "lx_", 2 * PI);
    SP.L[1] = read_key<double>(full, "ly_", 2 * PI);
    SP.L[2] = read_key<double>(full, "lz_", 2 * PI);
    SP.dt = read_key<double>(full, "dt_", 0.33333333333333);
    SP.nu = read_key<double>(full, "nu_", 0.01);
    SP.eta = read_key<double>(full, "eta_", 0.01);
    SP.viscosity_order = read_key<int>(full, "viscosity_order_", 2);
    SP.q = read_key<double>(full, "q_", 1.5);
    SP.omega = read_key<double>(full, "omega_", 1.0);
    SP.B0z = read_key<double>(full, "B0z_", 0.0);
    SP.remapQ = read_key<int>(full, "Remap?", 1) != 0;
    SP.QuasiLinearQ = read_key<int>(full, "QuasiLinear?", 1) != 0;
    SP.equations_to_use = read_key<std::string>(full, "equations_to_use_", std::string("MHD_BQlin"));
    SP.CFL = read_key<double>(full, "CFL_", 1.0);
    SP.f_noise = read_key<double>(full, "f_noise_", 0.0);
    SP.noise_range_low = read_key<double>(full, "noise_range_low_", 0.0);
    SP.noise_range_high = read_key<double>(full, "noise_range_high_", 1e16);
    SP.noise_seed = (unsigned long long)read_key<double>(full, "noise_seed_", 0.0);
    SP.drive_only_velocityQ = read_key<int>(full, "drive_only_velocity?", 0) != 0;
    SP.drive_only_magneticQ = read_key<int>(full, "drive_only_magnetic?", 0) != 0;
    const double tv_save = read_key<double>(full, "tv_save_", SP.dt < 0 ? -SP.dt : SP.dt);
    const int integ = read_key<int>(full, "integrator_", 0);  // 0 RK3CN_Elin (main.cpp:95), 1 RK3CN
    const int nsteps = std::atoi(argv[3]);
    try {
        qlgpu::Model* model = nullptr;
        if (SP.equations_to_use == "MHD_BQlin") model = new qlgpu::MHD_BQlin(SP);
        else if (SP.equations_to_use == "MHD_FullQlin") model = new qlgpu::MHD_FullQlin(SP);
        else {
            std::cerr << "ERROR: no matching model found!" << std::endl;  // main.cpp:71-74
            return 1;
        }
        qlgpu::solution sol(model);
        std::ifstream sin(argv[2], std::ios::binary);
        double t = 0;
        sin.read(reinterpret_cast<char*>(&t), sizeof(double));
        sin.read(reinterpret_cast<char*>(sol.lin.data()), sol.lin.size() * sizeof(qlgpu::dcmplx));
        sin.read(reinterpret_cast<char*>(sol.mf.data()), sol.mf.size() * sizeof(qlgpu::dcmplx));
        sin.read(reinterpret_cast<char*>(sol.kx0.data()), sol.kx0.size() * sizeof(double));
        if (!sin) {
            std::cerr << "state file too short" << std::endl;
            return 1;
        }
        const std::vector<qlgpu::dcmplx> mf0 = sol.mf;
        qlgpu::Integrator* integrator = integ == 1 ? static_cast<qlgpu::Integrator*>(new qlgpu::RK3CN(t, SP, model))
                                                   : static_cast<qlgpu::Integrator*>(new qlgpu::RK3CN_Elin(t, SP, model));
        // a record every tv_save_ of time at a fixed dt; with the CFL dt (dt_ < 0) every
        // tv_save_ / |dt_| steps
        const int every = (int)(tv_save / (SP.dt < 0 ? -SP.dt : SP.dt) + 0.5);
        std::vector<double> diag = integrator->Run(t, &sol, nsteps, every);
        double tout = 0;
        qlgpu_time(integrator->handle(), &tout);
        std::ofstream so(argv[4], std::ios::binary);
        so.write(reinterpret_cast<const char*>(&tout), sizeof(double));
        so.write(reinterpret_cast<const char*>(sol.lin.data()), sol.lin.size() * sizeof(qlgpu::dcmplx));
        so.write(reinterpret_cast<const char*>(sol.mf.data()), sol.mf.size() * sizeof(qlgpu::dcmplx));
        so.write(reinterpret_cast<const char*>(sol.kx0.data()), sol.kx0.size() * sizeof(double));
        std::ofstream sd(argv[5], std::ios::binary);
        sd.write(reinterpret_cast<const char*>(diag.data()), diag.size() * sizeof(double));
        std::printf("ql_main: %d steps, t = %.10g, %zu diagnostic records\n", nsteps, tout, diag.size() / 15);
        if (argc > 6) {
            // Output directory (SP.simulation_dir): the TimeVariables files (main.cpp:98-130) with a
            // record per diagnostic save and the mean fields at the start and the end, and a full
            // save of the final state when full_save_ > 0 (main.cpp:135-140).
            const std::string dir = std::string(argv[6]) + "/";
            const qlgpu_params gp = model->params();
            qlgpu_timevars_t* tv = nullptr;
            const int nrey = SP.equations_to_use == "MHD_BQlin" ? 5 : 4;
            char msg[256];
            if (qlgpu_timevars_open(dir.c_str(), model->num_MFs(), model->NZfull(), nrey, 0, &tv) != QLGPU_OK) {
                qlgpu_io_last_error(msg, sizeof(msg));
                std::cerr << "time variables: " << msg << std::endl;
                return 1;
            }
            qlgpu_timevars_save_mean_fields(tv, reinterpret_cast<const double*>(mf0.data()), model->NZ());
            for (size_t r = 0; r < diag.size() / 15; ++r) qlgpu_timevars_save_data(tv, diag.data() + 15 * r);
            qlgpu_timevars_save_mean_fields(tv, reinterpret_cast<const double*>(sol.mf.data()), model->NZ());
            qlgpu_timevars_close(tv);
            if (read_key<double>(full, "full_save_", 0.0) > 0.0 &&
                qlgpu_fullsave_write((dir + "FullSave.bin").c_str(), &gp, tout,
                                     reinterpret_cast<const double*>(sol.lin.data()),
                                     reinterpret_cast<const double*>(sol.mf.data()), sol.kx0.data()) != QLGPU_OK) {
                qlgpu_io_last_error(msg, sizeof(msg));
                std::cerr << "full save: " << msg << std::endl;
                return 1;
            }
        }
        delete integrator;
        delete model;
    } catch (const qlgpu::Error& e) {
        std::cerr << "qlgpu error " << e.code << ": " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
