// ql_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// CPU FP64 restatement of the quasi-linear shearing-box time step of
// Cxb1993/ql_dns: the wavenumber tables, the FFTW-convention z transforms with
// 2/3 dealiasing, the MHD_BQlin and MHD_FullQlin right-hand sides, linear
// operators, shearing-wave remap and energy / stress / dissipation
// diagnostics, both RK3 integrators (exponential and Crank-Nicolson) and the
// main-loop order.  Every function cites the reference file:line it follows.
//
// Parity status: UNPINNED against the reference itself.  The reference cannot
// be built in this environment (it needs FFTW3, Eigen, Boost.Random, HDF5 and
// MPI, none of which are installed, and two of its sources are missing) and it
// ships no golden vectors or tests.  This restatement is pinned instead by
// (1) numpy.fft for the transform convention, (2) an independent numpy
// restatement of one MHD_BQlin rhs / RK3 step, (3) physics checks (RK3 order,
// linear MRI growth, remap timing, invariants).  See tests/.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// this library.
//
// Two builds come from this file (oracle/Makefile):
//   liboracle_strict.so : -O2 -ffp-contract=off, serial    (parity)
//   liboracle_fast.so   : -O3 -march=native -ffast-math, OpenMP over modes
//                         (CPU baseline timing, mirrors SConstruct:6 flags and
//                          stands in for the MPI mode split MPIdata.cpp:30-33)

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <complex>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;
typedef std::vector<cd> cvec;
typedef std::vector<double> dvec;

static const double PI_ = 3.14159265358979323846;  // General_Definitions.h PI

extern "C" {
// Plain-old-data parameter block passed from Python (ctypes) to the oracle.
struct OracleParams {
    int model;            // 0 = MHD_BQlin, 1 = MHD_FullQlin
    int integrator;       // 0 = RK3CN_Elin (exponential), 1 = RK3CN (Crank-Nicolson)
    int nx, ny, NZ;       // Inputs::NXY[0], NXY[1], NZ  (Input_parameters.cpp:68-70)
    double L[3];          // Lx, Ly, Lz                   (Input_parameters.cpp:71-73)
    double q, omega;      // shear, rotation (omega used by FullQlin only, MHD_BQlin.cpp:19)
    double nu, eta, B0z;  // dissipation, mean vertical field
    int viscosity_order;  // FullQlin hyper-dissipation order (int, MHD_FullQlin.h:73)
    double dt;            // fixed time step (> 0)
    int remap;            // Remap?
    int quasilinear;      // QuasiLinear?
    int nthreads;         // OpenMP threads for the fast build (0 = default)
};
}

// ---------------------------------------------------------------------------
// FFT with FFTW's conventions: forward = exp(-2 pi i jk/N), backward =
// exp(+2 pi i jk/N), unnormalised both ways (fftwPlans.cpp:48-51).  Iterative
// radix-2 for powers of two, a direct O(N^2) DFT otherwise.
// ---------------------------------------------------------------------------
struct Fft1D {
    int N;
    bool pow2;
    std::vector<int> rev;
    cvec tw_fwd, tw_bwd;  // exp(-+2 pi i k / N), k < N
    explicit Fft1D(int n) : N(n) {
        pow2 = (N & (N - 1)) == 0;
        tw_fwd.resize(N);
        tw_bwd.resize(N);
        for (int k = 0; k < N; ++k) {
            double a = 2.0 * PI_ * (double)k / (double)N;
            tw_fwd[k] = cd(std::cos(a), -std::sin(a));
            tw_bwd[k] = cd(std::cos(a), std::sin(a));
        }
        if (pow2) {
            rev.resize(N);
            int lg = 0;
            while ((1 << lg) < N) ++lg;
            for (int i = 0; i < N; ++i) {
                int r = 0;
                for (int b = 0; b < lg; ++b)
                    if (i & (1 << b)) r |= 1 << (lg - 1 - b);
                rev[i] = r;
            }
        }
    }
    void exec(cd* x, bool forward) const {
        const cvec& tw = forward ? tw_fwd : tw_bwd;
        if (!pow2) {
            cvec y(N);
            for (int k = 0; k < N; ++k) {
                cd s(0.0, 0.0);
                for (int j = 0; j < N; ++j) s += x[j] * tw[(long)j * k % N];
                y[k] = s;
            }
            for (int k = 0; k < N; ++k) x[k] = y[k];
            return;
        }
        for (int i = 0; i < N; ++i)
            if (i < rev[i]) std::swap(x[i], x[rev[i]]);
        for (int len = 2; len <= N; len <<= 1) {
            int half = len >> 1, step = N / len;
            for (int s = 0; s < N; s += len)
                for (int j = 0; j < half; ++j) {
                    cd w = tw[j * step];
                    cd a = x[s + j], b = x[s + j + half] * w;
                    x[s + j] = a + b;
                    x[s + j + half] = a - b;
                }
        }
    }
};

// fftwPlans restatement (fftwPlans.h:33-97, fftwPlans.cpp:29-34).
struct Plans {
    int NZnd, nz, deal_low, deal_high;
    double fac;
    Fft1D fft;
    Plans(int NZ, int nzd) : NZnd(NZ), nz(nzd), fft(NZ) {
        fac = 1.0 / NZnd;                 // fftwPlans.cpp:30
        deal_low = (nz - 1) / 2 + 1;      // fftwPlans.cpp:33
        deal_high = NZnd - (nz - 1) / 2;  // fftwPlans.cpp:34
    }
    // pad_with_zeros then backward transform (fftwPlans.h:43-51,66-82)
    void inverse(const cd* in, cd* out) const {
        int i = 0, j = deal_low;
        while (i < deal_low) { out[i] = in[i]; ++i; }
        while (j < deal_high) { out[j] = 0.0; ++j; }
        while (j < NZnd) { out[j] = in[i]; ++i; ++j; }
        fft.exec(out, false);
    }
    // forward transform in place, then truncate (fftwPlans.h:33-41,84-97)
    void forward(cd* in, cd* out) const {
        fft.exec(in, true);
        int i = 0, j = deal_high;
        while (i < deal_low) { out[i] = in[i]; ++i; }
        while (j < NZnd) { out[i] = in[j]; ++i; ++j; }
    }
};

// ---------------------------------------------------------------------------
// Model dimensions (Model.h:27-38) and wavenumber tables (Kdata.cpp:11-120)
// ---------------------------------------------------------------------------
struct Dims {
    int NZ, nz, Nx, Ny, nxy;
    int nMF, nLin;
};

struct Kd {
    std::vector<double> kx, ky;  // imaginary parts of the purely imaginary kx, ky
    std::vector<int> kx_index, ky_index;
    cvec kz;
    dvec kz2;
    std::vector<dvec> lap2, ilap2;
    double kxLfac, kyLfac, kzLfac;
};

static Dims make_dims(const OracleParams& p) {
    Dims d;
    d.NZ = p.NZ;
    d.nz = 1 + 2 * int(p.NZ / 3.0);          // Model.h:34
    d.Nx = p.nx;                              // Model.h:32
    d.Ny = (p.ny / 2) * 2;                    // Model.h:33,66
    d.nxy = (p.nx - 1) * (p.ny / 2);          // Model.h:36
    d.nMF = p.model == 0 ? 2 : 4;             // MHD_BQlin.cpp:14, MHD_FullQlin.cpp:14
    d.nLin = 4;
    return d;
}

static Kd make_kdata(const OracleParams& p, const Dims& d) {
    Kd K;
    K.kxLfac = 2 * PI_ / p.L[0];  // Kdata.cpp:24-26
    K.kyLfac = 2 * PI_ / p.L[1];
    K.kzLfac = 2 * PI_ / p.L[2];
    int ny = d.Ny / 2, nx = d.Nx / 2;  // Kdata.cpp:29
    K.kx.assign(d.nxy, 0.0);
    K.ky.assign(d.nxy, 0.0);
    K.kx_index.assign(d.nxy, 0);
    K.ky_index.assign(d.nxy, 0);
    for (int i = 0; i < nx; ++i)          // Kdata.cpp:30-37
        for (int j = 0; j < ny; ++j) {
            K.kx[j + ny * i] = i * K.kxLfac;
            K.ky[j + ny * i] = j * K.kyLfac;
            K.kx_index[j + ny * i] = i;
            K.ky_index[j + ny * i] = j;
        }
    for (int i = nx + 1; i < 2 * nx; ++i)  // Kdata.cpp:39-46 (kx Nyquist dropped)
        for (int j = 0; j < ny; ++j) {
            K.kx[j + ny * (i - 1)] = (-2 * nx + i) * K.kxLfac;
            K.ky[j + ny * (i - 1)] = j * K.kyLfac;
            K.kx_index[j + ny * (i - 1)] = -2 * nx + i;
            K.ky_index[j + ny * (i - 1)] = j;
        }
    K.kz.assign(d.nz, 0.0);  // Kdata.cpp:72-80
    K.kz2.assign(d.nz, 0.0);
    int nzl = (d.nz - 1) / 2;
    for (int i = 0; i < nzl + 1; ++i) K.kz[i] = cd(0, i * K.kzLfac);
    for (int i = nzl + 1; i < 2 * nzl + 1; ++i) K.kz[i] = cd(0, (-2 * nzl + i - 1) * K.kzLfac);
    for (int i = 0; i < d.nz; ++i) K.kz2[i] = (K.kz[i] * K.kz[i]).real();
    K.lap2.resize(ny);  // Kdata.cpp:96-120
    K.ilap2.resize(ny);
    for (int i = 0; i < ny; ++i) {
        double kyr = K.ky[i];
        dvec l2(d.nz), il2(d.nz);
        for (int k = 0; k < d.nz; ++k) {
            l2[k] = -kyr * kyr + K.kz2[k];
            il2[k] = 1 / l2[k];
        }
        if (kyr == 0) {
            l2[0] = 0;
            il2[0] = 1;
        }
        K.lap2[i] = l2;
        K.ilap2[i] = il2;
    }
    return K;
}

// ---------------------------------------------------------------------------
// State (solution.h:23-49): lin[(i*nLin + v)*nz + k], mf[m*nz + k]
// ---------------------------------------------------------------------------
struct State {
    int nxy, nLin, nz, nMF;
    cvec lin, mf;
    void init(const Dims& d) {
        nxy = d.nxy; nLin = d.nLin; nz = d.nz; nMF = d.nMF;
        lin.assign((size_t)nxy * nLin * nz, 0.0);
        mf.assign((size_t)nMF * nz, 0.0);
    }
    cd* pLin(int i, int v) { return &lin[((size_t)i * nLin + v) * nz]; }
    cd* pMF(int m) { return &mf[(size_t)m * nz]; }
    const cd* pLin(int i, int v) const { return &lin[((size_t)i * nLin + v) * nz]; }
    const cd* pMF(int m) const { return &mf[(size_t)m * nz]; }
};

// Per-mode laplacians at time t (MHD_BQlin.cpp:493-509; MHD_FullQlin.cpp:722-738)
struct ModeK {
    cd kxc, kyc;
    double kx, ky;
    dvec lapF, ilapF, lap2, ilap2;
};

static void assign_laplacians(const OracleParams& p, const Dims& d, const Kd& K,
                              const std::vector<double>& kx0, int i, double t,
                              bool need_inverse, ModeK& m) {
    int ind_ky = K.ky_index[i];
    m.kyc = cd(0, K.ky[i]);
    m.ky = m.kyc.imag();
    m.kxc = cd(0, kx0[i]) + p.q * t * m.kyc;
    m.kx = m.kxc.imag();
    m.lap2 = K.lap2[ind_ky];
    m.lapF.resize(d.nz);
    for (int k = 0; k < d.nz; ++k) m.lapF[k] = -m.kx * m.kx + m.lap2[k];
    if (need_inverse) {
        m.ilap2 = K.ilap2[ind_ky];
        m.ilapF.resize(d.nz);
        for (int k = 0; k < d.nz; ++k) m.ilapF[k] = 1 / m.lapF[k];
        if (ind_ky == 0 && K.kx_index[i] == 0) m.ilapF[0] = 1.0;
    }
}

// ---------------------------------------------------------------------------
// Model: right-hand sides
// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter (c0..c3), key (k0, k1).
static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += W0; k1 += W1; }
        const uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    }
}

// Two standard normals from the counter (a, b, step) under key seed: Box-Muller
// on two 53-bit uniforms, u1 in (0, 1), u2 in [0, 1).
static void philox_normal_pair(unsigned long long seed, unsigned long long step, uint32_t a, uint32_t b,
                               double* z1, double* z2) {
    uint32_t c[4] = {a, b, (uint32_t)step, (uint32_t)(step >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t x = ((uint64_t)c[0] << 32) | c[1], y = ((uint64_t)c[2] << 32) | c[3];
    const double u1 = ((double)(x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(y >> 11) * (1.0 / 9007199254740992.0);
    const double r = std::sqrt(-2.0 * std::log(u1));
    *z1 = r * std::cos(2.0 * PI_ * u2);
    *z2 = r * std::sin(2.0 * PI_ * u2);
}

struct Model {
    OracleParams p;
    Dims d;
    Kd K;
    Plans fft;
    double reynolds_stress_ft_fac;
    long totalN2;
    int num_to_send;
    int nthreads;
    // max |profile|^2 over the NZ grid of the real-space mean fields of the last
    // rhs call's input (By_ / MBx_, MBy_, MUx_, MUy_ members, zero before the
    // first call: MHD_BQlin.cpp:105, MHD_FullQlin.cpp:151); Calculate_CFL reads them
    double mf_max2[4] = {0, 0, 0, 0};
    Model(const OracleParams& pp)
        : p(pp), d(make_dims(pp)), K(make_kdata(pp, d)), fft(pp.NZ, d.nz) {
        reynolds_stress_ft_fac = 1.0 / (d.Ny * d.Nx) / (d.Ny * d.Nx);  // MHD_BQlin.cpp:56
        totalN2 = (long)d.Nx * d.Ny * d.NZ;                             // MHD_BQlin.cpp:52-53
        totalN2 = totalN2 * totalN2;
        num_to_send = (d.nz - 1) / 2 + 1;                               // MHD_BQlin.cpp:63
        nthreads = 1;
#ifdef _OPENMP
        nthreads = p.nthreads > 0 ? p.nthreads : omp_get_max_threads();
#endif
    }

    static double max_abs2(const cvec& v) {
        double m = 0;
        for (const cd& x : v) m = std::max(m, std::norm(x));
        return m;
    }

    // Calculate_CFL: MHD_BQlin.cpp:540-552 (By from the last rhs, Bx from sol),
    // MHD_FullQlin.cpp:769-780 (all four from the last rhs); kmax of
    // MHD_BQlin.cpp:69-74 (dealias factors 2, 2, 3).
    double calculate_cfl(const State& sol) const {
        const double Ns[3] = {(double)d.Nx, (double)d.Ny, (double)d.NZ};
        const double dealias[3] = {2.0, 2.0, 3.0};
        double kmax = 0;
        for (int i = 0; i < 3; ++i) kmax = std::max(kmax, 2 * PI_ / p.L[i] * (Ns[i] / dealias[i]));
        if (p.model == 1)
            return kmax * (std::sqrt(mf_max2[1]) + std::sqrt(mf_max2[0]) + std::sqrt(mf_max2[2]) +
                           std::sqrt(mf_max2[3])) + p.q;
        cvec tmp(d.nz), bx(d.NZ);
        for (int k = 0; k < d.nz; ++k) tmp[k] = sol.pMF(0)[k] * fft.fac;
        fft.inverse(tmp.data(), bx.data());
        return kmax * std::sqrt(mf_max2[1]) + kmax * std::sqrt(max_abs2(bx)) + p.q;
    }

    // DrivingNoise of MHD_BQlin (MHD_BQlin.cpp:558-618; ky = 0 modes are not
    // driven, dont_drive_ky0_modes_ = 1 at :18) and of MHD_FullQlin
    // (MHD_FullQlin.cpp:786-1045: the same on ky != 0 modes, :795-848, with the
    // drive_only_velocity / drive_only_magnetic switches of :21-22, and ky = 0
    // driven, dont_drive_ky0_modes_ = 0 at :19).  For ky = 0 every kx < 0 mode
    // (Kdata.cpp:124-146: its kx > 0 partner has the same |kx|) draws noise at kz
    // indices 1..nz-1 (:969-1023) and the partner adds the reversed conjugate
    // buffer to indices 1..nz-1 (:1028-1040), pos[nz - k] += conj(noise_neg[k]).
    // The reference draws from a clock-seeded mt19937 (MHD_BQlin.cpp:22-23);
    // here every (step, mode, kz, field) has its own Philox4x32-10 counter and
    // Box-Muller pair, so runs are reproducible and the GPU draws the same numbers.
    void driving_noise(double t, double dt, State& sol, const std::vector<double>& kx0, double f_noise,
                       double k_lo, double k_hi, unsigned long long seed, unsigned long long step,
                       bool only_velocity = false, bool only_magnetic = false) {
        const double lo2 = k_lo * k_lo, hi2 = k_hi * k_hi;
        const double mult_noise_fac = (1.0 / (16 * 32 * 32)) * (1.0 / (16 * 32 * 32));  // :35-36
        const double multfac = dt * (double)totalN2 * mult_noise_fac;
        const double sd = f_noise / std::sqrt(2.0);
        const bool full = p.model == 1;
        const bool drive_v[4] = {!(full && only_magnetic), !(full && only_magnetic), !(full && only_velocity),
                                 !(full && only_velocity)};
        auto draw = [&](int i, int k, int v, double mult) {
            double z1, z2;
            philox_normal_pair(seed, step, (unsigned)i, (unsigned)(4 * k + v), &z1, &z2);
            return mult * cd(z1 * sd, z2 * sd);
        };
        for (int i = 0; i < d.nxy; ++i) {
            if (K.ky_index[i] == 0) continue;
            ModeK m;
            assign_laplacians(p, d, K, kx0, i, t, false, m);
            for (int k = 0; k < d.nz; ++k) {
                const double lapF = m.lapF[k], lap2 = m.lap2[k];
                if (!(lapF > -hi2 && lapF < -lo2)) continue;
                const double mu = std::sqrt(multfac * lap2 / lapF);
                const double mz = std::sqrt(-multfac * lap2);
                for (int v = 0; v < 4; ++v) {
                    if (!drive_v[v]) continue;
                    sol.pLin(i, v)[k] += draw(i, k, v, (v == 0 || v == 2) ? mu : mz);
                }
            }
        }
        if (!full) return;
        const int nx = d.Nx / 2, ny = d.Ny / 2;
        for (int a = 1; a < nx; ++a) {
            const int ipos = a * ny;                 // kx index a (Kdata.cpp:30-37)
            const int ineg = (2 * nx - a - 1) * ny;  // kx index -a (Kdata.cpp:39-46)
            ModeK m;
            assign_laplacians(p, d, K, kx0, ineg, t, false, m);
            for (int k = 1; k < d.nz; ++k) {
                const double lapF = m.lapF[k], lap2 = m.lap2[k];
                if (!(lapF > -hi2 && lapF < -lo2)) continue;
                const double mu = std::sqrt(multfac * lap2 / lapF);
                const double mz = std::sqrt(-multfac * lap2);
                for (int v = 0; v < 4; ++v) {
                    if (!drive_v[v]) continue;
                    const cd n = draw(ineg, k, v, (v == 0 || v == 2) ? mu : mz);
                    sol.pLin(ineg, v)[k] += n;
                    sol.pLin(ipos, v)[d.nz - k] += std::conj(n);
                }
            }
        }
    }

    // MHD_BQlin::rhs, MHD_BQlin.cpp:117-284.  kx0 holds the (possibly remapped)
    // unsheared kx of each mode (Kdata::kx).  linOp[(i*nLin+v)*nz+k].
    void rhs_bqlin(double t, double dt_lin, const State& in, State& out,
                   const std::vector<double>& kx0, dvec& linOp) {
        const int nz = d.nz, NZ = d.NZ;
        const double fac = fft.fac;
        const double Omega = 2.0 / 3.0 * p.q;  // MHD_BQlin.cpp:19
        // Mean fields in real space (:122-127)
        cvec By(NZ), dzBy(NZ), dzdzBy(NZ), tmp(nz);
        for (int k = 0; k < nz; ++k) tmp[k] = in.pMF(1)[k] * fac;
        fft.inverse(tmp.data(), By.data());
        for (int k = 0; k < nz; ++k) tmp[k] = fac * K.kz[k] * in.pMF(1)[k];
        fft.inverse(tmp.data(), dzBy.data());
        for (int k = 0; k < nz; ++k) tmp[k] = fac * K.kz2[k] * in.pMF(1)[k];
        fft.inverse(tmp.data(), dzdzBy.data());
        mf_max2[1] = max_abs2(By);

        std::vector<cvec> send_thr(nthreads, cvec(2 * num_to_send, 0.0));
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
        for (int i = 0; i < d.nxy; ++i) {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            cvec& send = send_thr[tid];
            ModeK m;
            assign_laplacians(p, d, K, kx0, i, t, true, m);  // :140
            const cd kxc = m.kxc, kyc = m.kyc;
            const cd* u = in.pLin(i, 0);
            const cd* ze = in.pLin(i, 1);
            const cd* b = in.pLin(i, 2);
            const cd* et = in.pLin(i, 3);
            cvec uy(nz), uz(nz), by(nz), bz(nz);
            for (int k = 0; k < nz; ++k) {  // :143-146
                uy[k] = ((-kyc * kxc) * u[k] + K.kz[k] * ze[k]) * m.ilap2[k];
                uz[k] = (-kxc * K.kz[k] * u[k] - kyc * ze[k]) * m.ilap2[k];
                by[k] = ((-kyc * kxc) * b[k] + K.kz[k] * et[k]) * m.ilap2[k];
                bz[k] = (-kxc * K.kz[k] * b[k] - kyc * et[k]) * m.ilap2[k];
            }
            cvec t1z(NZ), t2z(NZ), t3z(NZ), t1k(nz), t2k(nz), t3k(nz);
            cd* Fu = out.pLin(i, 0);
            cd* Fz = out.pLin(i, 1);
            cd* Fb = out.pLin(i, 2);
            cd* Fe = out.pLin(i, 3);
            // u  (:153-162)
            for (int k = 0; k < nz; ++k) t1k[k] = (fac * kyc) * b[k];
            fft.inverse(t1k.data(), t1z.data());
            for (int j = 0; j < NZ; ++j) t1z[j] *= By[j];
            for (int k = 0; k < nz; ++k) t2k[k] = (-2.0 * fac * kxc * kyc) * bz[k];
            fft.inverse(t2k.data(), t2z.data());
            for (int j = 0; j < NZ; ++j) t2z[j] *= dzBy[j];
            fft.forward(t1z.data(), Fu);
            fft.forward(t2z.data(), t2k.data());
            for (int k = 0; k < nz; ++k)
                Fu[k] += ((-2.0 * kxc * kyc * p.q) * u[k] + 2 * Omega * K.kz[k] * ze[k] + t2k[k]) * m.ilapF[k];
            // zeta (:166-178)
            for (int k = 0; k < nz; ++k) t1k[k] = (fac * kyc) * et[k];
            fft.inverse(t1k.data(), t1z.data());
            for (int j = 0; j < NZ; ++j) t1z[j] *= By[j];
            for (int k = 0; k < nz; ++k) t2k[k] = (-fac * kxc) * b[k];
            fft.inverse(t2k.data(), t2z.data());
            for (int j = 0; j < NZ; ++j) t2z[j] *= dzBy[j];
            for (int k = 0; k < nz; ++k) t3k[k] = fac * bz[k];
            fft.inverse(t3k.data(), t3z.data());
            for (int j = 0; j < NZ; ++j) t3z[j] *= dzdzBy[j];
            for (int j = 0; j < NZ; ++j) t1z[j] += t2z[j] + t3z[j];
            fft.forward(t1z.data(), Fz);
            for (int k = 0; k < nz; ++k) Fz[k] += (p.q - 2.0 * Omega) * K.kz[k] * u[k];
            // b (:182-185)
            for (int k = 0; k < nz; ++k) t1k[k] = (fac * kyc) * u[k];
            fft.inverse(t1k.data(), t1z.data());
            for (int j = 0; j < NZ; ++j) t1z[j] *= By[j];
            fft.forward(t1z.data(), Fb);
            // eta (:189-201)
            for (int k = 0; k < nz; ++k) t1k[k] = (fac * kyc) * ze[k];
            fft.inverse(t1k.data(), t1z.data());
            for (int j = 0; j < NZ; ++j) t1z[j] *= By[j];
            for (int k = 0; k < nz; ++k) t2k[k] = (-2 * fac * K.kz[k] * uz[k]) - (fac * kxc) * u[k];
            fft.inverse(t2k.data(), t2z.data());
            for (int j = 0; j < NZ; ++j) t2z[j] *= dzBy[j];
            for (int k = 0; k < nz; ++k) t3k[k] = -fac * uz[k];
            fft.inverse(t3k.data(), t3z.data());
            for (int j = 0; j < NZ; ++j) t3z[j] *= dzdzBy[j];
            for (int j = 0; j < NZ; ++j) t1z[j] += t2z[j] + t3z[j];
            fft.forward(t1z.data(), Fe);
            for (int k = 0; k < nz; ++k) Fe[k] -= p.q * K.kz[k] * b[k];

            // Reynolds stress / EMF (:212-241)
            double mult_fac = 2.0;
            if (m.ky == 0.0) mult_fac = 1.0;
            double ftfac = mult_fac * fac * fac * reynolds_stress_ft_fac;
            cvec rz(NZ);
            fft.inverse(uz.data(), t1z.data());
            fft.inverse(bz.data(), t2z.data());
            fft.inverse(u, t3z.data());
            for (int j = 0; j < NZ; ++j) rz[j] = (t2z[j] * std::conj(t3z[j])).real();
            fft.inverse(b, t3z.data());
            for (int j = 0; j < NZ; ++j) rz[j] -= (t1z[j] * std::conj(t3z[j])).real();
            fft.forward(rz.data(), t1k.data());
            for (int k = 0; k < num_to_send; ++k) send[k] += ftfac * (K.kz[k] * t1k[k]);
            fft.inverse(uy.data(), t3z.data());
            for (int j = 0; j < NZ; ++j) rz[j] = (t2z[j] * std::conj(t3z[j])).real();
            fft.inverse(by.data(), t3z.data());
            for (int j = 0; j < NZ; ++j) rz[j] -= (t1z[j] * std::conj(t3z[j])).real();
            fft.forward(rz.data(), t1k.data());
            for (int k = 0; k < num_to_send; ++k) send[num_to_send + k] += ftfac * (K.kz[k] * t1k[k]);

            // Linear operator at t + dt_lin (:248-252)
            double kxt = m.kx + p.q * dt_lin * m.ky;
            double* L0 = &linOp[((size_t)i * 4 + 0) * nz];
            for (int k = 0; k < nz; ++k) L0[k] = p.nu * ((-kxt * kxt - m.ky * m.ky) + K.kz2[k]);
            for (int k = 0; k < nz; ++k) {
                linOp[((size_t)i * 4 + 1) * nz + k] = L0[k];
                linOp[((size_t)i * 4 + 2) * nz + k] = (p.eta / p.nu) * L0[k];
                linOp[((size_t)i * 4 + 3) * nz + k] = (p.eta / p.nu) * L0[k];
            }
        }
        // Sum over "ranks" (:262) and unpack reverse-conjugate (:264-267)
        cvec recv(2 * num_to_send, 0.0);
        for (int th = 0; th < nthreads; ++th)
            for (int k = 0; k < 2 * num_to_send; ++k) recv[k] += send_thr[th][k];
        cvec emf_x(nz), emf_y(nz);
        unpack_half(recv.data(), emf_x.data());
        unpack_half(recv.data() + num_to_send, emf_y.data());
        // Mean-field rhs (:274-280)
        for (int k = 0; k < nz; ++k) {
            if (p.quasilinear) {
                out.pMF(1)[k] = -p.q * in.pMF(0)[k] + emf_y[k];
                out.pMF(0)[k] = emf_x[k];
            } else {
                out.pMF(1)[k] = 0.0;
                out.pMF(0)[k] = 0.0;
            }
        }
    }

    void unpack_half(const cd* half, cd* full) const {  // MHD_BQlin.cpp:264-267
        int n = num_to_send;
        for (int k = 0; k < n; ++k) full[k] = half[k];
        for (int k = 0; k < n - 1; ++k) full[n + k] = std::conj(half[n - 1 - k]);
    }

    // MHD_FullQlin::rhs, MHD_FullQlin.cpp:171-427
    void rhs_fullqlin(double t, double dt_lin, const State& in, State& out,
                      const std::vector<double>& kx0, dvec& linOp) {
        const int nz = d.nz, NZ = d.NZ;
        const double fac = fft.fac;
        const double Omega = p.omega, B0z = p.B0z, q = p.q;
        const double L_mult = 1;  // turn_off_fluct_Lorentz_force_ = 0 (:24,111)
        // Mean fields in real space (:180-198): Bx, By, Ux, Uy and their z derivatives
        cvec MF[4], dzMF[4], tmp(nz);
        for (int m = 0; m < 4; ++m) {
            MF[m].assign(NZ, 0.0);
            dzMF[m].assign(NZ, 0.0);
            for (int k = 0; k < nz; ++k) tmp[k] = in.pMF(m)[k] * fac;
            fft.inverse(tmp.data(), MF[m].data());
            for (int k = 0; k < nz; ++k) tmp[k] = fac * K.kz[k] * in.pMF(m)[k];
            fft.inverse(tmp.data(), dzMF[m].data());
            mf_max2[m] = max_abs2(MF[m]);
        }
        const cvec &MBx = MF[0], &MBy = MF[1], &MUx = MF[2], &MUy = MF[3];
        const cvec &dzMBx = dzMF[0], &dzMBy = dzMF[1], &dzMUx = dzMF[2], &dzMUy = dzMF[3];

        std::vector<cvec> send_thr(nthreads, cvec(4 * num_to_send, 0.0));
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
        for (int i = 0; i < d.nxy; ++i) {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            cvec& send = send_thr[tid];
            ModeK m;
            assign_laplacians(p, d, K, kx0, i, t, true, m);  // :214
            const cd kxc = m.kxc, kyc = m.kyc;
            const cd* u0 = in.pLin(i, 0);
            const cd* ze = in.pLin(i, 1);
            const cd* b0 = in.pLin(i, 2);
            const cd* et = in.pLin(i, 3);
            cvec fy(nz), fz(nz), t1k(nz), t2k(nz), t3k(nz), t1z(NZ), rz(NZ);
            cvec U[9], B[9];
            for (int c = 0; c < 9; ++c) { U[c].assign(NZ, 0.0); B[c].assign(NZ, 0.0); }
            // u and derivatives (:220-242)
            for (int k = 0; k < nz; ++k) {
                fy[k] = ((-kyc * kxc) * u0[k] + K.kz[k] * ze[k]) * m.ilap2[k];
                fz[k] = (-kxc * K.kz[k] * u0[k] - kyc * ze[k]) * m.ilap2[k];
            }
            build_derivs(fac, kxc, kyc, u0, fy.data(), fz.data(), U, t1k);
            // b and derivatives (:245-265)
            for (int k = 0; k < nz; ++k) {
                fy[k] = ((-kyc * kxc) * b0[k] + K.kz[k] * et[k]) * m.ilap2[k];
                fz[k] = (-kxc * K.kz[k] * b0[k] - kyc * et[k]) * m.ilap2[k];
            }
            build_derivs(fac, kxc, kyc, b0, fy.data(), fz.data(), B, t1k);
            // u.grad(u) - b.grad(b) (:271-280)
            for (int j = 0; j < NZ; ++j)
                t1z[j] = MUx[j] * U[3][j] + MUy[j] * U[6][j] + U[2][j] * dzMUx[j] -
                         L_mult * (MBx[j] * B[3][j] + MBy[j] * B[6][j] + B[2][j] * dzMBx[j]);
            fft.forward(t1z.data(), t1k.data());
            for (int j = 0; j < NZ; ++j)
                t1z[j] = MUx[j] * U[4][j] + MUy[j] * U[7][j] + U[2][j] * dzMUy[j] -
                         L_mult * (MBx[j] * B[4][j] + MBy[j] * B[7][j] + B[2][j] * dzMBy[j]);
            fft.forward(t1z.data(), t2k.data());
            for (int j = 0; j < NZ; ++j)
                t1z[j] = MUx[j] * U[5][j] + MUy[j] * U[8][j] - L_mult * (MBx[j] * B[5][j] + MBy[j] * B[8][j]);
            fft.forward(t1z.data(), t3k.data());
            cd* Fu = out.pLin(i, 0);
            cd* Fz = out.pLin(i, 1);
            cd* Fb = out.pLin(i, 2);
            cd* Fe = out.pLin(i, 3);
            for (int k = 0; k < nz; ++k) {  // :283-285
                Fu[k] = ((-2.0 * kxc * kyc * q) * u0[k] + 2 * Omega * K.kz[k] * ze[k] +
                         (kxc * kxc) * t1k[k] + (kxc * kyc) * t2k[k] + kxc * K.kz[k] * t3k[k]) * m.ilapF[k] +
                        B0z * K.kz[k] * b0[k] - t1k[k];
                Fz[k] = (q - 2.0 * Omega) * K.kz[k] * u0[k] + B0z * K.kz[k] * et[k] -
                        (K.kz[k] * t2k[k] - kyc * t3k[k]);
            }
            // u.grad(b) - b.grad(u) (:291-305)
            for (int j = 0; j < NZ; ++j)
                t1z[j] = MUx[j] * B[3][j] + MUy[j] * B[6][j] + U[2][j] * dzMBx[j] -
                         (MBx[j] * U[3][j] + MBy[j] * U[6][j] + B[2][j] * dzMUx[j]);
            fft.forward(t1z.data(), t1k.data());
            for (int j = 0; j < NZ; ++j)
                t1z[j] = MUx[j] * B[4][j] + MUy[j] * B[7][j] + U[2][j] * dzMBy[j] -
                         (MBx[j] * U[4][j] + MBy[j] * U[7][j] + B[2][j] * dzMUy[j]);
            fft.forward(t1z.data(), t2k.data());
            for (int j = 0; j < NZ; ++j)
                t1z[j] = MUx[j] * B[5][j] + MUy[j] * B[8][j] - (MBx[j] * U[5][j] + MBy[j] * U[8][j]);
            fft.forward(t1z.data(), t3k.data());
            for (int k = 0; k < nz; ++k) {
                Fb[k] = B0z * K.kz[k] * u0[k] - t1k[k];
                Fe[k] = -q * K.kz[k] * b0[k] + B0z * K.kz[k] * ze[k] - (K.kz[k] * t2k[k] - kyc * t3k[k]);
            }
            // Stresses (:314-362)
            double mult_fac = 2.0;
            if (m.ky == 0.0) mult_fac = 1.0;
            double ftfac = mult_fac * reynolds_stress_ft_fac;
            const int n = num_to_send;
            for (int j = 0; j < NZ; ++j)
                rz[j] = (B[2][j] * std::conj(U[0][j])).real() - (U[2][j] * std::conj(B[0][j])).real();
            fft.forward(rz.data(), t1k.data());
            for (int k = 0; k < n; ++k) send[k] += ftfac * (K.kz[k] * t1k[k]);
            for (int j = 0; j < NZ; ++j)
                rz[j] = (B[2][j] * std::conj(U[1][j])).real() - (U[2][j] * std::conj(B[1][j])).real();
            fft.forward(rz.data(), t1k.data());
            for (int k = 0; k < n; ++k) send[n + k] += ftfac * (K.kz[k] * t1k[k]);
            // Ux drive: needs dz(ux), dz(bx)
            for (int k = 0; k < nz; ++k) {
                t1k[k] = fac * K.kz[k] * u0[k];
                t2k[k] = fac * K.kz[k] * b0[k];
            }
            cvec dzu(NZ), dzb(NZ);
            fft.inverse(t1k.data(), dzu.data());
            fft.inverse(t2k.data(), dzb.data());
            for (int j = 0; j < NZ; ++j)
                rz[j] = -((U[0][j] * std::conj(U[3][j])).real() + (U[1][j] * std::conj(U[6][j])).real() +
                          (U[2][j] * std::conj(dzu[j])).real()) +
                        ((B[0][j] * std::conj(B[3][j])).real() + (B[1][j] * std::conj(B[6][j])).real() +
                         (B[2][j] * std::conj(dzb[j])).real());
            fft.forward(rz.data(), t1k.data());
            for (int k = 0; k < n; ++k) send[2 * n + k] += ftfac * t1k[k];
            // Uy drive: dz(uy) (fluct_z_ redefined as uy, :352) and dz(by) (fluct_y_ is by)
            for (int k = 0; k < nz; ++k)
                fz[k] = ((-kyc * kxc) * u0[k] + K.kz[k] * ze[k]) * m.ilap2[k];
            for (int k = 0; k < nz; ++k) {
                t1k[k] = fac * K.kz[k] * fz[k];
                t2k[k] = fac * K.kz[k] * fy[k];
            }
            fft.inverse(t1k.data(), dzu.data());
            fft.inverse(t2k.data(), dzb.data());
            for (int j = 0; j < NZ; ++j)
                rz[j] = -((U[0][j] * std::conj(U[4][j])).real() + (U[1][j] * std::conj(U[7][j])).real() +
                          (U[2][j] * std::conj(dzu[j])).real()) +
                        ((B[0][j] * std::conj(B[4][j])).real() + (B[1][j] * std::conj(B[7][j])).real() +
                         (B[2][j] * std::conj(dzb[j])).real());
            fft.forward(rz.data(), t1k.data());
            for (int k = 0; k < n; ++k) send[3 * n + k] += ftfac * t1k[k];
            // Linear part (:371-376): -|k^2|^(order/2) with integer order/2
            double kxt = m.kx + q * dt_lin * m.ky;
            for (int k = 0; k < nz; ++k) {
                double lapF = -std::pow(std::fabs((-kxt * kxt - m.ky * m.ky) + K.kz2[k]),
                                        (double)(p.viscosity_order / 2));
                linOp[((size_t)i * 4 + 0) * nz + k] = p.nu * lapF;
                linOp[((size_t)i * 4 + 1) * nz + k] = p.nu * lapF;
                linOp[((size_t)i * 4 + 2) * nz + k] = p.eta * lapF;
                linOp[((size_t)i * 4 + 3) * nz + k] = p.eta * lapF;
            }
        }
        cvec recv(4 * num_to_send, 0.0);
        for (int th = 0; th < nthreads; ++th)
            for (int k = 0; k < 4 * num_to_send; ++k) recv[k] += send_thr[th][k];
        cvec drive[4];
        for (int m = 0; m < 4; ++m) {  // :389-399
            drive[m].assign(nz, 0.0);
            unpack_half(recv.data() + m * num_to_send, drive[m].data());
        }
        for (int k = 0; k < nz; ++k) {  // :411-423
            if (p.quasilinear) {
                cd Bx = in.pMF(0)[k], By = in.pMF(1)[k], Ux = in.pMF(2)[k], Uy = in.pMF(3)[k];
                out.pMF(1)[k] = -q * Bx + B0z * K.kz[k] * Uy + drive[1][k];
                out.pMF(0)[k] = B0z * K.kz[k] * Ux + drive[0][k];
                out.pMF(2)[k] = 2 * Omega * Uy + B0z * K.kz[k] * Bx + drive[2][k];
                out.pMF(3)[k] = (q - 2.0 * Omega) * Ux + B0z * K.kz[k] * By + drive[3][k];
            } else {
                for (int mm = 0; mm < 4; ++mm) out.pMF(mm)[k] = 0.0;
            }
        }
    }

    // u_[0..8]: f, fy, fz, dx f, dx fy, dx fz, dy f, dy fy, dy fz in real space
    // (MHD_FullQlin.cpp:225-242)
    void build_derivs(double fac, cd kxc, cd kyc, const cd* f0, const cd* fy, const cd* fz,
                      cvec* R, cvec& tk) const {
        const int nz = d.nz;
        const cd* src[3] = {f0, fy, fz};
        for (int c = 0; c < 3; ++c) {
            for (int k = 0; k < nz; ++k) tk[k] = fac * src[c][k];
            fft.inverse(tk.data(), R[c].data());
        }
        for (int c = 0; c < 3; ++c) {
            for (int k = 0; k < nz; ++k) tk[k] = (fac * kxc) * src[c][k];
            fft.inverse(tk.data(), R[3 + c].data());
        }
        for (int c = 0; c < 3; ++c) {
            for (int k = 0; k < nz; ++k) tk[k] = (fac * kyc) * src[c][k];
            fft.inverse(tk.data(), R[6 + c].data());
        }
    }

    void rhs(double t, double dt_lin, const State& in, State& out, const std::vector<double>& kx0,
             dvec& linOp) {
        if (p.model == 0)
            rhs_bqlin(t, dt_lin, in, out, kx0, linOp);
        else
            rhs_fullqlin(t, dt_lin, in, out, kx0, linOp);
    }

    // linearOPs_Init: MHD_BQlin.cpp:286-306, MHD_FullQlin.cpp:429-456
    void linearOPs_Init(double t0, const std::vector<double>& kx0, dvec& linOp, dvec& linOpMF) {
        const int nz = d.nz;
        for (int i = 0; i < d.nxy; ++i) {
            ModeK m;
            assign_laplacians(p, d, K, kx0, i, t0, false, m);
            for (int k = 0; k < nz; ++k) {
                double l0, l2;
                if (p.model == 0) {
                    l0 = p.nu * m.lapF[k];
                    l2 = (p.eta / p.nu) * l0;
                } else {
                    double lf = -std::pow(std::fabs(m.lapF[k]), (double)(p.viscosity_order / 2));
                    l0 = p.nu * lf;
                    l2 = p.eta * lf;
                }
                linOp[((size_t)i * 4 + 0) * nz + k] = l0;
                linOp[((size_t)i * 4 + 1) * nz + k] = l0;
                linOp[((size_t)i * 4 + 2) * nz + k] = l2;
                linOp[((size_t)i * 4 + 3) * nz + k] = l2;
            }
        }
        for (int mm = 0; mm < d.nMF; ++mm)
            for (int k = 0; k < nz; ++k) {
                double coef = (p.model == 1 && mm >= 2) ? p.nu : p.eta;
                linOpMF[(size_t)mm * nz + k] = p.quasilinear ? coef * K.kz2[k] : 0.0;
            }
    }

    // ShearingBox_Remap: MHD_BQlin.cpp:314-331 (identical in MHD_FullQlin.cpp:464-481)
    void remap(double qt, State& sol, std::vector<double>& kx0) {
        double kxLfac = 2 * PI_ / p.L[0];
        int nx = d.Nx - 1;
        for (int i = 0; i < d.nxy; ++i) {
            double kxt = kx0[i] + qt * K.ky[i];
            if (kxt > nx / 2.0 * kxLfac) {
                kx0[i] = kx0[i] - nx * kxLfac;
                for (int v = 0; v < 4; ++v)
                    for (int k = 0; k < d.nz; ++k) sol.pLin(i, v)[k] = 0.0;
            }
        }
    }

    // Calc_Energy_AM_Diss: MHD_BQlin.cpp:337-488, MHD_FullQlin.cpp:487-717.
    // out[12] = energy[MU,MB,u,b], AM[MU,MB,u,b], diss[MU,MB,u,b]; out[12..13] = etaK_times_kmax
    void diagnostics(double t, const State& sol, const std::vector<double>& kx0, double* out) {
        const int nz = d.nz;
        double energy_u = 0, energy_b = 0, AM_u = 0, AM_b = 0, diss_u = 0, diss_b = 0;
        for (int i = 0; i < d.nxy; ++i) {
            ModeK m;
            assign_laplacians(p, d, K, kx0, i, t, true, m);
            int mult_fac = 2;
            if (m.ky == 0.0) mult_fac = 1;
            dvec l2(nz);
            for (int k = 0; k < nz; ++k) l2[k] = m.lapF[k] * m.ilap2[k];  // :373
            const cd* u = sol.pLin(i, 0);
            const cd* ze = sol.pLin(i, 1);
            const cd* b = sol.pLin(i, 2);
            const cd* et = sol.pLin(i, 3);
            double su = 0, sb = 0, au = 0, ab = 0, du = 0, db = 0;
            for (int k = 0; k < nz; ++k) {  // :380-381 (Eigen .sum() of the elementwise expression)
                su += l2[k] * std::norm(u[k]) - m.ilap2[k] * std::norm(ze[k]);
                sb += l2[k] * std::norm(b[k]) - m.ilap2[k] * std::norm(et[k]);
            }
            energy_u += mult_fac * su;
            energy_b += mult_fac * sb;
            for (int k = 0; k < nz; ++k) {  // :388-392
                cd uy = ((-m.kyc * m.kxc) * u[k] + K.kz[k] * ze[k]) * m.ilap2[k];
                cd by = ((-m.kyc * m.kxc) * b[k] + K.kz[k] * et[k]) * m.ilap2[k];
                au += (u[k] * std::conj(uy)).real();
                ab += (b[k] * std::conj(by)).real();
            }
            AM_u += mult_fac * au;
            AM_b += mult_fac * ab;
            for (int k = 0; k < nz; ++k) {  // :400-401
                du += -m.lapF[k] * (l2[k] * std::norm(u[k]) - m.ilap2[k] * std::norm(ze[k]));
                db += -m.lapF[k] * (l2[k] * std::norm(b[k]) - m.ilap2[k] * std::norm(et[k]));
            }
            diss_u += (mult_fac * p.nu) * du;
            diss_b += (mult_fac * p.eta) * db;
        }
        double divfac = p.L[2] / (double)totalN2;  // :420
        energy_u *= divfac; energy_b *= divfac;
        AM_u *= divfac; AM_b *= divfac;
        diss_u *= divfac; diss_b *= divfac;
        double divMF = p.L[2] / ((double)d.NZ * d.NZ);  // :434
        double eMB = 0, eMU = 0, aMB = 0, aMU = 0, dMB = 0, dMU = 0;
        for (int k = 0; k < nz; ++k) {
            eMB += std::norm(sol.pMF(0)[k]) + std::norm(sol.pMF(1)[k]);
            aMB += (sol.pMF(0)[k] * std::conj(sol.pMF(1)[k])).real();
            dMB += -K.kz2[k] * std::norm(sol.pMF(0)[k]) - K.kz2[k] * std::norm(sol.pMF(1)[k]);
            if (p.model == 1) {
                eMU += std::norm(sol.pMF(2)[k]) + std::norm(sol.pMF(3)[k]);
                aMU += (sol.pMF(2)[k] * std::conj(sol.pMF(3)[k])).real();
                dMU += -K.kz2[k] * std::norm(sol.pMF(2)[k]) - K.kz2[k] * std::norm(sol.pMF(3)[k]);
            }
        }
        eMB *= divMF; eMU *= divMF; aMB *= divMF; aMU *= divMF;
        dMB *= divMF * p.eta; dMU *= divMF * p.nu;
        out[0] = eMU / 2; out[1] = eMB / 2; out[2] = energy_u / 2; out[3] = energy_b / 2;  // :449-453
        out[4] = aMU; out[5] = aMB; out[6] = AM_u; out[7] = AM_b;
        out[8] = dMU; out[9] = dMB; out[10] = diss_u; out[11] = diss_b;
        double kzmax = 2 * PI_ / p.L[2] * (d.NZ / 3);  // :476-477 (integer N(2)/3)
        out[12] = std::pow(p.nu * p.nu * p.nu / (dMU + diss_u), 0.25) * kzmax;
        out[13] = std::pow(p.eta * p.eta * p.eta / (dMB + diss_b), 0.25) * kzmax;
    }
};

// ---------------------------------------------------------------------------
// Integrators: RK3CN_Elin::Step (RK3CN_Elin.cpp:74-188), RK3CN::Step (RK3CN.cpp:77-202)
// ---------------------------------------------------------------------------
struct Integrator {
    Model& M;
    State rhs1, rhs2;
    dvec linOp, linOpOld, linOpMF;
    const double a0 = 8.0 / 15.0, a1 = 5.0 / 12.0, a2 = 3.0 / 4.0, b1 = -17.0 / 60.0, b2 = -5.0 / 12.0;
    const double p1 = 8.0 / 15.0, p2 = 2.0 / 3.0;
    Integrator(Model& m, double t0, const std::vector<double>& kx0) : M(m) {
        rhs1.init(M.d);
        rhs2.init(M.d);
        size_t n = (size_t)M.d.nxy * 4 * M.d.nz;
        linOp.assign(n, 0.0);
        linOpOld.assign(n, 0.0);
        linOpMF.assign((size_t)M.d.nMF * M.d.nz, 0.0);
        // Elin initialises linOp (RK3CN_Elin.cpp:56); CN initialises linOpOld (RK3CN.cpp:57)
        M.linearOPs_Init(t0, kx0, M.p.integrator == 0 ? linOp : linOpOld, linOpMF);
    }

    // Exponential update of stage s: u <- exp(c L)(n1 F + n2 Fprev + u)
    void update_exp(State& sol, const State& F, const State* Fp, double linC, double n1, double n2) {
        const int nz = M.d.nz;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(M.nthreads)
#endif
        for (int i = 0; i < M.d.nxy; ++i)
            for (int j = 0; j < 4; ++j) {
                cd* u = sol.pLin(i, j);
                const cd* f = F.pLin(i, j);
                const double* L = &linOp[((size_t)i * 4 + j) * nz];
                for (int k = 0; k < nz; ++k) {
                    double e = std::exp(linC * L[k]);
                    if (Fp)
                        u[k] = e * (n1 * f[k] + n2 * Fp->pLin(i, j)[k] + u[k]);
                    else
                        u[k] = e * (n1 * f[k] + u[k]);
                }
            }
        for (int mm = 0; mm < M.d.nMF; ++mm)
            for (int k = 0; k < nz; ++k) {
                double e = std::exp(linC * linOpMF[(size_t)mm * nz + k]);
                cd* u = sol.pMF(mm);
                if (Fp)
                    u[k] = e * (n1 * F.pMF(mm)[k] + n2 * Fp->pMF(mm)[k] + u[k]);
                else
                    u[k] = e * (n1 * F.pMF(mm)[k] + u[k]);
            }
    }

    // Crank-Nicolson update of stage s (RK3CN.cpp:102-115).  advance_old = false leaves the
    // old operator in place (the tangent of the same stage is updated first with it).
    void update_cn(State& sol, const State& F, const State* Fp, double linC, double n1, double n2,
                   bool advance_old = true) {
        const int nz = M.d.nz;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(M.nthreads)
#endif
        for (int i = 0; i < M.d.nxy; ++i)
            for (int j = 0; j < 4; ++j) {
                cd* u = sol.pLin(i, j);
                const cd* f = F.pLin(i, j);
                const double* L = &linOp[((size_t)i * 4 + j) * nz];
                const double* Lo = &linOpOld[((size_t)i * 4 + j) * nz];
                for (int k = 0; k < nz; ++k) {
                    double denom = 1.0 / (1.0 - linC * L[k]);
                    if (Fp)
                        u[k] = n1 * denom * f[k] + n2 * denom * Fp->pLin(i, j)[k] + (1 + linC * Lo[k]) * denom * u[k];
                    else
                        u[k] = n1 * denom * f[k] + (1 + linC * Lo[k]) * denom * u[k];
                }
            }
        for (int mm = 0; mm < M.d.nMF; ++mm)
            for (int k = 0; k < nz; ++k) {
                double Lm = linOpMF[(size_t)mm * nz + k];
                double denom = 1.0 / (1.0 - linC * Lm);
                cd* u = sol.pMF(mm);
                if (Fp)
                    u[k] = n1 * denom * F.pMF(mm)[k] + n2 * denom * Fp->pMF(mm)[k] + (1 + linC * Lm) * denom * u[k];
                else
                    u[k] = n1 * denom * F.pMF(mm)[k] + (1 + linC * Lm) * denom * u[k];
            }
        if (advance_old) linOpOld = linOp;  // RK3CN.cpp:119-122
    }

    double step(double t, double dt, State& sol, const std::vector<double>& kx0) {
        bool cn = M.p.integrator == 1;
        double lc_fac = cn ? dt / 2 : dt;
        // Stage 1
        double linC = lc_fac * a0, NLC1 = a0 * dt, lin_dt = dt * p1;
        M.rhs(t, lin_dt, sol, rhs1, kx0, linOp);
        if (cn) update_cn(sol, rhs1, nullptr, linC, NLC1, 0);
        else update_exp(sol, rhs1, nullptr, linC, NLC1, 0);
        // Stage 2
        linC = lc_fac * (a1 + b1); NLC1 = a1 * dt; double NLC2 = b1 * dt; lin_dt = dt * (p2 - p1);
        M.rhs(t + dt * p1, lin_dt, sol, rhs2, kx0, linOp);
        if (cn) update_cn(sol, rhs2, &rhs1, linC, NLC1, NLC2);
        else update_exp(sol, rhs2, &rhs1, linC, NLC1, NLC2);
        // Stage 3
        linC = lc_fac * (a2 + b2); NLC1 = a2 * dt; NLC2 = b2 * dt; lin_dt = dt * (1.0 - p2);
        M.rhs(t + dt * p2, lin_dt, sol, rhs1, kx0, linOp);
        if (cn) update_cn(sol, rhs1, &rhs2, linC, NLC1, NLC2);
        else update_exp(sol, rhs1, &rhs2, linC, NLC1, NLC2);
        return dt;
    }
};

// ---------------------------------------------------------------------------
// C ABI for the ctypes wrapper (oracle/oracle.py)
// ---------------------------------------------------------------------------
extern "C" {

int oracle_dims(const OracleParams* p, int* nxy, int* nz, int* nmf) {
    Dims d = make_dims(*p);
    *nxy = d.nxy; *nz = d.nz; *nmf = d.nMF;
    return 0;
}

// Mode tables: kx0[nxy], ky[nxy], kx_index[nxy], ky_index[nxy], kz[nz] (imag parts)
int oracle_ktables(const OracleParams* p, double* kx, double* ky, int* kxi, int* kyi, double* kz) {
    Dims d = make_dims(*p);
    Kd K = make_kdata(*p, d);
    for (int i = 0; i < d.nxy; ++i) {
        kx[i] = K.kx[i]; ky[i] = K.ky[i]; kxi[i] = K.kx_index[i]; kyi[i] = K.ky_index[i];
    }
    for (int k = 0; k < d.nz; ++k) kz[k] = K.kz[k].imag();
    return 0;
}

// Raw transforms for convention tests: dir = +1 forward, -1 backward; interleaved re/im.
int oracle_fft(int N, int dir, double* data) {
    Fft1D f(N);
    f.exec(reinterpret_cast<cd*>(data), dir > 0);
    return 0;
}

// One right-hand-side evaluation: Model::rhs(t, dt_lin, in, out, linOp).
int oracle_rhs(const OracleParams* p, double t, double dt_lin, const double* lin_in, const double* mf_in,
               const double* kx0_in, double* lin_out, double* mf_out, double* linop_out) {
    Model M(*p);
    State in, out;
    in.init(M.d);
    out.init(M.d);
    std::memcpy(in.lin.data(), lin_in, in.lin.size() * sizeof(cd));
    std::memcpy(in.mf.data(), mf_in, in.mf.size() * sizeof(cd));
    std::vector<double> kx0(M.K.kx);
    if (kx0_in) kx0.assign(kx0_in, kx0_in + M.d.nxy);
    dvec linOp((size_t)M.d.nxy * 4 * M.d.nz);
    M.rhs(t, dt_lin, in, out, kx0, linOp);
    std::memcpy(lin_out, out.lin.data(), out.lin.size() * sizeof(cd));
    std::memcpy(mf_out, out.mf.data(), out.mf.size() * sizeof(cd));
    if (linop_out) std::memcpy(linop_out, linOp.data(), linOp.size() * sizeof(double));
    return 0;
}

// Diagnostics of a state at time t (14 doubles).
int oracle_diagnostics(const OracleParams* p, double t, const double* lin, const double* mf,
                       const double* kx0_in, double* out) {
    Model M(*p);
    State s;
    s.init(M.d);
    std::memcpy(s.lin.data(), lin, s.lin.size() * sizeof(cd));
    std::memcpy(s.mf.data(), mf, s.mf.size() * sizeof(cd));
    std::vector<double> kx0(M.K.kx);
    if (kx0_in) kx0.assign(kx0_in, kx0_in + M.d.nxy);
    M.diagnostics(t, s, kx0, out);
    return 0;
}

// main.cpp:108-154 loop for a fixed number of steps.  diag_every > 0 computes
// diagnostics (t followed by 14 doubles per record) at t0 and then whenever the
// time-variable accumulator is due (interval = diag_every*dt, same test as
// main.cpp:391).  kx0_io holds the unsheared kx of every mode and is updated by
// the remap.  Returns the number of diagnostic records written.
int oracle_run(const OracleParams* p, double* t_io, double* lin_io, double* mf_io, double* kx0_io,
               int nsteps, int diag_every, double* diag_out, int max_diag) {
    Model M(*p);
    State s;
    s.init(M.d);
    std::memcpy(s.lin.data(), lin_io, s.lin.size() * sizeof(cd));
    std::memcpy(s.mf.data(), mf_io, s.mf.size() * sizeof(cd));
    std::vector<double> kx0(kx0_io, kx0_io + M.d.nxy);
    double t = *t_io;
    Integrator I(M, t, kx0);
    int nrec = 0;
    auto record = [&](double tt) {
        if (diag_every > 0 && diag_out && nrec < max_diag) {
            diag_out[nrec * 15] = tt;
            M.diagnostics(tt, s, kx0, diag_out + nrec * 15 + 1);
            ++nrec;
        }
    };
    record(t);
    double interval = diag_every > 0 ? diag_every * p->dt : 0.0;
    double timevar_t = 0.0;
    int since = 0;
    for (int n = 0; n < nsteps; ++n) {
        double dt = I.step(t, p->dt, s, kx0);
        t += dt;
        timevar_t += dt;
        ++since;
        if (p->remap) M.remap(p->q * t, s, kx0);
        if (diag_every > 0 && timevar_t - interval > -1e-8) {
            record(t);
            timevar_t -= interval;
            since = 0;
        }
    }
    if (diag_every > 0 && since != 0) record(t);
    *t_io = t;
    std::memcpy(lin_io, s.lin.data(), s.lin.size() * sizeof(cd));
    std::memcpy(mf_io, s.mf.data(), s.mf.size() * sizeof(cd));
    std::memcpy(kx0_io, kx0.data(), kx0.size() * sizeof(double));
    return nrec;
}

// The main loop with forcing (main.cpp:108-133): optional variable dt
// (RK3CN_Elin.cpp:76-80: dt = cfl / Calculate_CFL, capped at dt_max) and
// driving noise after every step (main.cpp:112-113), then t += dt and the
// remap.  A diagnostic record after every diag_every-th step (and the initial
// one).  Returns the record count; *dt_mean_out = Integrator::mean_time_step.
int oracle_run_forced_fields(const OracleParams* p, double* t_io, double* lin_io, double* mf_io, double* kx0_io,
                             int nsteps, int diag_every, double* diag_out, int max_diag, double cfl, double dt_max,
                             double f_noise, double k_lo, double k_hi, unsigned long long seed, int only_velocity,
                             int only_magnetic, double* dt_mean_out) {
    Model M(*p);
    State s;
    s.init(M.d);
    std::memcpy(s.lin.data(), lin_io, s.lin.size() * sizeof(cd));
    std::memcpy(s.mf.data(), mf_io, s.mf.size() * sizeof(cd));
    std::vector<double> kx0(kx0_io, kx0_io + M.d.nxy);
    double t = *t_io;
    Integrator I(M, t, kx0);
    int nrec = 0;
    auto record = [&](double tt) {
        if (diag_every > 0 && diag_out && nrec < max_diag) {
            diag_out[nrec * 15] = tt;
            M.diagnostics(tt, s, kx0, diag_out + nrec * 15 + 1);
            ++nrec;
        }
    };
    record(t);
    double dt_sum = 0;
    for (int n = 0; n < nsteps; ++n) {
        double dt = p->dt;
        if (cfl > 0) {
            dt = cfl / M.calculate_cfl(s);
            if (dt > dt_max) dt = dt_max;
        }
        I.step(t, dt, s, kx0);
        dt_sum += dt;
        if (f_noise != 0.0)
            M.driving_noise(t, dt, s, kx0, f_noise, k_lo, k_hi, seed, (unsigned long long)n, only_velocity != 0,
                            only_magnetic != 0);
        t += dt;
        if (p->remap) M.remap(p->q * t, s, kx0);
        if (diag_every > 0 && (n + 1) % diag_every == 0) record(t);
    }
    *t_io = t;
    if (dt_mean_out) *dt_mean_out = nsteps > 0 ? dt_sum / nsteps : 0.0;
    std::memcpy(lin_io, s.lin.data(), s.lin.size() * sizeof(cd));
    std::memcpy(mf_io, s.mf.data(), s.mf.size() * sizeof(cd));
    std::memcpy(kx0_io, kx0.data(), kx0.size() * sizeof(double));
    return nrec;
}

int oracle_run_forced(const OracleParams* p, double* t_io, double* lin_io, double* mf_io, double* kx0_io,
                      int nsteps, int diag_every, double* diag_out, int max_diag, double cfl, double dt_max,
                      double f_noise, double k_lo, double k_hi, unsigned long long seed, double* dt_mean_out) {
    return oracle_run_forced_fields(p, t_io, lin_io, mf_io, kx0_io, nsteps, diag_every, diag_out, max_diag, cfl,
                                    dt_max, f_noise, k_lo, k_hi, seed, 0, 0, dt_mean_out);
}

// Philox4x32-10 of one counter (known-answer tests of the generator).
int oracle_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox4x32_10(c, key[0], key[1]);
    for (int i = 0; i < 4; ++i) out[i] = c[i];
    return 0;
}

// Tangent-linear run for MHD_BQlin with RK3CN_Elin or RK3CN (the checker of the
// adjoint).  J = (1/N) sum_{n=1..N} AM_b after each step (main.cpp:108-133, AM_b
// of MHD_BQlin.cpp:392,424) and its derivative dJ in the direction (dlin, dmf)
// of the initial state.  The state is propagated with the tangent alongside:
// the stage update is linear (RK3CN_Elin.cpp:102-104; RK3CN.cpp:105-107 with
// the operators of the stage and of the previous stage) and is applied to both;
// the remap zeroes the same modes in both; the derivative of the rhs and of
// AM_b, both polynomials of degree two in the state, is taken exactly by the
// polarization identity D f(x) d = (f(x + h d) - f(x - h d)) / (2 h).
int oracle_tlm_maxwell(const OracleParams* p, double t0, const double* lin_in, const double* mf_in,
                       const double* kx0_in, const double* dlin_in, const double* dmf_in, int nsteps, double* J,
                       double* dJ) {
    if (p->model != 0) return 1;
    const bool cn = p->integrator == 1;
    Model M(*p);
    State s, ds;
    s.init(M.d);
    ds.init(M.d);
    std::memcpy(s.lin.data(), lin_in, s.lin.size() * sizeof(cd));
    std::memcpy(s.mf.data(), mf_in, s.mf.size() * sizeof(cd));
    std::memcpy(ds.lin.data(), dlin_in, ds.lin.size() * sizeof(cd));
    if (dmf_in) std::memcpy(ds.mf.data(), dmf_in, ds.mf.size() * sizeof(cd));
    std::vector<double> kx0(M.K.kx);
    if (kx0_in) kx0.assign(kx0_in, kx0_in + M.d.nxy);
    double t = t0;
    Integrator I(M, t, kx0);
    auto norm = [](const State& x) {
        double a = 0;
        for (const cd& v : x.lin) a += std::norm(v);
        for (const cd& v : x.mf) a += std::norm(v);
        return std::sqrt(a);
    };
    auto axpy = [&](State& out, const State& x, double h, const State& d) {
        for (size_t i = 0; i < x.lin.size(); ++i) out.lin[i] = x.lin[i] + h * d.lin[i];
        for (size_t i = 0; i < x.mf.size(); ++i) out.mf[i] = x.mf[i] + h * d.mf[i];
    };
    State F1, F2, dF1, dF2, xp, xm, Fp, Fm;
    for (State* z : {&F1, &F2, &dF1, &dF2, &xp, &xm, &Fp, &Fm}) z->init(M.d);
    dvec dummy((size_t)M.d.nxy * 4 * M.d.nz);
    auto step_h = [&](const State& x, const State& d) {
        const double nx = norm(x), nd = norm(d);
        return (nd > 0 && nx > 0) ? nx / nd : 1.0;
    };
    // dF = D rhs(x) d
    auto tangent_rhs = [&](double tt, double ldt, const State& x, const State& d, State& dF) {
        const double h = step_h(x, d);
        axpy(xp, x, h, d);
        axpy(xm, x, -h, d);
        M.rhs(tt, ldt, xp, Fp, kx0, dummy);
        M.rhs(tt, ldt, xm, Fm, kx0, dummy);
        for (size_t i = 0; i < dF.lin.size(); ++i) dF.lin[i] = (Fp.lin[i] - Fm.lin[i]) / (2 * h);
        for (size_t i = 0; i < dF.mf.size(); ++i) dF.mf[i] = (Fp.mf[i] - Fm.mf[i]) / (2 * h);
    };
    double diag[14];
    auto amb = [&](double tt, const State& x) {
        M.diagnostics(tt, x, kx0, diag);
        return diag[7];  // AM_b: energy[4], AM[4] -> index 7 of the 14 values
    };
    const double dt = p->dt;
    const double a0 = I.a0, a1 = I.a1, a2 = I.a2, b1 = I.b1, b2 = I.b2, p1 = I.p1, p2 = I.p2;
    const double lf = cn ? dt / 2 : dt;  // RK3CN.cpp:86 (dt/2) or RK3CN_Elin.cpp:89 (dt)
    // one stage update of the tangent, then of the state (the CN old operator advances after both)
    auto update2 = [&](const State& F, const State* Fp, const State& dF, const State* dFp, double linC, double n1,
                       double n2) {
        if (cn) {
            I.update_cn(ds, dF, dFp, linC, n1, n2, false);
            I.update_cn(s, F, Fp, linC, n1, n2, true);
        } else {
            I.update_exp(ds, dF, dFp, linC, n1, n2);
            I.update_exp(s, F, Fp, linC, n1, n2);
        }
    };
    double sJ = 0, sdJ = 0;
    for (int n = 0; n < nsteps; ++n) {
        // RK3CN_Elin::Step (RK3CN_Elin.cpp:86-177) / RK3CN::Step (RK3CN.cpp:77-202) on the
        // state and the tangent
        M.rhs(t, dt * p1, s, F1, kx0, I.linOp);
        tangent_rhs(t, dt * p1, s, ds, dF1);
        update2(F1, nullptr, dF1, nullptr, lf * a0, a0 * dt, 0);
        M.rhs(t + dt * p1, dt * (p2 - p1), s, F2, kx0, I.linOp);
        tangent_rhs(t + dt * p1, dt * (p2 - p1), s, ds, dF2);
        update2(F2, &F1, dF2, &dF1, lf * (a1 + b1), a1 * dt, b1 * dt);
        M.rhs(t + dt * p2, dt * (1.0 - p2), s, F1, kx0, I.linOp);
        tangent_rhs(t + dt * p2, dt * (1.0 - p2), s, ds, dF1);
        update2(F1, &F2, dF1, &dF2, lf * (a2 + b2), a2 * dt, b2 * dt);
        t += dt;
        if (p->remap) {
            std::vector<double> k2 = kx0;
            M.remap(p->q * t, s, kx0);
            M.remap(p->q * t, ds, k2);
        }
        sJ += amb(t, s);
        const double h = step_h(s, ds);
        axpy(xp, s, h, ds);
        axpy(xm, s, -h, ds);
        sdJ += (amb(t, xp) - amb(t, xm)) / (2 * h);
    }
    *J = sJ / nsteps;
    *dJ = sdJ / nsteps;
    return 0;
}

}  // extern "C"
