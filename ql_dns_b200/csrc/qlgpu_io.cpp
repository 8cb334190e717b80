// qlgpu_io.cpp -- host-side output and restart files (include/qlgpu_io.h):
// the TimeVariables .dat files (QL_DNS/Auxiliary/TimeVariables.cpp) and the
// FullSave_Load groups (QL_DNS/Auxiliary/FullSave_Load.cpp) in a raw binary
// container.  Plain C++, no device code.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qlgpu_io.h"
#include "qlgpu_host.h"

namespace {

thread_local std::string g_io_error;

int io_fail(int code, const std::string& msg) {
    g_io_error = msg;
    return code;
}

const char kMagic[8] = {'Q', 'L', 'F', 'S', 'A', 'V', 'E', '1'};

// The reference writes the time-variable files by re-opening them in append
// mode for every save (TimeVariables.cpp:151-158); the same is done here so a
// crash leaves complete records.
bool append_bytes(const std::string& path, const void* data, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "ab");
    if (!f) return false;
    const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
    return std::fclose(f) == 0 && ok;
}

bool create_empty(const std::string& path, bool truncate) {
    FILE* f = std::fopen(path.c_str(), truncate ? "wb" : "ab");
    if (!f) return false;
    return std::fclose(f) == 0;
}

}  // namespace

struct qlgpu_timevars {
    std::string dir;
    int nmf = 2, NZ = 32, num_reynolds = 5;
};

extern "C" {

int qlgpu_io_last_error(char* buf, int buflen) {
    if (buf && buflen > 0) std::snprintf(buf, (size_t)buflen, "%s", g_io_error.c_str());
    return (int)g_io_error.size();
}

// TimeVariables constructor (TimeVariables.cpp:25-124): file names and open modes.
int qlgpu_timevars_open(const char* dir, int nmf, int NZ, int num_reynolds, int append, qlgpu_timevars_t** out) {
    if (!dir || !out || nmf < 1 || NZ < 1 || num_reynolds < 0) return io_fail(QLGPU_ERR_ARG, "bad argument");
    *out = nullptr;
    qlgpu_timevars* tv = new qlgpu_timevars();
    tv->dir = dir;
    tv->nmf = nmf;
    tv->NZ = NZ;
    tv->num_reynolds = num_reynolds;
    const char* names[] = {"energy.dat", "angular_momentum.dat", "dissipation.dat", "reynolds_stress.dat",
                           "mean_fields.dat", "time_vec.dat"};
    for (const char* n : names)
        if (!create_empty(tv->dir + n, append == 0)) {
            delete tv;
            return io_fail(QLGPU_ERR_ARG, std::string("cannot open ") + dir + n);
        }
    *out = tv;
    return QLGPU_OK;
}

// Save_Data(t) (TimeVariables.cpp:143-190) from a diagnostic record
// {t, energy[4], AM[4], diss[4], etaK[2]} (MHD_BQlin.cpp:449-467).
int qlgpu_timevars_save_data(qlgpu_timevars_t* tv, const double* rec15) {
    if (!tv || !rec15) return io_fail(QLGPU_ERR_ARG, "null argument");
    std::vector<double> rey((size_t)tv->num_reynolds, 0.0);
    const bool ok = append_bytes(tv->dir + "energy.dat", rec15 + 1, 4 * sizeof(double)) &&
                    append_bytes(tv->dir + "angular_momentum.dat", rec15 + 5, 4 * sizeof(double)) &&
                    append_bytes(tv->dir + "dissipation.dat", rec15 + 9, 4 * sizeof(double)) &&
                    (rey.empty() || append_bytes(tv->dir + "reynolds_stress.dat", rey.data(), rey.size() * sizeof(double))) &&
                    append_bytes(tv->dir + "time_vec.dat", rec15, sizeof(double));
    return ok ? QLGPU_OK : io_fail(QLGPU_ERR_ARG, "write failed in " + tv->dir);
}

// Save_Mean_Fields (TimeVariables.cpp:194-224): real part of fac1D * inverse(MF)
// with the inverse of fftwPlans (zero padding nz -> NZ between deal_low and
// deal_high, backward sign, unnormalised; fftwPlans.cpp:29-34).
int qlgpu_timevars_save_mean_fields(qlgpu_timevars_t* tv, const double* mf, int nz) {
    if (!tv || !mf || nz < 1 || nz > tv->NZ) return io_fail(QLGPU_ERR_ARG, "bad argument");
    const int NZ = tv->NZ;
    const int low = (nz - 1) / 2 + 1;  // stored kz 0..low-1, then the negative ones
    std::vector<double> out((size_t)tv->nmf * NZ);
    for (int m = 0; m < tv->nmf; ++m) {
        const double* f = mf + (size_t)m * nz * 2;
        for (int z = 0; z < NZ; ++z) {
            double re = 0.0;
            for (int s = 0; s < nz; ++s) {
                const int k = s < low ? s : NZ - (nz - s);  // position in the padded array
                const double ang = 2.0 * qlgpu::kPI * (double)((long)k * z % NZ) / (double)NZ;
                re += f[2 * s] * std::cos(ang) - f[2 * s + 1] * std::sin(ang);
            }
            out[(size_t)m * NZ + z] = re / NZ;
        }
    }
    return append_bytes(tv->dir + "mean_fields.dat", out.data(), out.size() * sizeof(double))
               ? QLGPU_OK
               : io_fail(QLGPU_ERR_ARG, "write failed in " + tv->dir);
}

int qlgpu_timevars_close(qlgpu_timevars_t* tv) {
    delete tv;
    return QLGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// FullSave_Load container
// ---------------------------------------------------------------------------
namespace {

struct Reader {
    FILE* f = nullptr;
    bool ok = true;
    template <class T>
    T get() {
        T v{};
        if (ok && std::fread(&v, sizeof(T), 1, f) != 1) ok = false;
        return v;
    }
    std::string str() {
        const uint32_t n = get<uint32_t>();
        if (!ok || n > (1u << 20)) {
            ok = false;
            return std::string();
        }
        std::string s(n, '\0');
        if (n && std::fread(&s[0], 1, n, f) != n) ok = false;
        return s;
    }
    bool skip(uint64_t bytes) { return ok && std::fseek(f, (long)bytes, SEEK_CUR) == 0; }
};

struct Writer {
    std::vector<unsigned char> buf;
    template <class T>
    void put(const T& v) {
        const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
        buf.insert(buf.end(), p, p + sizeof(T));
    }
    void str(const std::string& s) {
        put<uint32_t>((uint32_t)s.size());
        buf.insert(buf.end(), s.begin(), s.end());
    }
    void bytes(const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        buf.insert(buf.end(), c, c + n);
    }
};

struct Dims {
    int nlin = 4, nz = 0, nmf = 0, nxy = 0;
};

Dims dims_of(const qlgpu_params& p) {
    Dims d;
    d.nz = qlgpu::stored_nz(p.NZ);
    d.nmf = qlgpu::mean_field_count(p);
    d.nxy = qlgpu::mode_count(p);
    return d;
}

// Reads the file header; when `want` is given, checks the dimensions against it.
bool read_header(Reader& r, const Dims* want, std::string* err) {
    char m[8];
    if (std::fread(m, 1, 8, r.f) != 8 || std::memcmp(m, kMagic, 8) != 0) {
        *err = "not a QLFSAVE1 file";
        return false;
    }
    const int32_t nlin = r.get<int32_t>(), nz = r.get<int32_t>(), nmf = r.get<int32_t>(), nxy = r.get<int32_t>();
    if (!r.ok) {
        *err = "truncated header";
        return false;
    }
    if (want && (nlin != want->nlin || nz != want->nz || nmf != want->nmf || nxy != want->nxy)) {
        *err = "file dimensions (nlin, nz, nmf, nxy) = (" + std::to_string(nlin) + ", " + std::to_string(nz) + ", " +
               std::to_string(nmf) + ", " + std::to_string(nxy) + ") do not match the parameters";
        return false;
    }
    return true;
}

// Scan the groups: their times and file offsets.
bool scan_groups(const char* path, const Dims* d, std::vector<double>* times, std::vector<long>* offs,
                 std::string* err) {
    Reader r;
    r.f = std::fopen(path, "rb");
    if (!r.f) {
        *err = std::string("cannot open ") + path;
        return false;
    }
    bool ok = read_header(r, d, err);
    while (ok) {
        const long at = std::ftell(r.f);
        const uint32_t peek = r.get<uint32_t>();
        if (!r.ok) break;  // clean end of file
        if (peek > (1u << 20)) {
            *err = "corrupt group header";
            ok = false;
            break;
        }
        std::fseek(r.f, at, SEEK_SET);
        const std::string name = r.str();
        const double t = r.get<double>();
        const uint32_t nds = r.get<uint32_t>();
        for (uint32_t i = 0; i < nds && r.ok; ++i) {
            (void)r.str();
            const uint32_t type = r.get<uint32_t>();
            const uint64_t count = r.get<uint64_t>();
            r.skip(count * (type == 0 ? 8 : 4));
        }
        if (!r.ok) {
            *err = "truncated group " + name;
            ok = false;
            break;
        }
        times->push_back(t);
        offs->push_back(at);
    }
    std::fclose(r.f);
    return ok;
}

}  // namespace

extern "C" {

// SaveSolution (FullSave_Load.cpp:176-257)
int qlgpu_fullsave_write(const char* path, const qlgpu_params* p, double t, const double* lin, const double* mf,
                         const double* kx0) {
    if (!path || !p || !lin || !mf || !kx0) return io_fail(QLGPU_ERR_ARG, "null argument");
    const Dims d = dims_of(*p);
    std::vector<double> kx, ky;
    std::vector<int> kxi, kyi;
    qlgpu::ktables(*p, kx, ky, kxi, kyi);
    Writer w;
    bool fresh = false;
    {
        FILE* f = std::fopen(path, "rb");
        if (!f) {
            fresh = true;
        } else {
            Reader r;
            r.f = f;
            std::string err;
            const bool ok = read_header(r, &d, &err);
            std::fclose(f);
            if (!ok) return io_fail(QLGPU_ERR_ARG, err);
        }
    }
    if (fresh) {
        w.bytes(kMagic, 8);
        w.put<int32_t>(d.nlin);
        w.put<int32_t>(d.nz);
        w.put<int32_t>(d.nmf);
        w.put<int32_t>(d.nxy);
    }
    char gname[64];
    std::snprintf(gname, sizeof(gname), "/t=%.15g", t);
    w.str(gname);
    w.put<double>(t);
    w.put<uint32_t>((uint32_t)(d.nxy + 2));
    std::vector<float> buf;
    for (int j = 0; j < d.nxy; ++j) {
        char dn[96];
        std::snprintf(dn, sizeof(dn), "Ind %d: kx %d ky %d", j, kxi[j], kyi[j]);
        w.str(dn);
        w.put<uint32_t>(0);
        w.put<uint64_t>((uint64_t)d.nlin * d.nz);
        buf.resize((size_t)2 * d.nlin * d.nz);
        const double* src = lin + (size_t)j * d.nlin * d.nz * 2;
        for (size_t i = 0; i < buf.size(); ++i) buf[i] = (float)src[i];
        w.bytes(buf.data(), buf.size() * sizeof(float));
    }
    w.str("Mean");
    w.put<uint32_t>(0);
    w.put<uint64_t>((uint64_t)d.nmf * d.nz);
    buf.resize((size_t)2 * d.nmf * d.nz);
    for (size_t i = 0; i < buf.size(); ++i) buf[i] = (float)mf[i];
    w.bytes(buf.data(), buf.size() * sizeof(float));
    w.str("kx");
    w.put<uint32_t>(1);
    w.put<uint64_t>((uint64_t)d.nxy);
    buf.resize((size_t)d.nxy);
    for (int j = 0; j < d.nxy; ++j) buf[j] = (float)(kx0[j] + p->q * t * ky[j]);  // FullSave_Load.cpp:232
    w.bytes(buf.data(), buf.size() * sizeof(float));
    FILE* f = std::fopen(path, "ab");
    if (!f) return io_fail(QLGPU_ERR_ARG, std::string("cannot open ") + path);
    const bool ok = std::fwrite(w.buf.data(), 1, w.buf.size(), f) == w.buf.size();
    if (std::fclose(f) != 0 || !ok) return io_fail(QLGPU_ERR_ARG, std::string("write failed: ") + path);
    return QLGPU_OK;
}

int qlgpu_fullsave_times(const char* path, double* times, int max_times, int* ngroups) {
    if (!path || !ngroups) return io_fail(QLGPU_ERR_ARG, "null argument");
    std::vector<double> ts;
    std::vector<long> offs;
    std::string err;
    if (!scan_groups(path, nullptr, &ts, &offs, &err)) return io_fail(QLGPU_ERR_ARG, err);
    *ngroups = (int)ts.size();
    if (times)
        for (int i = 0; i < (int)ts.size() && i < max_times; ++i) times[i] = ts[i];
    return QLGPU_OK;
}

// LoadSolution_forRestart (FullSave_Load.cpp:265-329): the latest group.
int qlgpu_fullsave_read_latest(const char* path, const qlgpu_params* p, double* t, double* lin, double* mf,
                               double* kx0) {
    if (!path || !p) return io_fail(QLGPU_ERR_ARG, "null argument");
    const Dims d = dims_of(*p);
    std::vector<double> times;
    std::vector<long> offs;
    std::string err;
    if (!scan_groups(path, &d, &times, &offs, &err)) return io_fail(QLGPU_ERR_ARG, err);
    if (times.empty()) return io_fail(QLGPU_ERR_ARG, std::string("no saved groups in ") + path);
    size_t best = 0;
    for (size_t i = 1; i < times.size(); ++i)
        if (times[i] > times[best]) best = i;
    const double tmax = times[best];
    std::vector<double> kx, ky;
    std::vector<int> kxi, kyi;
    qlgpu::ktables(*p, kx, ky, kxi, kyi);
    Reader r;
    r.f = std::fopen(path, "rb");
    if (!r.f) return io_fail(QLGPU_ERR_ARG, std::string("cannot open ") + path);
    std::fseek(r.f, 0, SEEK_END);
    const long fsize = std::ftell(r.f);
    std::fseek(r.f, offs[best], SEEK_SET);
    (void)r.str();
    (void)r.get<double>();
    const uint32_t nds = r.get<uint32_t>();
    bool have_kx = false, have_mean = false;
    std::vector<char> seen((size_t)d.nxy, 0);
    std::vector<float> buf;
    for (uint32_t i = 0; i < nds && r.ok; ++i) {
        const std::string name = r.str();
        const uint32_t type = r.get<uint32_t>();
        const uint64_t count = r.get<uint64_t>();
        if (!r.ok) break;
        // the sizes come from the file: check them against what is left of it before any allocation
        const long pos = std::ftell(r.f);
        const uint64_t left = (pos >= 0 && fsize >= pos) ? (uint64_t)(fsize - pos) / sizeof(float) : 0;
        if (type > 1 || count > left / (type == 0 ? 2 : 1)) {
            std::fclose(r.f);
            return io_fail(QLGPU_ERR_ARG, "dataset " + name + " has an invalid type or size (corrupt file)");
        }
        const size_t nfl = (size_t)count * (type == 0 ? 2 : 1);
        try {
            buf.resize(nfl);
        } catch (...) {
            std::fclose(r.f);
            return io_fail(QLGPU_ERR_ARG, "dataset " + name + " is too large");
        }
        if (nfl && std::fread(buf.data(), sizeof(float), nfl, r.f) != nfl) {
            r.ok = false;
            break;
        }
        int jj = -1, a = 0, b = 0;
        if (std::sscanf(name.c_str(), "Ind %d: kx %d ky %d", &jj, &a, &b) == 3) {
            if (jj < 0 || jj >= d.nxy || type != 0 || count != (uint64_t)d.nlin * d.nz || a != kxi[jj] ||
                b != kyi[jj]) {
                std::fclose(r.f);
                return io_fail(QLGPU_ERR_ARG, "dataset " + name + " does not match the parameters");
            }
            seen[jj] = 1;
            if (lin)
                for (size_t k = 0; k < nfl; ++k) lin[(size_t)jj * d.nlin * d.nz * 2 + k] = (double)buf[k];
        } else if (name == "Mean") {
            if (type != 0 || count != (uint64_t)d.nmf * d.nz) {
                std::fclose(r.f);
                return io_fail(QLGPU_ERR_ARG, "dataset Mean does not match the parameters");
            }
            have_mean = true;
            if (mf)
                for (size_t k = 0; k < nfl; ++k) mf[k] = (double)buf[k];
        } else if (name == "kx") {
            if (type != 1 || count != (uint64_t)d.nxy) {
                std::fclose(r.f);
                return io_fail(QLGPU_ERR_ARG, "dataset kx does not match the parameters");
            }
            have_kx = true;
            // kx0 = kx(t) - q t_start ky (FullSave_Load.cpp:317-320)
            if (kx0)
                for (int j = 0; j < d.nxy; ++j) kx0[j] = (double)buf[j] - p->q * tmax * ky[j];
        }
    }
    std::fclose(r.f);
    if (!r.ok) return io_fail(QLGPU_ERR_ARG, std::string("truncated file ") + path);
    // every mode and the mean fields must be in the group (FullSave_Load.cpp:286-316 reads them all)
    for (int j = 0; j < d.nxy; ++j)
        if (!seen[j]) return io_fail(QLGPU_ERR_ARG, "group lacks dataset Ind " + std::to_string(j));
    if (!have_mean) return io_fail(QLGPU_ERR_ARG, "group lacks dataset Mean");
    // no kx dataset: kx as initialised (FullSave_Load.cpp:322-324)
    if (!have_kx && kx0)
        for (int j = 0; j < d.nxy; ++j) kx0[j] = kx[j];
    if (t) *t = tmax;
    return QLGPU_OK;
}

}  // extern "C"
