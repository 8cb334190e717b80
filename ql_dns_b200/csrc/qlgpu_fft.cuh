// qlgpu_fft.cuh -- FP64 z-transforms for one (kx,ky) column, held by a group
// of T threads with P = NZ/T points each (sm_100a).
//
// Conventions follow FFTW as used by the reference (QL_DNS/Auxiliary/
// fftwPlans.cpp:48-51): backward = exp(+2 pi i jk/N), forward =
// exp(-2 pi i jk/N), both unnormalised.
//
// Layouts (N = P*T, thread t = lane % T inside its group):
//   spectral  : thread t holds X[t + T*k2],            k2 = 0..P-1  (reg k2)
//   real space: thread t holds x[P*n1 + t + T*m],      m < P/T, n1 < T
//               in register j = m*T + n1.
// The inverse transform maps spectral -> real space and the forward transform
// maps real space -> spectral with no permutation, so pointwise products in
// real space need no reordering.  Each transform is one register DFT of size
// P, a twiddle, one padded shared-memory transpose among the T threads of the
// group and P/T register DFTs of size T.
#pragma once
#include <cuda_runtime.h>

namespace qlgpu {

struct __align__(16) cplx {
    double x, y;
};

__device__ __forceinline__ cplx mk(double a, double b) { cplx r; r.x = a; r.y = b; return r; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ cplx cscale(cplx a, double s) { return mk(a.x * s, a.y * s); }
// multiply by +i (DIR>0) or -i (DIR<0)
template <int DIR>
__device__ __forceinline__ cplx mul_i(cplx a) {
    return DIR > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}
__device__ __forceinline__ cplx conjc(cplx a) { return mk(a.x, -a.y); }

// ---------------------------------------------------------------------------
// In-register DFTs, natural order in and out.  DIR = +1 backward, -1 forward.
// ---------------------------------------------------------------------------
template <int DIR>
__device__ __forceinline__ void dft2(cplx& a, cplx& b) {
    cplx t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR>
__device__ __forceinline__ void dft4(cplx& x0, cplx& x1, cplx& x2, cplx& x3) {
    cplx y0 = cadd(x0, x2), y1 = csub(x0, x2);
    cplx y2 = cadd(x1, x3), y3 = mul_i<DIR>(csub(x1, x3));
    x0 = cadd(y0, y2);
    x2 = csub(y0, y2);
    x1 = cadd(y1, y3);
    x3 = csub(y1, y3);
}

// (1 + DIR i)/sqrt(2) * a  and (-1 + DIR i)/sqrt(2) * a
#define QLGPU_RSQRT2 0.70710678118654752440
template <int DIR>
__device__ __forceinline__ cplx w8_1(cplx a) {
    // (a.x + i a.y)(1 + D i)/sqrt2 = (a.x - D a.y, a.y + D a.x)/sqrt2
    return DIR > 0 ? mk((a.x - a.y) * QLGPU_RSQRT2, (a.y + a.x) * QLGPU_RSQRT2)
                   : mk((a.x + a.y) * QLGPU_RSQRT2, (a.y - a.x) * QLGPU_RSQRT2);
}
template <int DIR>
__device__ __forceinline__ cplx w8_3(cplx a) {
    // (a.x + i a.y)(-1 + D i)/sqrt2 = (-a.x - D a.y, -a.y + D a.x)/sqrt2
    return DIR > 0 ? mk((-a.x - a.y) * QLGPU_RSQRT2, (a.x - a.y) * QLGPU_RSQRT2)
                   : mk((a.y - a.x) * QLGPU_RSQRT2, (-a.y - a.x) * QLGPU_RSQRT2);
}

template <int DIR>
__device__ __forceinline__ void dft8(cplx* x) {
    cplx e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
    cplx o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
    dft4<DIR>(e0, e1, e2, e3);
    dft4<DIR>(o0, o1, o2, o3);
    o1 = w8_1<DIR>(o1);
    o2 = mul_i<DIR>(o2);
    o3 = w8_3<DIR>(o3);
    x[0] = cadd(e0, o0); x[4] = csub(e0, o0);
    x[1] = cadd(e1, o1); x[5] = csub(e1, o1);
    x[2] = cadd(e2, o2); x[6] = csub(e2, o2);
    x[3] = cadd(e3, o3); x[7] = csub(e3, o3);
}

// cos/sin(2 pi k/16), k = 1..3
#define QLGPU_C1 0.92387953251128675613
#define QLGPU_S1 0.38268343236508977173
template <int DIR>
__device__ __forceinline__ void dft16(cplx* x) {
    cplx e[8], o[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) { e[i] = x[2 * i]; o[i] = x[2 * i + 1]; }
    dft8<DIR>(e);
    dft8<DIR>(o);
    // o[k] *= exp(DIR 2 pi i k/16)
    const double D = (double)DIR;
    o[1] = cmul(o[1], mk(QLGPU_C1, D * QLGPU_S1));
    o[2] = w8_1<DIR>(o[2]);
    o[3] = cmul(o[3], mk(QLGPU_S1, D * QLGPU_C1));
    o[4] = mul_i<DIR>(o[4]);
    o[5] = cmul(o[5], mk(-QLGPU_S1, D * QLGPU_C1));
    o[6] = w8_3<DIR>(o[6]);
    o[7] = cmul(o[7], mk(-QLGPU_C1, D * QLGPU_S1));
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = cadd(e[k], o[k]);
        x[k + 8] = csub(e[k], o[k]);
    }
}

template <int M, int DIR>
__device__ __forceinline__ void dft(cplx* x) {
    if constexpr (M == 1) {
    } else if constexpr (M == 2) {
        dft2<DIR>(x[0], x[1]);
    } else if constexpr (M == 4) {
        dft4<DIR>(x[0], x[1], x[2], x[3]);
    } else if constexpr (M == 8) {
        dft8<DIR>(x);
    } else if constexpr (M == 16) {
        dft16<DIR>(x);
    } else {
        static_assert(M <= 16, "register DFT size");
    }
}

// ---------------------------------------------------------------------------
// Transform geometry for a z grid of NZ points
// ---------------------------------------------------------------------------
template <int NZ_>
struct Geom {
    static constexpr int NZ = NZ_;
    // threads per column and points per thread
    static constexpr int T = NZ_ >= 256 ? 16 : (NZ_ >= 64 ? 8 : 4);
    static constexpr int P = NZ_ / T;
    static constexpr int PT = P / T;  // register DFTs of size T per thread
    static_assert(P * T == NZ_ && PT * T == P, "NZ must be a power of two in [16, 256]");
    static constexpr int nz = 1 + 2 * (NZ_ / 3);  // Model.h:34 (NZ/3.0 truncated)
    static constexpr int H = (nz - 1) / 2;        // highest retained |kz| index
    // exchange buffer: P rows of T (+1 pad) complex; group stride chosen so two
    // 4-thread groups sharing a 128-byte phase hit disjoint banks.
    static constexpr int XROW = T + 1;
    static constexpr int XSIZE_RAW = P * XROW;
    static constexpr int XSIZE = (T == 4) ? (((XSIZE_RAW + 3) / 8) * 8 + 4) : XSIZE_RAW;
};

// spectral index k (0..NZ-1) -> stored dealiased index, or -1 when in the
// padding gap (fftwPlans.h:66-97)
template <class G>
__device__ __forceinline__ int stored_index(int k) {
    if (k <= G::H) return k;
    if (k >= G::NZ - G::H) return k - (G::NZ - G::nz);
    return -1;
}
// signed kz integer of spectral slot k (Kdata.cpp:74-78)
template <class G>
__device__ __forceinline__ int kz_int(int k) {
    return k <= G::H ? k : k - G::NZ;
}

// Twiddle table tw[n2*T + t] = exp(+2 pi i n2 t / NZ); forward uses the conjugate.
// Inverse: spectral regs (X[t+T k2]) -> real space regs.  xch = this group's
// exchange buffer (Geom::XSIZE complex); gmask = the lanes of this group.
template <class G>
__device__ __forceinline__ void inv_fft(cplx* x, cplx* xch, const cplx* tw, int t, unsigned gmask) {
    dft<G::P, +1>(x);
#pragma unroll
    for (int n2 = 0; n2 < G::P; ++n2) {
        if (n2 != 0) x[n2] = cmul(x[n2], tw[n2 * G::T + t]);
        xch[n2 * G::XROW + t] = x[n2];
    }
    __syncwarp(gmask);
#pragma unroll
    for (int m = 0; m < G::PT; ++m) {
        const int n2 = t + G::T * m;
#pragma unroll
        for (int k1 = 0; k1 < G::T; ++k1) x[m * G::T + k1] = xch[n2 * G::XROW + k1];
        dft<G::T, +1>(x + m * G::T);
    }
    __syncwarp(gmask);
}

// Forward: real-space regs -> spectral regs (X[t + T k2] in reg k2)
template <class G>
__device__ __forceinline__ void fwd_fft(cplx* x, cplx* xch, const cplx* tw, int t, unsigned gmask) {
#pragma unroll
    for (int m = 0; m < G::PT; ++m) {
        const int n2 = t + G::T * m;
        dft<G::T, -1>(x + m * G::T);
#pragma unroll
        for (int k1 = 0; k1 < G::T; ++k1) xch[n2 * G::XROW + k1] = x[m * G::T + k1];
    }
    __syncwarp(gmask);
#pragma unroll
    for (int n2 = 0; n2 < G::P; ++n2) {
        x[n2] = xch[n2 * G::XROW + t];
        if (n2 != 0) x[n2] = cmul(x[n2], conjc(tw[n2 * G::T + t]));
    }
    __syncwarp(gmask);
    dft<G::P, -1>(x);
}

// z coordinate of real-space register j of thread t
template <class G>
__device__ __forceinline__ int zpos(int t, int j) {
    const int m = j / G::T, n1 = j % G::T;
    return G::P * n1 + t + G::T * m;
}

}  // namespace qlgpu
