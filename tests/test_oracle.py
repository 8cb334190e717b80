"""The CPU oracle against numpy.fft, an independent numpy restatement, physics
pins and the committed golden fixtures.  No GPU needed."""
import numpy as np
import pytest

from oracle import oracle as O
from numpy_ref import NumpyQL
from ql_dns_b200.initial import initial_state
from ql_dns_b200.ktables import ktables
from ql_dns_b200.params import QLParams, mri_16x16_nz32


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("N", [8, 12, 16, 32, 64, 128, 256])
def test_fft_convention_matches_numpy(N):
    # fftwPlans.cpp:48-51: FFTW_FORWARD = exp(-2 pi i jk/N), unnormalised both ways
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    assert np.abs(O.fft(x, True) - np.fft.fft(x)).max() < 1e-13 * N
    assert np.abs(O.fft(x, False) - np.fft.ifft(x) * N).max() < 1e-13 * N


def small(model, integ, **kw):
    base = dict(nx=8, ny=8, NZ=16, model=model, integrator=integ,
                B0z=0.02 if model == 1 else 0.0, omega=1.0)
    base.update(kw)
    return mri_16x16_nz32(**base)


@pytest.mark.parametrize("model", [0, 1])
@pytest.mark.parametrize("integ", [0, 1])
def test_oracle_matches_numpy_restatement(model, integ):
    p = small(model, integ)
    lin, mf, kx0 = initial_state(p, 3, sigma=0.3, mean_u=0.03)
    R = NumpyQL(p)
    F, Fm, L = R.rhs(0.37, 0.002, lin, mf, kx0)
    F2, Fm2, L2 = O.rhs(p, 0.37, 0.002, lin, mf, kx0)
    assert rel(F2, F) < 1e-13 and rel(Fm2, Fm) < 1e-12 and rel(L2, L) < 1e-15
    l1, m1, _ = R.step(0.1, lin, mf, kx0)
    _, l2, m2, _, _ = O.run(p, 0.1, lin, mf, kx0, 1)
    assert rel(l2, l1) < 1e-13 and rel(m2, m1) < 1e-13
    d1 = R.diagnostics(0.3, lin, mf, kx0)
    d2 = O.diagnostics(p, 0.3, lin, mf, kx0)[:12]
    assert rel(d2, d1) < 1e-13


@pytest.mark.parametrize("integ", [0, 1])
@pytest.mark.parametrize("nu", [0.0, 1e-3])
def test_alfven_wave_exact_solution(integ, nu):
    # q=0 (so Omega=2q/3=0), uniform By=B0, nu=eta: every mode is an Alfven wave
    # u(t) = e^{nu lapF t}(cos(w t) u0 + i sin(w t) b0), w = ky B0.
    # Without diffusion both integrators are third order (Matlab/IntegratorTests.m:44).
    # With diffusion the reference's integrating factor exp(dt(a+b)L) is applied to
    # the previous-stage rhs as well (RK3CN_Elin.cpp:134-136), which makes the
    # exponential variant first order; the CN variant (RK3CN.cpp:105-107) drops to
    # between second and third.  The oracle reproduces both behaviours.
    B0 = 0.7
    nuv = nu if nu > 0 else 1e-300
    p = mri_16x16_nz32(nx=8, ny=8, NZ=16, q=0.0, nu=nuv, eta=nuv, quasilinear=0, remap=0, integrator=integ)
    lin, mf, kx0 = initial_state(p, 5, sigma=1.0)
    mf[:] = 0
    mf[1, 0] = B0 * p.NZ
    R = NumpyQL(p)
    T = 0.5
    errs = []
    for dt in (0.02, 0.01, 0.005):
        n = int(round(T / dt))
        _, l2, _, _, _ = O.run(p.replace(dt=dt), 0.0, lin, mf, kx0, n)
        w = R.ky[:, None] * B0
        lapF = (-R.kx0 ** 2)[:, None] + R.lap2
        dec = np.exp(nu * lapF * T)
        ex = np.empty_like(lin)
        for (a, c) in ((0, 2), (1, 3)):
            ex[:, a] = dec * (np.cos(w * T) * lin[:, a] + 1j * np.sin(w * T) * lin[:, c])
            ex[:, c] = dec * (1j * np.sin(w * T) * lin[:, a] + np.cos(w * T) * lin[:, c])
        errs.append(rel(l2, ex))
    r1, r2 = errs[0] / errs[1], errs[1] / errs[2]
    if nu == 0.0:
        assert 7.9 < r1 < 8.1 and 7.9 < r2 < 8.1, errs
    elif integ == 0:
        assert 1.9 < r1 < 2.1 and 1.9 < r2 < 2.1, errs
    else:
        assert 4.0 < r1 < 8.1 and 4.0 < r2 < 8.1, errs


def mri_growth(q, Om, vA, kz):
    kap2 = 2 * (2 - q) * Om ** 2
    a = kap2 + 2 * kz ** 2 * vA ** 2
    c = kz ** 2 * vA ** 2 * (kz ** 2 * vA ** 2 - 2 * q * Om ** 2)
    s2 = (-a + np.sqrt(a * a - 4 * c)) / 2
    return np.sqrt(s2)


def test_channel_mri_growth_rate_fullqlin():
    # Mean fields of MHD_FullQlin with a vertical field B0z and no fluctuations
    # obey the ideal axisymmetric MRI (MHD_FullQlin.cpp:411-417).
    vA = 0.15
    p = mri_16x16_nz32(nx=4, ny=4, NZ=16, model=1, B0z=vA, nu=0.0, eta=0.0, dt=0.005, omega=1.0, remap=0)
    lin = np.zeros((p.nxy, 4, p.nz), complex)
    mf = np.zeros((4, p.nz), complex)
    mf[0, 1] = 1e-6 * p.NZ
    mf[0, -1] = 1e-6 * p.NZ
    kx0 = ktables(p)["kx"]
    t, _, m1, _, d = O.run(p, 0.0, lin, mf, kx0, 1200, diag_every=200)
    e = d[:, 2] + d[:, 1]  # mean field energies MU + MB
    rate = 0.5 * np.log(e[-1] / e[-2]) / (d[-1, 0] - d[-2, 0])
    expect = mri_growth(1.5, 1.0, vA, 2 * np.pi)
    assert abs(rate - expect) / expect < 1e-3, (rate, expect)


def test_remap_zeroes_mode_at_predicted_step():
    # MHD_BQlin.cpp:314-331: a mode is zeroed (and its kx shifted by -(Nx-1)kxL)
    # right after the step at which kx0 + q t ky first exceeds (Nx-1)/2 kxL.
    p = mri_16x16_nz32(nx=8, ny=8, NZ=16, dt=0.05)
    lin, mf, kx0 = initial_state(p, 2, sigma=0.1)
    kxL = 2 * np.pi / p.L[0]
    ky = NumpyQL(p).ky
    t = 0.0
    state = (lin, mf, kx0)
    for n in range(40):
        t_before = t
        t, l2, m2, k2, _ = O.run(p, t, *state, 1)
        newly = (k2 != state[2])
        pred = (state[2] + p.q * t * ky > (p.nx - 1) / 2 * kxL)
        assert np.array_equal(newly, pred)
        if newly.any():
            assert np.all(l2[newly] == 0)
            assert np.allclose(k2[newly], state[2][newly] - (p.nx - 1) * kxL)
        state = (l2, m2, k2)


def test_energy_conservation_ideal():
    # nu=eta=0, q=0, static uniform field, QuasiLinear off: fluctuation energy is
    # conserved up to the RK3 truncation error, which falls ~8x per halving of dt.
    p = mri_16x16_nz32(nx=8, ny=8, NZ=16, q=0.0, nu=1e-300, eta=1e-300, quasilinear=0, remap=0)
    lin, mf, kx0 = initial_state(p, 7, sigma=1.0)
    mf[:] = 0
    mf[1, 0] = 0.5 * p.NZ
    errs = []
    for dt in (0.02, 0.01):
        n = int(round(1.0 / dt))
        _, _, _, _, d = O.run(p.replace(dt=dt), 0.0, lin, mf, kx0, n, diag_every=n)
        e0 = d[0, 3] + d[0, 4]
        e1 = d[-1, 3] + d[-1, 4]
        errs.append(abs(e1 - e0) / e0)
    assert errs[0] < 1e-5 and errs[0] / errs[1] > 7.0, errs


from golden_cases import load, names  # noqa: E402
from ql_dns_b200.initial import initial_state as _ic  # noqa: E402


@pytest.mark.parametrize("name", names())
def test_oracle_reproduces_golden(name):
    p, g = load(name)
    lin, mf, kx0 = _ic(p, int(g["seed"]), sigma=float(g["sigma"]), mean_u=float(g["mean_u"]))
    # the seeded initial-condition law is itself pinned by the fixture
    assert np.array_equal(lin, g["lin0"]) and np.array_equal(mf, g["mf0"]) and np.array_equal(kx0, g["kx00"])
    t, lo, mo, ko, d = O.run(p, 0.0, lin, mf, kx0, int(g["nsteps"]), diag_every=1)
    assert t == g["t"]
    assert rel(lo, g["lin"]) < 1e-13 and rel(mo, g["mf"]) < 1e-13
    assert np.array_equal(ko, g["kx0"])
    assert rel(d[:, 1:13], g["diag"][:, 1:13]) < 1e-12
