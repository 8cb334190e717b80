"""Parity of the sm_100a step (through the C ABI) with the CPU oracle.

Tolerance: relative L2 error <= 1e-10 for the state after N steps and for the
energy / stress / dissipation series (the bar stated for this path).  The
oracle is the strict FP64 build of oracle/ql_oracle.cpp.
"""
import numpy as np
import pytest

from gpu_util import rel, require_gpu
from golden_cases import load, names
from oracle import oracle as O
from ql_dns_b200.initial import initial_state
from ql_dns_b200.params import mri_16x16_nz32, mri_64x64_nz128
from ql_dns_b200.solver import QLSolver

pytestmark = pytest.mark.gpu
TOL = 1e-10


def run_gpu(p, lin, mf, kx0, n, diag_every=1, t0=0.0):
    require_gpu()
    with QLSolver(p) as s:
        s.set_state(t0, lin, mf, kx0)
        d0 = s.diagnostics()
        d = s.step(n, diag_every=diag_every)
        t, lo, mo, ko = s.get_state()
    return t, lo, mo, ko, np.vstack([d0[None], d]) if diag_every else d


def series_rel(dg, do):
    # every column of the 12 diagnostics, relative to its own scale
    errs = []
    for c in range(1, 13):
        scale = np.abs(do[:, c]).max()
        if scale > 0:
            errs.append(np.abs(dg[:, c] - do[:, c]).max() / scale)
    return max(errs)


@pytest.mark.parametrize("name", names())
def test_golden_fixture(name):
    p, g = load(name)
    n = int(g["nsteps"])
    t, lo, mo, ko, d = run_gpu(p, g["lin0"], g["mf0"], g["kx00"], n)
    assert t == g["t"]
    assert np.array_equal(ko, g["kx0"]), "remap decisions differ"
    assert rel(lo, g["lin"]) < TOL
    assert rel(mo, g["mf"]) < TOL
    assert d.shape == g["diag"].shape
    assert np.array_equal(d[:, 0], g["diag"][:, 0])
    assert series_rel(d, g["diag"]) < TOL


@pytest.mark.parametrize("model", [0, 1])
@pytest.mark.parametrize("integ", [0, 1])
def test_rhs_matches_oracle(model, integ):
    require_gpu()
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32, integrator=integ, model=model, B0z=0.03 if model else 0.0, omega=0.8)
    lin, mf, kx0 = initial_state(p, 21, sigma=0.5, mean_u=0.02)
    with QLSolver(p) as s:
        s.set_state(0.0, lin, mf, kx0)
        F, Fm, Lop = s.rhs(0.731, 0.0023, lin, mf)
    F2, Fm2, L2 = O.rhs(p, 0.731, 0.0023, lin, mf, kx0)
    assert rel(F, F2) < 1e-12
    assert rel(Fm, Fm2) < 1e-11
    assert rel(Lop, L2) < 1e-15


@pytest.mark.parametrize("model", [0, 1])
@pytest.mark.parametrize("NZ", [16, 32, 64, 128, 256])
def test_each_nz_three_steps(NZ, model):
    p = mri_16x16_nz32(nx=8, ny=6, NZ=NZ, model=model, B0z=0.02 if model else 0.0)
    lin, mf, kx0 = initial_state(p, NZ, sigma=0.3, mean_u=0.02)
    _, lo, mo, ko, d = run_gpu(p, lin, mf, kx0, 3)
    _, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 3, diag_every=1)
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL
    assert series_rel(d, d2) < TOL


@pytest.mark.parametrize("integ", [0, 1])
def test_mri_16x16_500_steps(integ):
    # 16x16 modes x NZ=32, Re=Rm=2000, dt=0.01, 500 steps, diagnostics every step
    p = mri_16x16_nz32(integrator=integ)
    lin, mf, kx0 = initial_state(p, 0, sigma=1e-3)
    t, lo, mo, ko, d = run_gpu(p, lin, mf, kx0, 500)
    t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 500, diag_every=1)
    assert t == t2 and np.array_equal(ko, ko2)
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL
    assert series_rel(d, d2) < TOL


def test_mri_16x16_strong_coupling_500_steps():
    # sigma = 0.1: the quasi-linear feedback changes the mean field by O(1)
    p = mri_16x16_nz32()
    lin, mf, kx0 = initial_state(p, 0, sigma=0.1)
    t, lo, mo, ko, d = run_gpu(p, lin, mf, kx0, 500)
    t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 500, diag_every=1)
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL
    assert series_rel(d, d2) < TOL


def test_mri_64x64_nz128_short():
    # production size 64x64 modes x NZ=128: 10 steps against the oracle
    p = mri_64x64_nz128()
    lin, mf, kx0 = initial_state(p, 1, sigma=1e-3)
    t, lo, mo, ko, d = run_gpu(p, lin, mf, kx0, 10)
    t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 10, diag_every=1)
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL
    assert series_rel(d, d2) < TOL


def test_deterministic_bitwise():
    p = mri_16x16_nz32(nx=16, ny=16, NZ=64)
    lin, mf, kx0 = initial_state(p, 4, sigma=0.2)
    a = run_gpu(p, lin, mf, kx0, 20)
    b = run_gpu(p, lin, mf, kx0, 20)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and np.array_equal(a[4], b[4])


def test_nonfinite_state_reports_status():
    from ql_dns_b200._capi import QLGPUError
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    lin, mf, kx0 = initial_state(p, 5, sigma=0.3)
    mf[1, 1] = np.nan
    require_gpu()
    with QLSolver(p) as s:
        s.set_state(0.0, lin, mf, kx0)
        with pytest.raises(QLGPUError) as ei:
            s.step(2)
        assert ei.value.code == 4
        assert s.status() & 1
        # the handle stays usable after resetting the state
        mf[1, 1] = 0.0
        s.set_state(0.0, lin, mf, kx0)
        s.step(1)
        assert s.status() == 0


@pytest.mark.parametrize("integ", [0, 1])
@pytest.mark.parametrize("order", [2, 4])
def test_fullqlin_200_steps(integ, order):
    # MHD_FullQlin with a vertical field, rotation, mean U and (order 4) hyper-dissipation
    p = mri_16x16_nz32(model=1, integrator=integ, B0z=0.05, omega=1.0, viscosity_order=order,
                nu=1e-4 if order == 4 else 1 / 2000, eta=2e-4 if order == 4 else 1 / 2000)
    lin, mf, kx0 = initial_state(p, 3, sigma=0.05, mean_u=0.02)
    t, lo, mo, ko, d = run_gpu(p, lin, mf, kx0, 200)
    t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 200, diag_every=1)
    assert t == t2 and np.array_equal(ko, ko2)
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL
    assert series_rel(d, d2) < TOL


@pytest.mark.parametrize("nx,ny", [(2, 2), (4, 2), (2, 4), (6, 10), (4, 18), (96, 6)])
@pytest.mark.parametrize("model", [0, 1])
def test_ragged_and_tiny_mode_grids(nx, ny, model):
    # a single column (the mean-field column only), ky = 0 only, kx = 0 only, mode counts
    # that are not multiples of the pairs per CTA, and many kx with few ky: the mode split
    # over CTAs and transform pairs has ragged tails
    p = mri_16x16_nz32(nx=nx, ny=ny, NZ=32, model=model, B0z=0.02 if model else 0.0, dt=0.02)
    lin, mf, kx0 = initial_state(p, nx * 10 + ny, sigma=0.3, mean_u=0.02)
    _, lo, mo, ko, d = run_gpu(p, lin, mf, kx0, 6)
    _, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 6, diag_every=1)
    assert np.array_equal(ko, ko2)
    assert (np.linalg.norm(lo2) == 0 and np.abs(lo).max() == 0) or rel(lo, lo2) < TOL
    assert rel(mo, mo2) < TOL
    assert series_rel(d, d2) < TOL


def test_odd_mode_counts_are_refused():
    # Kdata fills (nx/2) + (nx/2 - 1) kx values while Model::Dimxy counts nx - 1
    # (Kdata.cpp:29-46, Model.h:36): an odd nx would leave a column unset in the reference
    from ql_dns_b200._capi import QLGPUError
    require_gpu()
    for nx, ny in ((5, 8), (8, 7)):
        with pytest.raises(QLGPUError) as ei:
            QLSolver(mri_16x16_nz32(nx=nx, ny=ny))
        assert ei.value.code == 1 and "even" in str(ei.value)
