"""Driving noise (qlgpu_set_noise) and the CFL time step (qlgpu_set_cfl) on the
GPU against the oracle's forced main loop (oracle_run_forced), through the C ABI.

Both draw the same Philox4x32-10 numbers, so the bar is the parity bar of the
plain step: relative L2 <= 1e-10 for the state and the diagnostic series, the
time and Integrator::mean_time_step to round-off.
"""
import numpy as np
import pytest

from gpu_util import rel, require_gpu
from oracle import oracle as O
from ql_dns_b200.initial import initial_state
from ql_dns_b200.params import QLParams
from ql_dns_b200.solver import QLSolver

pytestmark = pytest.mark.gpu
TOL = 1e-10


def series_rel(dg, do):
    errs = []
    for c in range(1, 13):
        scale = np.abs(do[:, c]).max()
        if scale > 0:
            errs.append(np.abs(dg[:, c] - do[:, c]).max() / scale)
    return max(errs)


def run_gpu(p, st, n, diag_every, noise=None, cfl=None):
    require_gpu()
    with QLSolver(p) as s:
        s.set_state(0.0, *st)
        if noise:
            s.set_noise(*noise)
        if cfl:
            s.set_cfl(*cfl)
        d = s.step(n, diag_every=diag_every)
        t, lo, mo, ko = s.get_state()
        return t, lo, mo, ko, d, s.mean_time_step()


@pytest.mark.parametrize("integ", [0, 1])
def test_noise_matches_oracle(integ):
    p = QLParams(nx=16, ny=16, NZ=32, dt=0.02, integrator=integ)
    st = initial_state(p, 4, sigma=1e-3)
    n, noise = 40, (0.05, 1.0, 30.0, 1234)
    t, lo, mo, ko, d, dtm = run_gpu(p, st, n, 4, noise=noise)
    t2, lo2, mo2, ko2, d2, dtm2 = O.run_forced(p, 0.0, *st, n, diag_every=4, f_noise=noise[0], k_lo=noise[1],
                                              k_hi=noise[2], seed=noise[3])
    assert not np.array_equal(ko2, st[2])  # remaps happened
    assert t == t2 and np.array_equal(ko, ko2) and dtm == dtm2
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (rel(lo, lo2), rel(mo, mo2))
    # the initial record is the oracle's first row
    assert d.shape[0] == d2.shape[0] - 1 and series_rel(d, d2[1:]) < TOL
    # the noise is visible: without it the state differs at O(1)
    t3, lo3, *_ = O.run(p, 0.0, *st, n)
    assert rel(lo3, lo2) > 1e-2


@pytest.mark.parametrize("model", [0, 1])
def test_cfl_matches_oracle(model):
    p = QLParams(model=model, nx=16, ny=16, NZ=64, dt=0.01, B0z=0.01 if model else 0.0, omega=1.0)
    st = initial_state(p, 5, sigma=0.05, B0=0.2, mean_u=0.05 if model else 0.0)
    n, cfl = 30, (0.3, 0.02)
    t, lo, mo, ko, d, dtm = run_gpu(p, st, n, 5, cfl=cfl)
    t2, lo2, mo2, ko2, d2, dtm2 = O.run_forced(p, 0.0, *st, n, diag_every=5, cfl=cfl[0], dt_max=cfl[1])
    assert dtm2 < cfl[1]  # the CFL limit is active
    assert abs(t - t2) <= 1e-13 * t2 and abs(dtm - dtm2) <= 1e-13 * dtm2
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (rel(lo, lo2), rel(mo, mo2))
    assert series_rel(d, d2[1:]) < TOL


def test_noise_and_cfl_together_and_off_again():
    p = QLParams(nx=16, ny=16, NZ=32, dt=0.02)
    st = initial_state(p, 6, sigma=1e-3, B0=0.1)
    n = 25
    require_gpu()
    with QLSolver(p) as s:
        s.set_state(0.0, *st)
        s.set_noise(0.02, 0.5, 50.0, 7)
        s.set_cfl(0.4, 0.03)
        s.step(n)
        t, lo, mo, ko = s.get_state()
        s.set_noise(0.0, 0.0, 0.0)
        s.set_cfl(0.0)
        s.set_state(0.0, *st)
        s.step(10)
        t4, lo4, mo4, ko4 = s.get_state()
    t2, lo2, mo2, ko2, _, _ = O.run_forced(p, 0.0, *st, n, cfl=0.4, dt_max=0.03, f_noise=0.02, k_lo=0.5, k_hi=50.0,
                                           seed=7)
    assert abs(t - t2) <= 1e-13 * t2 and rel(lo, lo2) < TOL and rel(mo, mo2) < TOL
    t5, lo5, mo5, ko5, _ = O.run(p, 0.0, *st, 10)
    assert t4 == t5 and rel(lo4, lo5) < TOL


@pytest.mark.parametrize("integ", [0, 1])
@pytest.mark.parametrize("only", [None, "velocity", "magnetic"])
def test_fullqlin_noise_matches_oracle(integ, only):
    # MHD_FullQlin::DrivingNoise with its ky = 0 conjugate pairs (MHD_FullQlin.cpp:786-1045)
    # and the drive_only_* switches (:21-22)
    p = QLParams(model=1, integrator=integ, nx=16, ny=16, NZ=32, dt=0.02, B0z=0.01, omega=1.0)
    st = initial_state(p, 8, sigma=1e-3, B0=0.05, mean_u=0.01)
    n, noise = 30, (0.05, 0.5, 40.0, 4321)
    kw = dict(drive_only_velocity=only == "velocity", drive_only_magnetic=only == "magnetic")
    require_gpu()
    with QLSolver(p) as s:
        s.set_state(0.0, *st)
        s.set_noise(*noise, **kw)
        d = s.step(n, diag_every=5)
        t, lo, mo, ko = s.get_state()
    t2, lo2, mo2, ko2, d2, _ = O.run_forced(p, 0.0, *st, n, diag_every=5, f_noise=noise[0], k_lo=noise[1],
                                            k_hi=noise[2], seed=noise[3], **kw)
    assert t == t2 and np.array_equal(ko, ko2)
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (rel(lo, lo2), rel(mo, mo2))
    assert series_rel(d, d2[1:]) < TOL
    t3, lo3, *_ = O.run(p, 0.0, *st, n)
    assert rel(lo3, lo2) > 1e-2


def test_drive_only_switches_refused_for_bqlin():
    from ql_dns_b200._capi import QLGPUError
    require_gpu()
    with QLSolver(QLParams(model=0, nx=8, ny=8, NZ=32)) as s:
        s.set_noise(0.1, 1.0, 10.0)
        with pytest.raises(QLGPUError) as ei:
            s.set_noise(0.1, 1.0, 10.0, drive_only_velocity=True)
        assert ei.value.code == 2
