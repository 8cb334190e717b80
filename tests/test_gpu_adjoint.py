"""Discrete adjoint of the MHD_BQlin step with RK3CN_Elin and with RK3CN
(Crank-Nicolson) on the GPU (qlgpu_adjoint_maxwell) against the oracle's
tangent-linear model and central finite differences of the GPU forward run.

J = mean over N steps of the fluctuation Maxwell stress.  Bars: the adjoint
directional derivative Re <grad, d> agrees with the tangent-linear dJ to 1e-8
relative and with central differences (eps = 1e-6) to 1e-6 relative; J agrees
with the oracle to 1e-10.
"""
import numpy as np
import pytest

from adjoint_torch import maxwell_stress_mean
from gpu_util import rel, require_gpu
from oracle import oracle as O
from ql_dns_b200.initial import initial_state
from ql_dns_b200.params import QLParams, mri_16x16_nz32
from ql_dns_b200.solver import QLSolver

pytestmark = pytest.mark.gpu


def directions(shape, n, seed, scale):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        d = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        out.append(d * (scale / np.linalg.norm(d)))
    return out


def gpu_J(p, lin, mf, kx0, n):
    with QLSolver(p) as s:
        s.set_state(0.0, lin, mf, kx0)
        d = s.step(n, diag_every=1)
    return d[:, 8].mean()


@pytest.mark.parametrize("integ,NZ", [(0, 16), (0, 32), (0, 64), (0, 128), (1, 16), (1, 32), (1, 64), (1, 128)])
def test_adjoint_matches_tangent_linear(integ, NZ):
    require_gpu()
    p = mri_16x16_nz32(nx=8, ny=8, NZ=NZ, integrator=integ)
    lin, mf, kx0 = initial_state(p, 7, sigma=0.2)
    n = 24
    with QLSolver(p) as s:
        J, g, gm = s.adjoint_maxwell(0.0, lin, mf, kx0, n, checkpoint_every=5)
    Jo, _ = O.tlm_maxwell(p, 0.0, lin, mf, kx0, np.zeros_like(lin), None, n)
    assert abs(J - Jo) <= 1e-10 * abs(Jo)
    for d in directions(lin.shape, 3, NZ, np.linalg.norm(lin)):
        _, dJ = O.tlm_maxwell(p, 0.0, lin, mf, kx0, d, None, n)
        adj = float(np.real(np.vdot(g, d)))
        assert abs(adj - dJ) <= 1e-8 * abs(dJ), (adj, dJ)
    # the mean-field gradient along a real mean-field profile (Hermitian in kz): the step
    # keeps the real part of the mean-field profiles, which is all a real field has
    dm = directions(mf.shape, 1, 99, np.linalg.norm(mf))[0]
    nzs = mf.shape[1]
    dm[:, 0] = dm[:, 0].real
    for s_ in range(1, (nzs - 1) // 2 + 1):
        dm[:, nzs - s_] = np.conj(dm[:, s_])
    _, dJm = O.tlm_maxwell(p, 0.0, lin, mf, kx0, np.zeros_like(lin), dm, n)
    assert abs(float(np.real(np.vdot(gm, dm))) - dJm) <= 1e-8 * abs(dJm)


@pytest.mark.parametrize("integ", [0, 1])
def test_adjoint_through_remaps_vs_tangent_linear(integ):
    # high-ky modes shear past the remap threshold during the run
    require_gpu()
    p = QLParams(nx=8, ny=12, NZ=32, dt=0.02, integrator=integ)
    lin, mf, kx0 = initial_state(p, 11, sigma=0.3)
    n = 60
    t, lo, mo, ko, _ = O.run(p, 0.0, lin, mf, kx0, n)
    assert not np.array_equal(ko, kx0), "no remap happened"
    with QLSolver(p) as s:
        J, g, _ = s.adjoint_maxwell(0.0, lin, mf, kx0, n, checkpoint_every=13)
    for d in directions(lin.shape, 3, 5, np.linalg.norm(lin)):
        _, dJ = O.tlm_maxwell(p, 0.0, lin, mf, kx0, d, None, n)
        assert abs(float(np.real(np.vdot(g, d))) - dJ) <= 1e-8 * abs(dJ)


@pytest.mark.parametrize("integ", [0, 1])
def test_adjoint_matches_central_differences(integ):
    require_gpu()
    p = mri_16x16_nz32(nx=16, ny=16, NZ=32, integrator=integ)
    lin, mf, kx0 = initial_state(p, 3, sigma=0.05)
    n = 40
    with QLSolver(p) as s:
        J, g, _ = s.adjoint_maxwell(0.0, lin, mf, kx0, n, checkpoint_every=10)
    eps = 1e-6
    for d in directions(lin.shape, 4, 17, 1.0):
        d = d * np.linalg.norm(lin)  # unit direction in units of |lin0|
        fd = (gpu_J(p, lin + eps * d, mf, kx0, n) - gpu_J(p, lin - eps * d, mf, kx0, n)) / (2 * eps)
        adj = float(np.real(np.vdot(g, d)))
        assert abs(adj - fd) <= 1e-6 * abs(fd), (adj, fd)


def test_adjoint_checkpoint_interval_does_not_change_the_gradient():
    require_gpu()
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    lin, mf, kx0 = initial_state(p, 2, sigma=0.2)
    with QLSolver(p) as s:
        J1, g1, m1 = s.adjoint_maxwell(0.0, lin, mf, kx0, 30, checkpoint_every=30)
        J2, g2, m2 = s.adjoint_maxwell(0.0, lin, mf, kx0, 30, checkpoint_every=4)
        # the handle is left at the end of the forward run
        t, lo, mo, ko = s.get_state()
    assert J1 == J2 and np.array_equal(g1, g2) and np.array_equal(m1, m2)
    t2, lo2, mo2, ko2, _ = O.run(p, 0.0, lin, mf, kx0, 30)
    assert abs(t - t2) < 1e-12 and rel(lo, lo2) < 1e-10


def test_torch_autograd_wrapper():
    require_gpu()
    import torch
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    lin, mf, kx0 = initial_state(p, 4, sigma=0.2)
    with QLSolver(p) as s:
        x = torch.from_numpy(lin.copy()).requires_grad_(True)
        J = maxwell_stress_mean(x, s, mf, kx0, 16, 8)
        (gx,) = torch.autograd.grad(J, x)
        _, g, _ = s.adjoint_maxwell(0.0, lin, mf, kx0, 16, 8)
    assert np.array_equal(gx.numpy(), g)
    d = directions(lin.shape, 1, 8, np.linalg.norm(lin))[0]
    _, dJ = O.tlm_maxwell(p, 0.0, lin, mf, kx0, d, None, 16)
    assert abs(float(np.real(np.vdot(gx.numpy(), d))) - dJ) <= 1e-8 * abs(dJ)


@pytest.mark.parametrize("mode", ["persistent", "streams"])
def test_batch_of_seeds_equals_single_calls(mode, monkeypatch):
    # persistent (default): the seeds' forward sweep and window recompute run in the
    # persistent batch kernel, whose reduction order differs from the single-case kernel:
    # equal to round-off.  streams: every seed's single-case path interleaved on its own
    # stream: bit for bit.
    require_gpu()
    if mode == "streams":
        monkeypatch.setenv("QLGPU_ADJ_BATCH", "streams")
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    sts = [initial_state(p, 20 + k, sigma=0.2) for k in range(3)]
    n, ck = 18, 5
    singles = []
    for lin, mf, kx0 in sts:
        with QLSolver(p) as s:
            singles.append(s.adjoint_maxwell(0.0, lin, mf, kx0, n, checkpoint_every=ck))
    solvers = [QLSolver(p) for _ in sts]
    try:
        J, gl, gm = QLSolver.adjoint_maxwell_batch(solvers, 0.0, [s[0] for s in sts], [s[1] for s in sts],
                                                   [s[2] for s in sts], n, ck)
        for k in range(3):
            if mode == "streams":
                assert J[k] == singles[k][0]
                assert np.array_equal(gl[k], singles[k][1]) and np.array_equal(gm[k], singles[k][2])
            else:
                assert abs(J[k] - singles[k][0]) <= 1e-12 * abs(singles[k][0])
                assert rel(gl[k], singles[k][1]) < 1e-10 and rel(gm[k], singles[k][2]) < 1e-10
            # the handles are left at the end of the forward run
            t, lo, mo, ko = solvers[k].get_state()
            t2, lo2, mo2, ko2, _ = O.run(p, 0.0, *sts[k], n)
            assert rel(lo, lo2) < 1e-10 and np.array_equal(ko, ko2)
        # the gradient against the tangent-linear model, through the persistent path too
        d = directions(sts[0][0].shape, 1, 3, np.linalg.norm(sts[0][0]))[0]
        _, dJ = O.tlm_maxwell(p, 0.0, *sts[0], d, None, n)
        assert abs(float(np.real(np.vdot(gl[0], d))) - dJ) <= 1e-8 * abs(dJ)
    finally:
        for s in solvers:
            s.close()


def test_window_graphs_equal_direct_launches(monkeypatch):
    # QLGPU_ADJ_GRAPH=1 with an even checkpoint interval: every full window is one graph launch per sweep;
    # the partial last window runs with direct launches; results are bitwise those of
    # direct launches throughout
    require_gpu()
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    lin, mf, kx0 = initial_state(p, 9, sigma=0.2)
    with QLSolver(p) as s:
        monkeypatch.setenv("QLGPU_ADJ_GRAPH", "1")
        a = s.adjoint_maxwell(0.0, lin, mf, kx0, 22, checkpoint_every=4)
        monkeypatch.setenv("QLGPU_ADJ_GRAPH", "0")
        b = s.adjoint_maxwell(0.0, lin, mf, kx0, 22, checkpoint_every=4)
    assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


def test_batch_reverse_graphs_equal_direct_launches(monkeypatch):
    # QLGPU_ADJ_REVERSE=streams with QLGPU_ADJ_GRAPH=1: the persistent path replays every full
    # reverse window (even checkpoint interval) as one graph per seed; with 0 every kernel is
    # launched directly
    require_gpu()
    monkeypatch.setenv("QLGPU_ADJ_REVERSE", "streams")
    monkeypatch.setenv("QLGPU_ADJ_GRAPH", "1")
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    sts = [initial_state(p, 30 + k, sigma=0.2) for k in range(2)]
    args = (0.0, [s[0] for s in sts], [s[1] for s in sts], [s[2] for s in sts], 22, 6)
    solvers = [QLSolver(p) for _ in sts]
    try:
        a = QLSolver.adjoint_maxwell_batch(solvers, *args)
        monkeypatch.setenv("QLGPU_ADJ_GRAPH", "0")
        b = QLSolver.adjoint_maxwell_batch(solvers, *args)
    finally:
        for s in solvers:
            s.close()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    with QLSolver(p) as s:
        J, g, _ = s.adjoint_maxwell(0.0, *sts[1], 22, 6)
    assert abs(a[0][1] - J) <= 1e-12 * abs(J) and rel(a[1][1], g) < 1e-10


@pytest.mark.parametrize("ck", [6, 5])
def test_seed_batched_reverse_equals_per_seed_reverse(ck, monkeypatch):
    # default: the reverse sweep launches each kernel once for all seeds (grid row = seed);
    # QLGPU_ADJ_REVERSE=streams: every seed's reverse on its own stream.  Same arithmetic per
    # seed, so the gradients agree bit for bit (odd and even checkpoint intervals, a partial
    # last window, remaps inside the run)
    require_gpu()
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    sts = [initial_state(p, 40 + k, sigma=0.2) for k in range(3)]
    args = (0.0, [s[0] for s in sts], [s[1] for s in sts], [s[2] for s in sts], 23, ck)
    solvers = [QLSolver(p) for _ in sts]
    try:
        monkeypatch.setenv("QLGPU_ADJ_REVERSE", "seeds")
        a = QLSolver.adjoint_maxwell_batch(solvers, *args)
        monkeypatch.setenv("QLGPU_ADJ_REVERSE", "streams")
        b = QLSolver.adjoint_maxwell_batch(solvers, *args)
        for k in range(3):
            t, lo, mo, ko = solvers[k].get_state()
            t2, lo2, mo2, ko2, _ = O.run(p, 0.0, *sts[k], 23)
            assert rel(lo, lo2) < 1e-10 and np.array_equal(ko, ko2)
    finally:
        for s in solvers:
            s.close()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    d = directions(sts[2][0].shape, 1, 5, np.linalg.norm(sts[2][0]))[0]
    _, dJ = O.tlm_maxwell(p, 0.0, *sts[2], d, None, 23)
    assert abs(float(np.real(np.vdot(a[1][2], d))) - dJ) <= 1e-8 * abs(dJ)


def test_seeds_with_different_parameters_reverse_per_seed():
    # seeds whose parameters differ (here eta) cannot share the batched reverse launches: each
    # runs its own reverse sweep, with the same gradient as a single-seed call to round-off
    require_gpu()
    p1 = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    p2 = mri_16x16_nz32(nx=8, ny=8, NZ=32, eta=p1.eta * 2)
    sts = [initial_state(p1, 50 + k, sigma=0.2) for k in range(2)]
    solvers = [QLSolver(p1), QLSolver(p2)]
    try:
        J, gl, gm = QLSolver.adjoint_maxwell_batch(solvers, 0.0, [s[0] for s in sts], [s[1] for s in sts],
                                                   [s[2] for s in sts], 12, 4)
    finally:
        for s in solvers:
            s.close()
    for k, pk in enumerate((p1, p2)):
        with QLSolver(pk) as s:
            J1, g1, m1 = s.adjoint_maxwell(0.0, *sts[k], 12, 4)
        assert abs(J[k] - J1) <= 1e-12 * abs(J1) and rel(gl[k], g1) < 1e-10 and rel(gm[k], m1) < 1e-10


def test_crank_nicolson_batch_of_seeds_against_tangent_linear():
    # RK3CN through the persistent path: the window recompute records every stage's
    # old-operator clock fields, which the stage adjoint of the seeds' reverse sweep reads
    require_gpu()
    p = mri_16x16_nz32(nx=8, ny=8, NZ=64, integrator=1)
    sts = [initial_state(p, 60 + k, sigma=0.2) for k in range(2)]
    n, ck = 17, 5
    solvers = [QLSolver(p) for _ in sts]
    try:
        J, gl, gm = QLSolver.adjoint_maxwell_batch(solvers, 0.0, [s[0] for s in sts], [s[1] for s in sts],
                                                   [s[2] for s in sts], n, ck)
    finally:
        for s_ in solvers:
            s_.close()
    for k in range(2):
        Jo, _ = O.tlm_maxwell(p, 0.0, *sts[k], np.zeros_like(sts[k][0]), None, n)
        assert abs(J[k] - Jo) <= 1e-10 * abs(Jo)
        for d in directions(sts[k][0].shape, 2, 70 + k, np.linalg.norm(sts[k][0])):
            _, dJ = O.tlm_maxwell(p, 0.0, *sts[k], d, None, n)
            assert abs(float(np.real(np.vdot(gl[k], d))) - dJ) <= 1e-8 * abs(dJ)
