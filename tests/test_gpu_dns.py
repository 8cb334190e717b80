"""The 3-D DNS on the GPU (include/qlgpu_dns.h through ql_dns_b200.dns.QLDns)
against the numpy DNS oracle (oracle/dns_oracle.py).

Bars: one right-hand side to 1e-12 relative (L2), states after N steps and the
diagnostic series to 1e-10 relative; at 64 x 128 x 64 the ideal energy budget
of the GPU right-hand side (dE/dt = q sum w Re(u_x u_y^* - b_x b_y^*)) to
1e-12 of |u||F| and the divergence of the stepped state to round-off.
"""
import numpy as np
import pytest

from gpu_util import rel, require_gpu
from oracle.dns_oracle import DNSOracle
from ql_dns_b200.initial import dns_initial_state
from ql_dns_b200.params import DNSParams, dns_64x128x64

pytestmark = pytest.mark.gpu


def series_rel(d1, d2):
    return max(np.abs(d1[:, c] - d2[:, c]).max() / max(np.abs(d2[:, c]).max(), 1e-300) for c in range(1, 15))


def make(p, seed, sigma=0.3, B0=0.1, t=0.0):
    D = DNSOracle(p)
    lin, kx0 = dns_initial_state(p, seed, sigma=sigma, B0=B0)
    if t:
        lin = D.constrain(t, lin, kx0)
    return D, lin, kx0


@pytest.mark.parametrize("grid", [(16, 32, 16), (32, 64, 32), (16, 16, 64), (64, 32, 16), (32, 256, 32),
                                  (64, 128, 64)])
def test_rhs_matches_oracle(grid):
    require_gpu()
    from ql_dns_b200.dns import QLDns
    Mx, My, NZ = grid
    p = DNSParams(Mx=Mx, My=My, NZ=NZ, B0z=0.05, q=1.5, omega=1.0)
    t = 0.137
    D, lin, kx0 = make(p, 11, t=t)
    with QLDns(p) as g:
        g.set_state(t, lin, kx0)
        F = g.rhs(t)
    Fo = D.rhs(t, lin, kx0)
    assert rel(F, Fo) < 1e-12, rel(F, Fo)


@pytest.mark.parametrize("integ", [0, 1])
def test_steps_match_oracle(integ):
    require_gpu()
    from ql_dns_b200.dns import QLDns
    p = DNSParams(Mx=16, My=32, NZ=16, dt=0.01, B0z=0.02, integrator=integ, nu=1 / 500, eta=1 / 700)
    D, lin, kx0 = make(p, 6, sigma=0.3)
    n = 40
    t2, lo, ko, d2 = D.run(0.0, lin, kx0, n, diag_every=1)
    assert (ko != kx0).sum() > 0  # remaps happened
    with QLDns(p) as g:
        g.set_state(0.0, lin, kx0)
        d = g.step(n, diag_every=1)
        t, lg, kg = g.get_state()
        assert g.status() == 0
    assert t == t2 and np.array_equal(kg, ko)
    assert rel(lg, lo) < 1e-10, rel(lg, lo)
    assert d.shape == d2.shape and series_rel(d, d2) < 1e-10


def test_chunked_steps_equal_one_call():
    require_gpu()
    from ql_dns_b200.dns import QLDns
    p = DNSParams(Mx=32, My=64, NZ=32, dt=0.01, B0z=0.01)
    _, lin, kx0 = make(p, 8, sigma=0.2)
    with QLDns(p) as g:
        g.set_state(0.0, lin, kx0)
        g.step(12)
        a = g.get_state()
        g.set_state(0.0, lin, kx0)
        g.step(5)
        g.step(7, diag_every=7)
        b = g.get_state()
    assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


def test_production_grid_short_run_matches_oracle():
    # 64 x 128 x 64, Re = Rm = 4000, dt = 0.005, sigma = 1e-2, seed 2: three steps
    require_gpu()
    from ql_dns_b200.dns import QLDns
    p = dns_64x128x64()
    D, lin, kx0 = make(p, 2, sigma=1e-2, B0=0.05)
    n = 3
    t2, lo, ko, d2 = D.run(0.0, lin, kx0, n, diag_every=1)
    with QLDns(p) as g:
        g.set_state(0.0, lin, kx0)
        d = g.step(n, diag_every=1)
        t, lg, kg = g.get_state()
    assert rel(lg, lo) < 1e-10 and series_rel(d, d2) < 1e-10


def test_production_grid_energy_budget_and_divergence():
    require_gpu()
    from ql_dns_b200.dns import QLDns
    p = dns_64x128x64(nu=0.0, eta=0.0, B0z=0.03)
    D, lin, kx0 = make(p, 2, sigma=0.3, B0=0.1, t=0.21)
    with QLDns(p) as g:
        g.set_state(0.21, lin, kx0)
        F = g.rhs(0.21)
        w = np.where(D.ky == 0.0, 1.0, 2.0)[:, None]
        rate = float(np.sum(w[:, :, None] * np.real(np.conj(lin) * F)))
        work = p.q * np.sum(w * (np.real(lin[:, 0] * np.conj(lin[:, 1])) - np.real(lin[:, 3] * np.conj(lin[:, 4]))))
        scale = np.sqrt(np.sum(np.abs(lin) ** 2) * np.sum(np.abs(F) ** 2))
        assert abs(rate - work) < 1e-12 * scale
        g.step(20)
        t, lg, kg = g.get_state()
    Kx, Ky, Kz = D.kvec(t, kg)
    for b in (0, 3):
        div = Kx * lg[:, b] + Ky * lg[:, b + 1] + Kz * lg[:, b + 2]
        assert np.abs(div).max() < 1e-12 * np.abs(lg).max() * np.abs(Kx).max()


def test_nonfinite_state_sets_status():
    require_gpu()
    from ql_dns_b200._capi import QLGPUError
    from ql_dns_b200.dns import QLDns
    p = DNSParams(Mx=16, My=32, NZ=16)
    _, lin, kx0 = make(p, 1)
    lin[5, 2, 3] = np.nan
    with QLDns(p) as g:
        g.set_state(0.0, lin, kx0)
        with pytest.raises(QLGPUError) as ei:
            g.step(1)
        assert ei.value.code == 4
        assert g.status() & 1
        _, lin2, kx2 = make(p, 1)
        g.set_state(0.0, lin2, kx2)
        g.step(2)
        assert g.status() == 0


def test_unsupported_grid_is_refused():
    require_gpu()
    from ql_dns_b200._capi import QLGPUError
    from ql_dns_b200.dns import QLDns
    with pytest.raises(QLGPUError) as ei:
        QLDns(DNSParams(Mx=128, My=128, NZ=64))
    assert ei.value.code == 2


@pytest.mark.parametrize("name", ["dns_exp", "dns_cn_hyper"])
def test_golden_fixtures_on_gpu(name):
    # the frozen oracle trajectories (tests/golden/make_dns_golden.py), incl. RK3CN with order-4 dissipation
    require_gpu()
    import os
    from ql_dns_b200.dns import QLDns
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    p = DNSParams(integrator=int(g["integrator"]), Mx=int(g["Mx"]), My=int(g["My"]), NZ=int(g["NZ"]),
                  L=tuple(g["L"]), q=float(g["q"]), omega=float(g["omega"]), nu=float(g["nu"]), eta=float(g["eta"]),
                  B0z=float(g["B0z"]), viscosity_order=int(g["viscosity_order"]), dt=float(g["dt"]),
                  remap=int(g["remap"]), dealias_xy=int(g["dealias_xy"]))
    with QLDns(p) as d:
        d.set_state(0.0, g["lin0"], g["kx00"])
        rec = d.step(int(g["nsteps"]), diag_every=1)
        t, lo, ko = d.get_state()
    assert t == float(g["t"]) and np.array_equal(ko, g["kx0"])
    assert rel(lo, g["lin"]) < 1e-10 and series_rel(rec, g["diag"]) < 1e-10


def test_bad_kx0_is_refused():
    require_gpu()
    from ql_dns_b200._capi import QLGPUError
    from ql_dns_b200.dns import QLDns
    p = DNSParams(Mx=16, My=32, NZ=16)
    _, lin, kx0 = make(p, 1)
    with QLDns(p) as g:
        bad = kx0.copy()
        bad[7] += 0.3  # off the lattice
        with pytest.raises(QLGPUError) as ei:
            g.set_state(0.0, lin, bad)
        assert ei.value.code == 1
        bad = kx0.copy()
        Kyn = g.ny // 2
        bad[Kyn] = bad[2 * Kyn]  # two columns of the ky = 0 plane in one x bin
        with pytest.raises(QLGPUError):
            g.set_state(0.0, lin, bad)
        g.set_state(0.0, lin, kx0)
        g.step(1)
