"""The 3-D DNS oracle (oracle/dns_oracle.py) on the CPU.

Pins: the QL projection of its products reproduces the MHD_FullQlin oracle
(oracle/ql_oracle.cpp, itself pinned in test_oracle.py) to round-off through
remaps, for both integrators; its transforms against closed forms; and the
ideal identities of the full nonlinear terms (energy, cross helicity, the
shear work q(R - M), the divergence constraint of the shearing frame).
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle.dns_oracle import DNSOracle, from_ql, to_ql
from ql_dns_b200.initial import dns_initial_state, initial_state
from ql_dns_b200.ktables import ktables
from ql_dns_b200.params import DNSParams


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def series_rel(d1, d2):
    return max(np.abs(d1[:, c] - d2[:, c]).max() / max(np.abs(d2[:, c]).max(), 1e-300) for c in range(1, 15))


@pytest.mark.parametrize("integ,order", [(0, 2), (1, 2), (1, 4)])
def test_ql_projection_reproduces_fullqlin(integ, order):
    p = DNSParams(Mx=16, My=32, NZ=16, B0z=0.03, dt=0.01, integrator=integ, viscosity_order=order,
                  nu=1 / 300 if order == 2 else 1e-5, eta=1 / 500 if order == 2 else 2e-5)
    q = p.ql()
    lin, mf, kx0 = initial_state(q, 5, sigma=0.3, B0=0.1, mean_u=0.05)
    kt = ktables(q)
    lin[kt["ky_index"] == 0] = 0.0  # no zonal fluctuations: the (u, zeta) layout holds every mode
    n = 40
    t2, lo, mo, ko, d2 = O.run(q, 0.0, lin, mf, kx0, n, diag_every=1)
    D = DNSOracle(p)
    l6 = from_ql(p, 0.0, lin, mf, kx0)
    l4b, mfb = to_ql(p, 0.0, l6, kx0)
    assert np.abs(l4b - lin).max() <= 1e-15 * np.abs(lin).max() and np.array_equal(mfb, mf)
    t, l6n, kxn, dd = D.run(0.0, l6, kx0, n, diag_every=1, ql=True)
    assert t == t2 and np.array_equal(kxn, ko) and (ko != kx0).sum() > 0  # remaps happened
    l4n, mfn = to_ql(p, t, l6n, kxn)
    assert rel(l4n, lo) < 1e-13 and rel(mfn, mo) < 1e-13
    assert series_rel(dd, d2[1:]) < 1e-13


def test_transforms_single_mode():
    p = DNSParams(Mx=16, My=32, NZ=16)
    D = DNSOracle(p)
    kt = D.kt
    # column with kx index 2, ky index 3; kz index -1 (stored slot nz-1)
    i = int(np.where((kt["kx_index"] == 2) & (kt["ky_index"] == 3))[0][0])
    lin = np.zeros((D.nxy, 1, D.nz), dtype=complex)
    amp = 0.3 - 0.2j
    lin[i, 0, D.nz - 1] = amp * D.norm
    f = D.to_phys(lin, kt["kx"])[0]
    x = np.arange(p.Mx)[:, None, None] * p.L[0] / p.Mx
    y = np.arange(p.My)[None, :, None] * p.L[1] / p.My
    z = np.arange(p.NZ)[None, None, :] * p.L[2] / p.NZ
    ph = kt["kx"][i] * x + kt["ky"][i] * y + kt["kz"][D.nz - 1] * z
    ref = 2 * np.real(amp * np.exp(1j * ph))  # the ky > 0 mode and its conjugate
    assert np.abs(f - ref).max() < 1e-14
    back = D.from_phys(f[None], kt["kx"])
    assert abs(back[i, 0, D.nz - 1] - amp * D.norm) < 1e-12 * D.norm
    back[i, 0, D.nz - 1] = 0
    assert np.abs(back).max() < 1e-12 * D.norm


def energy_rate(D, lin, F):
    w = np.where(D.ky == 0.0, 1.0, 2.0)[:, None, None]
    return float(np.sum(w * np.real(np.conj(lin) * F)))


def test_nonlinear_terms_conserve_energy_and_cross_helicity():
    p = DNSParams(Mx=16, My=32, NZ=16, q=0.0, omega=0.0, B0z=0.0, nu=0.0, eta=0.0)
    D = DNSOracle(p)
    lin, kx0 = dns_initial_state(p, 3, sigma=0.5, B0=0.2)
    F = D.rhs(0.0, lin, kx0)
    scale = np.sqrt(np.sum(np.abs(lin) ** 2) * np.sum(np.abs(F) ** 2))
    assert abs(energy_rate(D, lin, F)) < 1e-13 * scale
    w = np.where(D.ky == 0.0, 1.0, 2.0)[:, None]
    hc = np.sum(w * np.real(np.conj(lin[:, 0:3]) * F[:, 3:6]).sum(axis=1)) + \
        np.sum(w * np.real(np.conj(lin[:, 3:6]) * F[:, 0:3]).sum(axis=1))
    assert abs(hc) < 1e-13 * scale


def test_shear_work_and_divergence_constraint():
    # with rotation, shear and B0z the energy changes only through the stresses:
    # dE/dt = q sum w Re(u_x u_y^* - b_x b_y^*); k(t).F_u = -q ky u_x, k(t).F_b = -q ky b_x
    p = DNSParams(Mx=16, My=32, NZ=16, q=1.5, omega=1.0, B0z=0.07, nu=0.0, eta=0.0)
    D = DNSOracle(p)
    lin, kx0 = dns_initial_state(p, 4, sigma=0.5, B0=0.2)
    lin[0, 0] = 0.02 * D.norm * np.exp(1j * np.arange(D.nz))  # a mean flow too
    lin[0, 0] = 0.5 * (lin[0, 0] + np.conj(lin[0, 0][(D.nz - np.arange(D.nz)) % D.nz]))
    t = 0.3
    lin = D.constrain(t, lin, kx0)  # the state the stages hold at t: masked, divergence-free at k(t)
    F = D.rhs(t, lin, kx0)
    w = np.where(D.ky == 0.0, 1.0, 2.0)[:, None]
    work = p.q * np.sum(w * (np.real(lin[:, 0] * np.conj(lin[:, 1])) - np.real(lin[:, 3] * np.conj(lin[:, 4]))))
    scale = np.sqrt(np.sum(np.abs(lin) ** 2) * np.sum(np.abs(F) ** 2))
    assert abs(energy_rate(D, lin, F) - work) < 1e-13 * scale
    Kx, Ky, Kz = D.kvec(t, kx0)
    keep = D.keep(t, kx0)[:, None]
    for b in (0, 3):
        kF = Kx * F[:, b] + Ky * F[:, b + 1] + Kz * F[:, b + 2]
        expect = np.where(keep, -p.q * Ky * lin[:, b], 0.0)
        assert np.abs(kF - expect).max() < 1e-12 * np.abs(F).max() * np.abs(Kx).max()


def test_steps_keep_divergence_free_and_hermitian():
    p = DNSParams(Mx=16, My=32, NZ=16, dt=0.01, B0z=0.02)
    D = DNSOracle(p)
    lin, kx0 = dns_initial_state(p, 6, sigma=0.3, B0=0.1)
    t, lo, ko, _ = D.run(0.0, lin, kx0, 25)
    Kx, Ky, Kz = D.kvec(t, ko)
    for b in (0, 3):
        div = Kx * lo[:, b] + Ky * lo[:, b + 1] + Kz * lo[:, b + 2]
        assert np.abs(div).max() < 1e-12 * np.abs(lo).max() * np.abs(Kx).max()
    kt = D.kt
    flip = (D.nz - np.arange(D.nz)) % D.nz
    pos = {int(kt["kx_index"][i]): i for i in range(D.nxy) if kt["ky_index"][i] == 0}
    for kxi, i in pos.items():
        j = pos.get(-kxi)
        if j is not None:
            assert np.abs(lo[j] - np.conj(lo[i][:, flip])).max() < 1e-12 * np.abs(lo).max()
    # the 2/3 rule in x: no retained column beyond Mx/3 (2 pi / Lx)
    kxt = ko + p.q * t * D.ky
    assert not np.any(lo[np.abs(kxt) > p.Mx / 3 * D.dkx])


def test_initial_state_law():
    p = DNSParams(Mx=16, My=32, NZ=16)
    lin, kx0 = dns_initial_state(p, 2, sigma=1e-2, B0=0.05)
    D = DNSOracle(p)
    Kx, Ky, Kz = D.kvec(0.0, kx0)
    for b in (0, 3):
        div = Kx * lin[:, b] + Ky * lin[:, b + 1] + Kz * lin[:, b + 2]
        assert np.abs(div).max() < 1e-12 * np.abs(lin).max() * 50
    ph = D.to_phys(lin, kx0)
    z = np.arange(p.NZ) / p.NZ
    by_mean = ph[4].mean(axis=(0, 1))
    assert np.abs(by_mean - 0.05 * np.sin(2 * np.pi * z)).max() < 1e-14
    lin2, _ = dns_initial_state(p, 2, sigma=1e-2, B0=0.05)
    assert np.array_equal(lin, lin2)


@pytest.mark.parametrize("Mx,My,NZ", [(16, 32, 16), (64, 128, 64), (6, 10, 32), (2, 2, 16)])
def test_oracle_wavenumber_tables_agree_with_the_package(Mx, My, NZ):
    # the oracle restates Kdata on its own; the package's tables (used to build the
    # GPU initial state) must be the same numbers
    from oracle.dns_oracle import kdata
    q = DNSParams(Mx=Mx, My=My, NZ=NZ).ql()
    a, b = kdata(q), ktables(q)
    for key in ("kx_index", "ky_index"):
        assert np.array_equal(a[key], b[key]), key
    for key in ("kx", "ky", "kz"):
        assert np.array_equal(a[key], b[key]), key
