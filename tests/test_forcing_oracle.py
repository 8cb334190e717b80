"""Driving noise and the CFL time step in the CPU oracle (oracle/ql_oracle.cpp:
driving_noise, calculate_cfl, oracle_run_forced).

The reference's noise comes from a clock-seeded mt19937 (QL_DNS/Models/
MHD_BQlin.cpp:22-23) and cannot be reproduced, so the restatement is checked
statistically: one step from a zero fluctuation field leaves exactly the noise
increments, whose per-entry amplitude follows MHD_BQlin.cpp:570-580 and whose
normalised values must be complex normals of variance f_noise^2.  The generator
is pinned by the Philox4x32-10 known-answer vectors of its authors.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from ql_dns_b200.initial import initial_state
from ql_dns_b200.ktables import ktables
from ql_dns_b200.params import QLParams


def test_philox_known_answers():
    kat = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
           ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
           ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, out in kat:
        assert list(O.philox(ctr, key)) == out


def noise_amplitudes(p, t, dt, klo, khi):
    """Per (mode, kz) multipliers (u, zeta) of MHD_BQlin::DrivingNoise, restated in numpy."""
    kt = ktables(p)
    kx = kt["kx"] + p.q * t * kt["ky"]
    kz2 = -(kt["kz"] ** 2)
    lap2 = -(kt["ky"][:, None] ** 2) + kz2[None, :]
    lapF = -(kx[:, None] ** 2) + lap2
    tot = float(p.nx * (p.ny // 2 * 2) * p.NZ)
    m = dt * tot * tot * (1.0 / (16 * 32 * 32)) ** 2
    drive = (lapF > -khi * khi) & (lapF < -klo * klo) & (kt["ky_index"][:, None] != 0)
    with np.errstate(invalid="ignore", divide="ignore"):
        mu = np.where(drive, np.sqrt(m * lap2 / lapF), 0.0)
        mz = np.where(drive, np.sqrt(-m * lap2), 0.0)
    return drive, mu, mz


def test_noise_statistics_and_amplitudes():
    p = QLParams(nx=32, ny=32, NZ=32, dt=0.01, remap=0)
    lin, mf, kx0 = initial_state(p, 0, sigma=0.0)
    f, klo, khi = 0.7, 2.0, 40.0
    t, lo, mo, ko, _, dtm = O.run_forced(p, 0.0, lin, mf, kx0, 1, f_noise=f, k_lo=klo, k_hi=khi, seed=99)
    assert dtm == p.dt
    drive, mu, mz = noise_amplitudes(p, 0.0, p.dt, klo, khi)
    assert drive.sum() > 1000
    # undriven entries (ky = 0, outside the band) stay exactly zero; the mean field only evolves
    for v in range(4):
        assert not np.any(lo[:, v][~drive])
    z = np.concatenate([lo[:, v][drive] / (mu if v in (0, 2) else mz)[drive] for v in range(4)])
    n = z.size
    # complex normal, variance f^2 (f/sqrt(2) per part), independent parts
    assert abs(z.real.mean()) < 4 * f / math.sqrt(2 * n) and abs(z.imag.mean()) < 4 * f / math.sqrt(2 * n)
    var = np.mean(np.abs(z) ** 2)
    assert abs(var / f ** 2 - 1) < 4 * math.sqrt(2.0 / n)
    assert abs(np.mean(z.real * z.imag)) < 4 * (f * f / 2) / math.sqrt(n)
    # kurtosis of a normal part: 3
    r = z.real / (f / math.sqrt(2))
    assert abs(np.mean(r ** 4) - 3) < 8 * math.sqrt(96.0 / n)
    # a different seed gives different numbers, the same seed the same
    _, lo2, *_ = O.run_forced(p, 0.0, lin, mf, kx0, 1, f_noise=f, k_lo=klo, k_hi=khi, seed=99)
    _, lo3, *_ = O.run_forced(p, 0.0, lin, mf, kx0, 1, f_noise=f, k_lo=klo, k_hi=khi, seed=100)
    assert np.array_equal(lo, lo2) and not np.array_equal(lo, lo3)


def test_noise_off_equals_plain_run():
    p = QLParams(nx=8, ny=8, NZ=32, dt=0.01)
    lin, mf, kx0 = initial_state(p, 3, sigma=0.2)
    a = O.run(p, 0.0, lin, mf, kx0, 20, diag_every=5)
    b = O.run_forced(p, 0.0, lin, mf, kx0, 20, diag_every=5)
    assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert np.array_equal(a[4], b[4])


@pytest.mark.parametrize("model", [0, 1])
def test_cfl_time_step(model):
    p = QLParams(model=model, nx=8, ny=8, NZ=32, dt=0.01, B0z=0.01 if model else 0.0)
    lin, mf, kx0 = initial_state(p, 3, sigma=0.2, B0=0.08, mean_u=0.02 if model else 0.0)
    cfl, dtmax = 0.2, 0.05
    t, lo, mo, ko, d, dtm = O.run_forced(p, 0.0, lin, mf, kx0, 1, cfl=cfl, dt_max=dtmax)
    # before the first rhs the stored mean-field profiles are zero: BQlin reads Bx of the
    # state (zero here), FullQlin only the stored profiles -> dt = cfl / q
    assert t == pytest.approx(min(cfl / p.q, dtmax), rel=1e-15)
    t, lo, mo, ko, d, dtm = O.run_forced(p, 0.0, lin, mf, kx0, 12, diag_every=3, cfl=cfl, dt_max=dtmax)
    assert len(d) == 5 and abs(t - 12 * dtm) < 1e-14 and dtm < cfl / p.q
    kmax = max(2 * math.pi / p.L[0] * p.nx / 2, 2 * math.pi / p.L[1] * p.ny / 2, 2 * math.pi / p.L[2] * p.NZ / 3)
    assert dtm > cfl / (kmax * 0.2 + p.q)


def ky0_pairs(p):
    """(kx > 0, kx < 0) mode indices of the ky = 0 pairs (Kdata.cpp:124-146)."""
    kt = ktables(p)
    pos = {int(kt["kx_index"][i]): i for i in range(p.nxy) if kt["ky_index"][i] == 0}
    return [(pos[a], pos[-a]) for a in range(1, p.nx // 2)]


def test_fullqlin_noise_ky0_conjugate_pairs():
    # MHD_FullQlin::DrivingNoise (MHD_FullQlin.cpp:786-1045): ky != 0 as MHD_BQlin, and
    # ky = 0 driven so that f(-kx, 0, -kz) = conj f(kx, 0, kz) holds exactly
    p = QLParams(model=1, nx=16, ny=16, NZ=48, dt=0.01, remap=0, B0z=0.0, omega=1.0)
    lin, mf, kx0 = initial_state(p, 0, sigma=0.0, B0=0.0)
    f, klo, khi = 0.3, 0.5, 60.0
    _, lo, *_ = O.run_forced(p, 0.0, lin, mf, kx0, 1, f_noise=f, k_lo=klo, k_hi=khi, seed=5)
    kt = ktables(p)
    ky0 = kt["ky_index"] == 0
    drive, mu, mz = noise_amplitudes(p, 0.0, p.dt, klo, khi)
    # ky != 0: exactly MHD_BQlin's entries
    pb = QLParams(model=0, nx=16, ny=16, NZ=48, dt=0.01, remap=0)
    lb, mb, kb = initial_state(pb, 0, sigma=0.0, B0=0.0)
    _, lob, *_ = O.run_forced(pb, 0.0, lb, mb, kb, 1, f_noise=f, k_lo=klo, k_hi=khi, seed=5)
    assert np.array_equal(lo[~ky0], lob[~ky0])
    # ky = 0: the (0, 0) mode and kz = 0 stay zero; every pair is conjugate at mirrored kz
    i00 = [i for i in range(p.nxy) if ky0[i] and kt["kx_index"][i] == 0][0]
    assert not np.any(lo[i00]) and not np.any(lo[ky0][:, :, 0])
    nz = p.nz
    mirror = (nz - np.arange(1, nz)) % nz
    driven = 0
    for ip, ineg in ky0_pairs(p):
        assert np.array_equal(lo[ip][:, 1:], np.conj(lo[ineg][:, mirror]))
        kx = kt["kx"][ineg]
        lapF = -kx * kx - kt["kz"][1:] ** 2
        band = (lapF > -khi * khi) & (lapF < -klo * klo)
        assert np.all(lo[ineg][:, 1:][:, band] != 0) and not np.any(lo[ineg][:, 1:][:, ~band])
        driven += band.sum()
    assert driven > 50
    # the normalised ky = 0 draws are complex normals of variance f^2 as well
    tot = float(p.nx * p.ny * p.NZ)
    m = p.dt * tot * tot * (1.0 / (16 * 32 * 32)) ** 2
    z = []
    for ip, ineg in ky0_pairs(p):
        kz = kt["kz"][1:]
        lap2 = -kz * kz
        lapF = -kt["kx"][ineg] ** 2 + lap2
        band = (lapF > -khi * khi) & (lapF < -klo * klo)
        amp = [np.sqrt(m * lap2 / lapF), np.sqrt(-m * lap2)]
        for v in range(4):
            z.append(lo[ineg][v, 1:][band] / amp[v % 2][band])
    z = np.concatenate(z)
    assert abs(np.mean(np.abs(z) ** 2) / f ** 2 - 1) < 5 * math.sqrt(2.0 / z.size)


@pytest.mark.parametrize("only", ["velocity", "magnetic"])
def test_fullqlin_drive_only_switches(only):
    # drive_only_velocity / drive_only_magnetic (MHD_FullQlin.cpp:21-22): the other pair of
    # fields stays undriven, the driven pair draws the same numbers as with both on
    p = QLParams(model=1, nx=8, ny=16, NZ=32, dt=0.01, remap=0, omega=1.0)
    lin, mf, kx0 = initial_state(p, 0, sigma=0.0, B0=0.0)
    kw = dict(f_noise=0.2, k_lo=0.5, k_hi=60.0, seed=11)
    _, both, *_ = O.run_forced(p, 0.0, lin, mf, kx0, 1, **kw)
    _, one, *_ = O.run_forced(p, 0.0, lin, mf, kx0, 1, drive_only_velocity=only == "velocity",
                              drive_only_magnetic=only == "magnetic", **kw)
    on, off = ((0, 1), (2, 3)) if only == "velocity" else ((2, 3), (0, 1))
    assert np.array_equal(one[:, on], both[:, on]) and np.any(one[:, on])
    assert not np.any(one[:, off])
