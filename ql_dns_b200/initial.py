"""Seeded initial conditions for the quasi-linear shearing box.

The reference seeds its fluctuations from ``clock()`` (QL_DNS/Models/
MHD_BQlin.cpp:41) and so never reproduces a run.  This module defines a
deterministic law instead, used identically for the GPU path and the CPU
oracle:

* fluctuations: every (kx, ky, kz) entry of each field (u, zeta, b, eta) is a
  complex Gaussian of physical standard deviation ``sigma * |k|^-2`` (real and
  imaginary parts each ``sigma |k|^-2 / sqrt(2)``), drawn from numpy's PCG64
  with the given seed in (mode, field, kz) order.  The reference stores
  coefficients as unnormalised transforms of the real-space field, so the
  stored value is the physical one times Nx*Ny*NZ (the energy normalisation
  of QL_DNS/Models/MHD_BQlin.cpp:52-53,420);
* the kx=ky=0 column and all ky=kz=0 entries are zero;
* ky=0 columns are Hermitian: f(-kx, 0, -kz) = conj f(kx, 0, kz), the pairing
  the reference enforces for its noise (QL_DNS/Models/MHD_BQlin.cpp:613-615,
  QL_DNS/Auxiliary/Kdata.cpp:124-146);
* mean field: Bx = 0, By(z) = B0 sin(2 pi z / Lz) sampled on the NZ real grid
  and forward transformed with the unnormalised FFTW convention, then
  truncated to the dealiased length (QL_DNS/solution.cpp:105,159-161).

Divergence-freeness holds by construction: (u, zeta) = (u_x, omega_x) fix the
other components (QL_DNS/Models/MHD_BQlin.cpp:143-146).
"""
from __future__ import annotations

import numpy as np

from .params import QLParams
from .ktables import ktables


def dealias_indices(NZ: int, nz: int) -> np.ndarray:
    """Positions in a length-NZ transform that the dealiased vector keeps
    (fftwPlans.h:84-97): 0..(nz-1)/2 then NZ-(nz-1)/2..NZ-1."""
    h = (nz - 1) // 2
    return np.concatenate([np.arange(h + 1), np.arange(NZ - h, NZ)])


def mean_field_profile(p: QLParams, bx_real: np.ndarray, by_real: np.ndarray) -> np.ndarray:
    """Spectral mean fields [nmf, nz] from real-space profiles on the NZ grid."""
    idx = dealias_indices(p.NZ, p.nz)
    mf = np.zeros((p.nmf, p.nz), dtype=np.complex128)
    mf[0] = np.fft.fft(bx_real.astype(np.complex128))[idx]
    mf[1] = np.fft.fft(by_real.astype(np.complex128))[idx]
    return hermitian(mf)


def hermitian(a: np.ndarray) -> np.ndarray:
    """Project the last (dealiased kz) axis onto exact conjugate symmetry, the
    spectrum of a real z profile."""
    nz = a.shape[-1]
    flip = (nz - np.arange(nz)) % nz
    return 0.5 * (a + np.conj(a[..., flip]))


def initial_state(p: QLParams, seed: int, sigma: float = 1e-3, B0: float = 0.05,
                  mean_u: float = 0.0):
    """Return (lin[nxy, 4, nz] c128, mf[nmf, nz] c128, kx0[nxy] f64).

    ``mean_u`` adds Ux = Uy = mean_u cos(2 pi z / Lz) for MHD_FullQlin runs
    (zero by default)."""
    kt = ktables(p)
    nxy, nz = p.nxy, p.nz
    kx = kt["kx"][:, None]
    ky = kt["ky"][:, None]
    kz = kt["kz"][None, :]
    k2 = kx * kx + ky * ky + kz * kz
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(k2 > 0, sigma / k2, 0.0) * float(p.nx * (p.ny // 2 * 2) * p.NZ)
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal((nxy, 4, nz, 2))
    lin = (g[..., 0] + 1j * g[..., 1]) * (amp[:, None, :] / np.sqrt(2.0))
    kxi, kyi = kt["kx_index"], kt["ky_index"]
    # zero the mean-field column and the ky=kz=0 entries
    lin[(kxi == 0) & (kyi == 0)] = 0.0
    lin[kyi == 0, :, 0] = 0.0
    # Hermitian pairing of the ky=0 columns: negative kx from positive kx
    flip = (nz - np.arange(nz)) % nz  # stored index of -kz
    pos = {int(kxi[i]): i for i in range(nxy) if kyi[i] == 0}
    for i in range(nxy):
        if kyi[i] == 0 and kxi[i] < 0:
            j = pos[-int(kxi[i])]
            lin[i] = np.conj(lin[j][:, flip])
    zg = np.arange(p.NZ) * (p.L[2] / p.NZ)
    by = B0 * np.sin(2 * np.pi * zg / p.L[2])
    mf = mean_field_profile(p, np.zeros(p.NZ), by)
    if p.nmf == 4 and mean_u != 0.0:
        idx = dealias_indices(p.NZ, p.nz)
        prof = mean_u * np.cos(2 * np.pi * zg / p.L[2])
        mf[2] = hermitian(np.fft.fft(prof.astype(np.complex128))[idx])
        mf[3] = mf[2]
    return np.ascontiguousarray(lin), np.ascontiguousarray(mf), kt["kx"].copy()


def dns_initial_state(p, seed: int, sigma: float = 1e-2, B0: float = 0.05):
    """Seeded initial state of the 3-D DNS (``DNSParams`` p).

    Returns (lin[nxy, 6, nz] c128 = (u_x, u_y, u_z, b_x, b_y, b_z) per mode
    column, kx0[nxy] f64).  Every (kx, ky, kz) entry of each Cartesian
    component is a complex Gaussian of physical standard deviation
    ``sigma |k|^-2`` (PCG64 with the given seed, (mode, component, kz) order),
    then projected onto the plane normal to k (divergence-free); k = 0 entries
    and the kx=ky=0 column are zero; ky=0 columns are Hermitian,
    f(-kx, 0, -kz) = conj f(kx, 0, kz).  The kx=ky=0 column carries the mean
    field By(z) = B0 sin(2 pi z / Lz), Bx = Ux = Uy = 0.  Stored values are the
    physical ones times Mx*My*NZ (unnormalised forward transform)."""
    q = p.ql()
    kt = ktables(q)
    nxy, nz = q.nxy, q.nz
    kx = kt["kx"][:, None]
    ky = kt["ky"][:, None]
    kz = kt["kz"][None, :]
    k2 = kx * kx + ky * ky + kz * kz
    norm = float(p.Mx * p.My * p.NZ)
    with np.errstate(divide="ignore"):
        amp = np.where(k2 > 0, sigma / k2, 0.0) * norm
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal((nxy, 6, nz, 2))
    lin = (g[..., 0] + 1j * g[..., 1]) * (amp[:, None, :] / np.sqrt(2.0))
    kv = [np.broadcast_to(kx, k2.shape), np.broadcast_to(ky, k2.shape), np.broadcast_to(kz, k2.shape)]
    with np.errstate(invalid="ignore", divide="ignore"):
        ik2 = np.where(k2 > 0, 1.0 / k2, 0.0)
    for base in (0, 3):
        kdot = sum(kv[c] * lin[:, base + c] for c in range(3))
        for c in range(3):
            lin[:, base + c] -= kv[c] * kdot * ik2
    kxi, kyi = kt["kx_index"], kt["ky_index"]
    lin[(kxi == 0) & (kyi == 0)] = 0.0
    flip = (nz - np.arange(nz)) % nz
    pos = {int(kxi[i]): i for i in range(nxy) if kyi[i] == 0}
    for i in range(nxy):
        if kyi[i] == 0 and kxi[i] < 0:
            lin[i] = np.conj(lin[pos[-int(kxi[i])]][:, flip])
    zg = np.arange(p.NZ) * (p.L[2] / p.NZ)
    by = B0 * np.sin(2 * np.pi * zg / p.L[2])
    idx = dealias_indices(p.NZ, nz)
    lin[0, 4] = hermitian(np.fft.fft(by.astype(np.complex128))[idx]) * float(p.Mx * p.My)
    return np.ascontiguousarray(lin), kt["kx"].copy()
