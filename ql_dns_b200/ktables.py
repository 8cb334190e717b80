"""Wavenumber tables, restating QL_DNS/Auxiliary/Kdata.cpp:11-120.

Modes are ordered ``j + (Ny/2) * i`` with kx = i*2pi/Lx for i < Nx/2, then the
negative kx with the Nyquist frequency dropped; ky = j*2pi/Ly >= 0 only; kz in
dealiased order 0..(nz-1)/2, -(nz-1)/2..-1.  All are returned as the real
multipliers of i (the reference stores them as purely imaginary complexes).
"""
from __future__ import annotations

import math

import numpy as np

from .params import QLParams


def ktables(p: QLParams) -> dict:
    kxL = 2 * math.pi / p.L[0]
    kyL = 2 * math.pi / p.L[1]
    kzL = 2 * math.pi / p.L[2]
    ny, nx = (p.ny // 2 * 2) // 2, p.nx // 2
    nxy = p.nxy
    kx = np.zeros(nxy)
    ky = np.zeros(nxy)
    kxi = np.zeros(nxy, dtype=np.int32)
    kyi = np.zeros(nxy, dtype=np.int32)
    for i in range(nx):
        for j in range(ny):
            kx[j + ny * i] = i * kxL
            ky[j + ny * i] = j * kyL
            kxi[j + ny * i] = i
            kyi[j + ny * i] = j
    for i in range(nx + 1, 2 * nx):
        for j in range(ny):
            kx[j + ny * (i - 1)] = (-2 * nx + i) * kxL
            ky[j + ny * (i - 1)] = j * kyL
            kxi[j + ny * (i - 1)] = -2 * nx + i
            kyi[j + ny * (i - 1)] = j
    nz = p.nz
    nzl = (nz - 1) // 2
    kz = np.zeros(nz)
    for i in range(nzl + 1):
        kz[i] = i * kzL
    for i in range(nzl + 1, 2 * nzl + 1):
        kz[i] = (-2 * nzl + i - 1) * kzL
    return {"kx": kx, "ky": ky, "kx_index": kxi, "ky_index": kyi, "kz": kz}
