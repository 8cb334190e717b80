"""ctypes wrapper of the CPU oracle (oracle/ql_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the ql_dns_b200 package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int), ("integrator", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("NZ", ctypes.c_int),
        ("L", ctypes.c_double * 3),
        ("q", ctypes.c_double), ("omega", ctypes.c_double),
        ("nu", ctypes.c_double), ("eta", ctypes.c_double), ("B0z", ctypes.c_double),
        ("viscosity_order", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("remap", ctypes.c_int), ("quasilinear", ctypes.c_int),
        ("nthreads", ctypes.c_int),
    ]


def build(native: bool = False) -> None:
    target = ["native"] if native else []
    subprocess.run(["make", "-s", "-C", HERE] + target, check=True)


_LIBS = {}


def lib(kind: str = "strict"):
    """kind: 'strict' (parity), 'strict_omp' (parity, OpenMP over modes), 'fast' (portable timing
    build) or 'native'."""
    if kind in _LIBS:
        return _LIBS[kind]
    if kind == "native":
        path = os.path.join(BUILD, "native", "liboracle_fast.so")
    else:
        path = os.path.join(BUILD, f"liboracle_{kind}.so")
    if not os.path.exists(path):
        build(native=(kind == "native"))
    L = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    L.oracle_run.argtypes = [ctypes.POINTER(OracleParams), dp, dp, dp, dp,
                             ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
    L.oracle_rhs.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_double, ctypes.c_double,
                             dp, dp, dp, dp, dp, dp]
    L.oracle_diagnostics.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_double, dp, dp, dp, dp]
    L.oracle_fft.argtypes = [ctypes.c_int, ctypes.c_int, dp]
    L.oracle_tlm_maxwell.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_double, dp, dp, dp, dp, dp,
                                     ctypes.c_int, dp, dp]
    L.oracle_run_forced.argtypes = [ctypes.POINTER(OracleParams), dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, dp,
                                    ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_ulonglong, dp]
    L.oracle_run_forced_fields.argtypes = L.oracle_run_forced.argtypes[:-1] + [ctypes.c_int, ctypes.c_int, dp]
    u32p = ctypes.POINTER(ctypes.c_uint32)
    L.oracle_philox.argtypes = [u32p, u32p, u32p]
    _LIBS[kind] = L
    return L


def _params(p, nthreads: int = 0) -> OracleParams:
    return OracleParams(p.model, p.integrator, p.nx, p.ny, p.NZ, (ctypes.c_double * 3)(*p.L),
                        p.q, p.omega, p.nu, p.eta, p.B0z, p.viscosity_order, p.dt,
                        p.remap, p.quasilinear, nthreads)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fft(x: np.ndarray, forward: bool, kind: str = "strict") -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib(kind).oracle_fft(a.size, 1 if forward else -1, _dp(a))
    return a


def rhs(p, t, dt_lin, lin, mf, kx0=None, kind: str = "strict"):
    """One Model::rhs evaluation -> (Flin, Fmf, linOp[nxy,4,nz])."""
    lin = np.ascontiguousarray(lin, dtype=np.complex128)
    mf = np.ascontiguousarray(mf, dtype=np.complex128)
    Fl = np.zeros_like(lin)
    Fm = np.zeros_like(mf)
    L = np.zeros(lin.shape, dtype=np.float64)
    k = None if kx0 is None else _dp(np.ascontiguousarray(kx0, dtype=np.float64))
    pp = _params(p)
    lib(kind).oracle_rhs(ctypes.byref(pp), t, dt_lin, _dp(lin), _dp(mf), k, _dp(Fl), _dp(Fm), _dp(L))
    return Fl, Fm, L


def diagnostics(p, t, lin, mf, kx0=None, kind: str = "strict") -> np.ndarray:
    lin = np.ascontiguousarray(lin, dtype=np.complex128)
    mf = np.ascontiguousarray(mf, dtype=np.complex128)
    out = np.zeros(14)
    k = None if kx0 is None else _dp(np.ascontiguousarray(kx0, dtype=np.float64))
    pp = _params(p)
    lib(kind).oracle_diagnostics(ctypes.byref(pp), t, _dp(lin), _dp(mf), k, _dp(out))
    return out


def run(p, t0, lin, mf, kx0, nsteps, diag_every=0, kind: str = "strict", nthreads: int = 0):
    """main.cpp loop for nsteps -> (t, lin, mf, kx0, diag[nrec, 15])."""
    lin = np.ascontiguousarray(lin, dtype=np.complex128).copy()
    mf = np.ascontiguousarray(mf, dtype=np.complex128).copy()
    kx0 = np.ascontiguousarray(kx0, dtype=np.float64).copy()
    t = np.array([t0], dtype=np.float64)
    maxd = (nsteps + 2) if diag_every > 0 else 1
    diag = np.zeros((maxd, 15))
    pp = _params(p, nthreads)
    n = lib(kind).oracle_run(ctypes.byref(pp), _dp(t), _dp(lin), _dp(mf), _dp(kx0), nsteps,
                             diag_every, _dp(diag), maxd)
    return float(t[0]), lin, mf, kx0, diag[:n]


def run_forced(p, t0, lin, mf, kx0, nsteps, diag_every=0, cfl=0.0, dt_max=0.0, f_noise=0.0, k_lo=0.0,
               k_hi=0.0, seed=0, kind: str = "strict", drive_only_velocity=False, drive_only_magnetic=False):
    """main.cpp loop with variable dt (cfl > 0) and driving noise (f_noise != 0); a
    record after every diag_every-th step -> (t, lin, mf, kx0, diag[nrec, 15], dt_mean).
    drive_only_velocity / drive_only_magnetic: the MHD_FullQlin switches
    (MHD_FullQlin.cpp:21-22)."""
    lin = np.ascontiguousarray(lin, dtype=np.complex128).copy()
    mf = np.ascontiguousarray(mf, dtype=np.complex128).copy()
    kx0 = np.ascontiguousarray(kx0, dtype=np.float64).copy()
    t = np.array([t0], dtype=np.float64)
    maxd = (nsteps + 2) if diag_every > 0 else 1
    diag = np.zeros((maxd, 15))
    dtm = np.zeros(1)
    pp = _params(p)
    n = lib(kind).oracle_run_forced_fields(ctypes.byref(pp), _dp(t), _dp(lin), _dp(mf), _dp(kx0), nsteps,
                                           diag_every, _dp(diag), maxd, cfl, dt_max, f_noise, k_lo, k_hi, seed,
                                           int(bool(drive_only_velocity)), int(bool(drive_only_magnetic)), _dp(dtm))
    return float(t[0]), lin, mf, kx0, diag[:n], float(dtm[0])


def philox(ctr, key, kind: str = "strict"):
    """Philox4x32-10 of one counter (4 x uint32) under a key (2 x uint32)."""
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    lib(kind).oracle_philox(c.ctypes.data_as(u32p), k.ctypes.data_as(u32p), out.ctypes.data_as(u32p))
    return out


def tlm_maxwell(p, t0, lin, mf, kx0, dlin, dmf=None, nsteps: int = 1, kind: str = "strict"):
    """Tangent-linear run (MHD_BQlin with RK3CN_Elin or RK3CN): (J, dJ) with J the mean
    over the steps of the fluctuation Maxwell stress and dJ its derivative along (dlin, dmf)."""
    lin = np.ascontiguousarray(lin, dtype=np.complex128)
    mf = np.ascontiguousarray(mf, dtype=np.complex128)
    dlin = np.ascontiguousarray(dlin, dtype=np.complex128)
    k = None if kx0 is None else _dp(np.ascontiguousarray(kx0, dtype=np.float64))
    dm = None if dmf is None else _dp(np.ascontiguousarray(dmf, dtype=np.complex128))
    J = np.zeros(1)
    dJ = np.zeros(1)
    pp = _params(p)
    rc = lib(kind).oracle_tlm_maxwell(ctypes.byref(pp), t0, _dp(lin), _dp(mf), k, _dp(dlin), dm, nsteps,
                                      _dp(J), _dp(dJ))
    if rc:
        raise ValueError("the tangent-linear oracle covers MHD_BQlin")
    return float(J[0]), float(dJ[0])
