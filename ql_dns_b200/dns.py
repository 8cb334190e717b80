"""Python host API of the full 3-D shearing-box MHD DNS (include/qlgpu_dns.h).

``QLDns`` owns one ``qlgpu_dns`` handle (device state + stream).  Its methods
follow ``QLSolver``: ``set_state`` / ``get_state`` / ``step`` /
``diagnostics`` / ``rhs``, with the state as columns lin[nxy, 6, nz] =
(u_x, u_y, u_z, b_x, b_y, b_z) in the Kdata mode order of the QL models
(QL_DNS/Auxiliary/Kdata.cpp:30-46) and column 0 holding the mean fields.
There is no CPU path: without the library or a device every call raises.

    python -m ql_dns_b200.dns [--steps 1000] [--diag-every 100]

runs the 64 x 128 x 64 MRI case (Re=Rm=4000, dt=0.005, seed 2) and prints the
energy / stress record every --diag-every steps as JSON lines.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import _capi
from .params import DNSParams, dns_64x128x64


class QLDns:
    def __init__(self, p: DNSParams, device: int = -1):
        self.p = p
        self.L = _capi.load()
        h = ctypes.c_void_p()
        cp = _capi.to_c_dns(p)
        _capi.check_dns(self.L.qlgpu_dns_create(ctypes.byref(cp), device, ctypes.byref(h)), None)
        self.h = h
        nxy, nz, nx, ny = (ctypes.c_int() for _ in range(4))
        self.L.qlgpu_dns_dims(h, ctypes.byref(nxy), ctypes.byref(nz), ctypes.byref(nx), ctypes.byref(ny))
        self.nxy, self.nz, self.nx, self.ny = nxy.value, nz.value, nx.value, ny.value

    def close(self):
        if getattr(self, "h", None):
            self.L.qlgpu_dns_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, t: float, lin: np.ndarray, kx0: np.ndarray | None = None):
        lin = np.ascontiguousarray(lin, dtype=np.complex128)
        assert lin.shape == (self.nxy, 6, self.nz)
        k = None
        if kx0 is not None:
            kx0 = np.ascontiguousarray(kx0, dtype=np.float64)
            k = _capi.dptr(kx0)
        _capi.check_dns(self.L.qlgpu_dns_set_state(self.h, float(t), _capi.dptr(lin), k), self.h)

    def get_state(self):
        lin = np.empty((self.nxy, 6, self.nz), dtype=np.complex128)
        kx0 = np.empty(self.nxy)
        t = ctypes.c_double()
        _capi.check_dns(self.L.qlgpu_dns_get_state(self.h, ctypes.byref(t), _capi.dptr(lin), _capi.dptr(kx0)),
                        self.h)
        return t.value, lin, kx0

    def step(self, nsteps: int, diag_every: int = 0) -> np.ndarray | None:
        nd = ctypes.c_int()
        if diag_every:
            cap = nsteps // diag_every
            out = np.zeros((max(cap, 1), 15))
            _capi.check_dns(self.L.qlgpu_dns_step(self.h, nsteps, diag_every, _capi.dptr(out), cap,
                                                  ctypes.byref(nd)), self.h)
            return out[:nd.value]
        _capi.check_dns(self.L.qlgpu_dns_step(self.h, nsteps, 0, None, 0, ctypes.byref(nd)), self.h)
        return None

    def step_timed(self, nsteps: int) -> float:
        ms = ctypes.c_float()
        _capi.check_dns(self.L.qlgpu_dns_step_timed(self.h, nsteps, ctypes.byref(ms)), self.h)
        return ms.value

    def diagnostics(self) -> np.ndarray:
        out = np.zeros(15)
        _capi.check_dns(self.L.qlgpu_dns_diagnostics(self.h, _capi.dptr(out)), self.h)
        return out

    def rhs(self, t: float) -> np.ndarray:
        F = np.empty((self.nxy, 6, self.nz), dtype=np.complex128)
        _capi.check_dns(self.L.qlgpu_dns_rhs(self.h, float(t), _capi.dptr(F)), self.h)
        return F

    def status(self) -> int:
        st = ctypes.c_int()
        _capi.check_dns(self.L.qlgpu_dns_status(self.h, ctypes.byref(st)), self.h)
        return st.value

    def stream(self) -> int:
        return self.L.qlgpu_dns_stream(self.h) or 0


def main(argv=None):
    from .initial import dns_initial_state
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--diag-every", type=int, default=100)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--integrator", type=int, default=0)
    a = ap.parse_args(argv)
    p = dns_64x128x64(integrator=a.integrator)
    lin, kx0 = dns_initial_state(p, a.seed, sigma=1e-2, B0=0.05)
    with QLDns(p) as d:
        d.set_state(0.0, lin, kx0)
        t0 = time.perf_counter()
        recs = d.step(a.steps, diag_every=a.diag_every)
        wall = time.perf_counter() - t0
        for r in recs:
            print(json.dumps({"t": r[0], "energy": list(r[1:5]), "AM": list(r[5:9]), "diss": list(r[9:13])}))
        print(json.dumps({"steps": a.steps, "wall_s": wall, "ms_per_step": 1e3 * wall / max(a.steps, 1),
                          "grid": [p.Mx, p.My, p.NZ], "modes": d.nxy, "nz": d.nz}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
