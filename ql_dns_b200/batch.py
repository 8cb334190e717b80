"""Batched ensemble of quasi-linear cases on one GPU (qlgpu_batch_* of include/qlgpu.h).

Many independent cases (their own mode grid, NZ, nu, eta, mean field) step
together in one persistent cooperative kernel launch per call.  The reference
runs one case per MPI job (QL_DNS/main.cpp); per case the arithmetic is the
same fused RK3 step as ``QLSolver``.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _capi
from .params import QLParams


class QLBatch:
    """A batch of cases resident on one GPU."""

    def __init__(self, cases: list[QLParams], device: int = -1):
        self.cases = list(cases)
        self._pending = []  # max_diag of each outstanding step_async call
        self.L = _capi.load()
        arr = (_capi.qlgpu_params * len(cases))(*[_capi.to_c(p) for p in cases])
        b = ctypes.c_void_p()
        _capi.check_batch(self.L.qlgpu_batch_create(arr, len(cases), device, ctypes.byref(b)), None)
        self.b = b
        self.dims = []
        for c in range(len(cases)):
            nxy, nz, nmf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            self.L.qlgpu_batch_dims(b, c, ctypes.byref(nxy), ctypes.byref(nz), ctypes.byref(nmf))
            self.dims.append((nxy.value, nz.value, nmf.value))

    def close(self):
        if getattr(self, "b", None):
            self.L.qlgpu_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __len__(self):
        return len(self.cases)

    # -- state ---------------------------------------------------------------
    def set_state(self, c: int, t: float, lin: np.ndarray, mf: np.ndarray, kx0: np.ndarray | None = None):
        nxy, nz, nmf = self.dims[c]
        lin = np.ascontiguousarray(lin, dtype=np.complex128)
        mf = np.ascontiguousarray(mf, dtype=np.complex128)
        assert lin.shape == (nxy, 4, nz) and mf.shape == (nmf, nz)
        k = None
        if kx0 is not None:
            kx0 = np.ascontiguousarray(kx0, dtype=np.float64)
            k = _capi.dptr(kx0)
        _capi.check_batch(self.L.qlgpu_batch_set_state(self.b, c, float(t), _capi.dptr(lin), _capi.dptr(mf), k),
                          self.b)

    def get_state(self, c: int):
        nxy, nz, nmf = self.dims[c]
        lin = np.empty((nxy, 4, nz), dtype=np.complex128)
        mf = np.empty((nmf, nz), dtype=np.complex128)
        kx0 = np.empty(nxy)
        t = ctypes.c_double()
        _capi.check_batch(self.L.qlgpu_batch_get_state(self.b, c, ctypes.byref(t), _capi.dptr(lin), _capi.dptr(mf),
                                                       _capi.dptr(kx0)), self.b)
        return t.value, lin, mf, kx0

    def set_states(self, t: float, states):
        """Every case's (lin, mf, kx0) at once (kx0 may be None); one synchronisation.  Pinned
        host arrays (e.g. from torch pin_memory) copy asynchronously."""
        nc = len(self.cases)
        arrs = []
        P = ctypes.POINTER(ctypes.c_double)
        lp, mp, kp = (P * nc)(), (P * nc)(), (P * nc)()
        for c, (lin, mf, kx0) in enumerate(states):
            nxy, nz, nmf = self.dims[c]
            lin = np.ascontiguousarray(lin, dtype=np.complex128)
            mf = np.ascontiguousarray(mf, dtype=np.complex128)
            assert lin.shape == (nxy, 4, nz) and mf.shape == (nmf, nz)
            arrs += [lin, mf]
            lp[c], mp[c] = _capi.dptr(lin), _capi.dptr(mf)
            if kx0 is not None:
                kx0 = np.ascontiguousarray(kx0, dtype=np.float64)
                arrs.append(kx0)
                kp[c] = _capi.dptr(kx0)
        _capi.check_batch(self.L.qlgpu_batch_set_states(self.b, float(t), lp, mp, kp), self.b)

    def get_states(self, out=None):
        """Every case's (t, lin, mf, kx0); `out` = per-case (lin, mf, kx0) host arrays to fill
        (pinned for asynchronous copies), else new arrays."""
        nc = len(self.cases)
        if out is None:
            out = [(np.empty((d[0], 4, d[1]), dtype=np.complex128), np.empty((d[2], d[1]), dtype=np.complex128),
                    np.empty(d[0])) for d in self.dims]
        P = ctypes.POINTER(ctypes.c_double)
        lp, mp, kp = (P * nc)(), (P * nc)(), (P * nc)()
        for c, (lin, mf, kx0) in enumerate(out):
            lp[c], mp[c], kp[c] = _capi.dptr(lin), _capi.dptr(mf), _capi.dptr(kx0)
        t = np.zeros(nc)
        _capi.check_batch(self.L.qlgpu_batch_get_states(self.b, _capi.dptr(t), lp, mp, kp), self.b)
        return [(t[c], lin, mf, kx0) for c, (lin, mf, kx0) in enumerate(out)]

    def diagnostics(self, c: int) -> np.ndarray:
        out = np.zeros(15)
        _capi.check_batch(self.L.qlgpu_batch_diagnostics(self.b, c, _capi.dptr(out)), self.b)
        return out

    # -- stepping ------------------------------------------------------------
    def step(self, nsteps: int, diag_every: int = 0) -> list[np.ndarray]:
        """nsteps steps of every case; per case the diagnostic records [n, 15]."""
        nc = len(self.cases)
        if diag_every > 0:
            cap = nsteps // diag_every + 2
            out = np.zeros((nc, cap, 15))
            nd = (ctypes.c_int * nc)()
            _capi.check_batch(self.L.qlgpu_batch_step(self.b, int(nsteps), int(diag_every), _capi.dptr(out), cap, nd),
                              self.b)
            return [out[c, : nd[c]] for c in range(nc)]
        _capi.check_batch(self.L.qlgpu_batch_step(self.b, int(nsteps), 0, None, 0, None), self.b)
        return [np.zeros((0, 15)) for _ in range(nc)]

    def step_async(self, nsteps: int, diag_every: int = 0) -> None:
        """Queues nsteps steps of every case and returns at once (at most two outstanding);
        step_collect() returns the oldest call's records."""
        cap = nsteps // diag_every + 2 if diag_every > 0 else 0
        _capi.check_batch(self.L.qlgpu_batch_step_async(self.b, int(nsteps), int(diag_every), cap), self.b)
        self._pending.append(cap)

    def step_collect(self) -> list[np.ndarray]:
        """Waits for the oldest step_async call; per case its diagnostic records [n, 15]."""
        nc = len(self.cases)
        cap = self._pending.pop(0) if self._pending else 0  # none outstanding: the C call refuses
        if cap > 0:
            out = np.zeros((nc, cap, 15))
            nd = (ctypes.c_int * nc)()
            _capi.check_batch(self.L.qlgpu_batch_step_collect(self.b, _capi.dptr(out), cap, nd), self.b)
            return [out[c, : nd[c]] for c in range(nc)]
        _capi.check_batch(self.L.qlgpu_batch_step_collect(self.b, None, 0, None), self.b)
        return [np.zeros((0, 15)) for _ in range(nc)]

    def step_timed(self, nsteps: int) -> float:
        """nsteps steps without diagnostics; device time of the launch in ms."""
        ms = ctypes.c_float()
        _capi.check_batch(self.L.qlgpu_batch_step_timed(self.b, int(nsteps), ctypes.byref(ms)), self.b)
        return float(ms.value)

    def tune(self, probe_steps: int = 3) -> float:
        best = ctypes.c_double()
        _capi.check_batch(self.L.qlgpu_batch_tune(self.b, int(probe_steps), ctypes.byref(best)), self.b)
        return best.value

    def mapping(self) -> dict:
        """CTA width, grid, CTAs per SM, shared memory and per case its CTAs (work-item engine) or
        chunks per stage (queue engine, with the passes per chunk of NZ = 16, 32, 64, 128)."""
        info = (ctypes.c_int * 4)()
        nc = len(self.cases)
        k = (ctypes.c_int * nc)()
        _capi.check_batch(self.L.qlgpu_batch_mapping(self.b, info, k), self.b)
        out = {"warps": info[0], "grid": info[1], "ctas_per_sm": info[2], "smem": info[3], "ncta": list(k)}
        if self.engine() == "queue":
            p4 = (ctypes.c_int * 4)()
            _capi.check_batch(self.L.qlgpu_batch_chunks(self.b, p4), self.b)
            out["chunk_passes"] = dict(zip([16, 32, 64, 128], list(p4)))
        return out

    def cost_model(self) -> dict:
        """The planner's cost model (fitted by tune()): alpha = us per stage per launch,
        beta = us per work item per stage, r = us per pipeline pass per NZ class."""
        v = (ctypes.c_double * 7)()
        _capi.check_batch(self.L.qlgpu_batch_cost_model(self.b, v), self.b)
        return {"alpha_us": v[0], "beta_us": v[1], "r_us": dict(zip([16, 32, 64, 128, 256], list(v)[2:]))}

    def set_mapping(self, warps: int, ncta: list[int]):
        k = (ctypes.c_int * len(ncta))(*ncta)
        _capi.check_batch(self.L.qlgpu_batch_set_mapping(self.b, int(warps), k), self.b)

    def set_noise(self, c: int, f_noise: float, k_low: float, k_high: float, seed: int = 0,
                  drive_only_velocity: bool = False, drive_only_magnetic: bool = False):
        """Driving noise of case c after every step (as QLSolver.set_noise); f_noise = 0: off."""
        _capi.check_batch(self.L.qlgpu_batch_set_noise(self.b, int(c), float(f_noise), float(k_low), float(k_high),
                                                       int(seed), int(bool(drive_only_velocity)),
                                                       int(bool(drive_only_magnetic))), self.b)

    ENGINES = {"auto": 0, "items": 1, "queue": 2}

    def set_engine(self, engine: str):
        """'queue' (chunk queue: MHD_BQlin, NZ <= 128), 'items' (work items: every case) or 'auto'."""
        _capi.check_batch(self.L.qlgpu_batch_set_engine(self.b, self.ENGINES[engine]), self.b)

    def engine(self) -> str:
        e = ctypes.c_int()
        _capi.check_batch(self.L.qlgpu_batch_engine(self.b, ctypes.byref(e)), self.b)
        return {1: "items", 2: "queue"}[e.value]

    def set_chunks(self, passes: list[int]):
        """Queue engine: CTA passes per chunk for NZ = 16, 32, 64, 128."""
        k = (ctypes.c_int * 4)(*passes)
        _capi.check_batch(self.L.qlgpu_batch_set_chunks(self.b, k), self.b)

    def queue_trace(self) -> dict:
        """Queue engine, QLGPU_TRACE=1: per-CTA averages of the last launch."""
        v = (ctypes.c_double * 4)()
        _capi.check_batch(self.L.qlgpu_batch_queue_trace(self.b, v), self.b)
        return {"wait_us": v[0], "chunk_us": v[1], "mean_field_us": v[2], "chunks": v[3]}

    def status(self):
        nc = len(self.cases)
        st = (ctypes.c_int * nc)()
        ls = ctypes.c_int()
        _capi.check_batch(self.L.qlgpu_batch_status(self.b, st, ctypes.byref(ls)), self.b)
        return list(st), ls.value

    def set_wait(self, seconds: float):
        _capi.check_batch(self.L.qlgpu_batch_set_wait(self.b, float(seconds)), self.b)

    def debug_drop_item(self, c: int):
        """Failure-detection test aid (qlgpu_batch_debug_drop_item)."""
        _capi.check_batch(self.L.qlgpu_batch_debug_drop_item(self.b, int(c)), self.b)

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _capi.check_batch(self.L.qlgpu_batch_stream(self.b, ctypes.byref(s)), self.b)
        return s.value or 0


# Mode grids, NZ and Pm of the ensemble law.
ENSEMBLE_GRIDS = (16, 32, 48, 64)
ENSEMBLE_NZ = (32, 64, 128)
ENSEMBLE_PM = (1, 2, 4)


def mri_ensemble(ncases: int = 48, draw_seed: int = 12345, dt: float = 0.01, **kw):
    """The QL MRI ensemble: per case a square mode grid from {16, 32, 48, 64},
    NZ from {32, 64, 128}, Rm log-uniform in [500, 16000], Pm from {1, 2, 4}
    (eta = 1/Rm, nu = Pm/Rm, as Python/WriteMRIDNSinput.py:22-23 sets them) and
    a mean-field amplitude B0 uniform in [0.01, 0.1], all drawn from one numpy
    generator seeded with draw_seed.  Case c uses initial-condition seed c.

    Returns (cases, b0s, seeds)."""
    rng = np.random.default_rng(draw_seed)
    cases, b0s = [], []
    for _ in range(ncases):
        n = int(rng.choice(ENSEMBLE_GRIDS))
        NZ = int(rng.choice(ENSEMBLE_NZ))
        Rm = float(math.exp(rng.uniform(math.log(500.0), math.log(16000.0))))
        Pm = int(rng.choice(ENSEMBLE_PM))
        B0 = float(rng.uniform(0.01, 0.1))
        cases.append(QLParams(nx=n, ny=n, NZ=NZ, nu=Pm / Rm, eta=1.0 / Rm, dt=dt).replace(**kw))
        b0s.append(B0)
    return cases, b0s, list(range(ncases))
