"""Python host API over the C ABI: the reference's Model / Integrator /
solution objects for the quasi-linear step, running on the B200.

``QLSolver`` owns one libqlgpu handle (device state + stream).  The thin
classes below mirror the reference names so that a driver written against
QL_DNS/main.cpp reads the same:

* ``MHD_BQlin`` / ``MHD_FullQlin`` - Model (QL_DNS/Models/Model.h:24-112):
  ``rhs``, ``Dimxy``, ``NZ``, ``NZfull``, ``num_MFs``, ``num_Lin``,
  ``Calc_Energy_AM_Diss``;
* ``RK3CN_Elin`` / ``RK3CN`` - Integrator (QL_DNS/Integrators/Integrator.h:20-28):
  ``Step(t, sol) -> dt``, ``mean_time_step``;
* ``solution`` - state container (QL_DNS/solution.h:23-49): ``pLin(i, V)``,
  ``pMF(i)``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from .params import (INTEGRATOR_RK3_CN, INTEGRATOR_RK3_EXP, MODEL_BQLIN, MODEL_FULLQLIN, QLParams)


class QLSolver:
    """One quasi-linear case resident on a GPU."""

    def __init__(self, p: QLParams, device: int = -1):
        self.p = p
        self.L = _capi.load()
        h = ctypes.c_void_p()
        cp = _capi.to_c(p)
        _capi.check(self.L.qlgpu_create(ctypes.byref(cp), device, ctypes.byref(h)), None)
        self.h = h
        nxy, nlin, nz, nmf = (ctypes.c_int() for _ in range(4))
        self.L.qlgpu_dims(h, ctypes.byref(nxy), ctypes.byref(nlin), ctypes.byref(nz), ctypes.byref(nmf))
        self.nxy, self.nlin, self.nz, self.nmf = nxy.value, nlin.value, nz.value, nmf.value

    def close(self):
        if getattr(self, "h", None):
            self.L.qlgpu_destroy(self.h)
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

    # -- state -------------------------------------------------------------
    def set_state(self, t: float, lin: np.ndarray, mf: np.ndarray, kx0: np.ndarray | None = None):
        lin = np.ascontiguousarray(lin, dtype=np.complex128)
        mf = np.ascontiguousarray(mf, dtype=np.complex128)
        assert lin.shape == (self.nxy, 4, self.nz) and mf.shape == (self.nmf, self.nz)
        k = None
        if kx0 is not None:
            kx0 = np.ascontiguousarray(kx0, dtype=np.float64)
            k = _capi.dptr(kx0)
        _capi.check(self.L.qlgpu_set_state(self.h, float(t), _capi.dptr(lin), _capi.dptr(mf), k), self.h)

    def get_state(self):
        lin = np.empty((self.nxy, 4, self.nz), dtype=np.complex128)
        mf = np.empty((self.nmf, self.nz), dtype=np.complex128)
        kx0 = np.empty(self.nxy)
        t = ctypes.c_double()
        _capi.check(self.L.qlgpu_get_state(self.h, ctypes.byref(t), _capi.dptr(lin), _capi.dptr(mf),
                                           _capi.dptr(kx0)), self.h)
        return t.value, lin, mf, kx0

    def set_state_device(self, t: float, lin_ptr: int, mf_ptr: int, kx0_ptr: int | None = None):
        _capi.check(self.L.qlgpu_set_state_device(self.h, float(t), ctypes.c_void_p(lin_ptr),
                                                  ctypes.c_void_p(mf_ptr),
                                                  None if kx0_ptr is None else ctypes.c_void_p(kx0_ptr)), self.h)

    def get_state_device(self, lin_ptr: int, mf_ptr: int, kx0_ptr: int | None = None) -> float:
        t = ctypes.c_double()
        _capi.check(self.L.qlgpu_get_state_device(self.h, ctypes.byref(t), ctypes.c_void_p(lin_ptr),
                                                  ctypes.c_void_p(mf_ptr),
                                                  None if kx0_ptr is None else ctypes.c_void_p(kx0_ptr)), self.h)
        return t.value

    # -- time stepping -------------------------------------------------------
    def step(self, nsteps: int, diag_every: int = 0) -> np.ndarray:
        """main.cpp loop body nsteps times; returns diagnostic records [n, 15]."""
        if diag_every > 0:
            cap = nsteps // diag_every + 2
            out = np.zeros((cap, 15))
            n = ctypes.c_int()
            _capi.check(self.L.qlgpu_step(self.h, int(nsteps), int(diag_every), _capi.dptr(out), cap,
                                          ctypes.byref(n)), self.h)
            return out[: n.value]
        _capi.check(self.L.qlgpu_step(self.h, int(nsteps), 0, None, 0, None), self.h)
        return np.zeros((0, 15))

    def set_noise(self, f_noise: float, k_low: float, k_high: float, seed: int = 0,
                  drive_only_velocity: bool = False, drive_only_magnetic: bool = False):
        """Model::DrivingNoise after every step; f_noise = 0 turns it off.  MHD_FullQlin also
        drives ky = 0 modes in conjugate pairs and takes the drive_only_* switches."""
        _capi.check(self.L.qlgpu_set_noise(self.h, float(f_noise), float(k_low), float(k_high), int(seed)), self.h)
        _capi.check(self.L.qlgpu_set_noise_fields(self.h, int(bool(drive_only_velocity)),
                                                  int(bool(drive_only_magnetic))), self.h)

    def set_cfl(self, cfl: float, dt_max: float = 0.0):
        """Variable dt = cfl / Calculate_CFL capped at dt_max (cfl = 0: fixed dt)."""
        _capi.check(self.L.qlgpu_set_cfl(self.h, float(cfl), float(dt_max)), self.h)

    def mean_time_step(self) -> float:
        """Integrator::mean_time_step(): mean dt since set_state."""
        v = ctypes.c_double()
        _capi.check(self.L.qlgpu_mean_time_step(self.h, ctypes.byref(v)), self.h)
        return v.value

    def step_timed(self) -> np.ndarray:
        """One step; returns the device time (ms) of each of its three stage kernels."""
        ms = (ctypes.c_float * 3)()
        _capi.check(self.L.qlgpu_step_timed(self.h, ms), self.h)
        return np.array(list(ms), dtype=np.float64)

    def diagnostics(self) -> np.ndarray:
        out = np.zeros(15)
        _capi.check(self.L.qlgpu_diagnostics(self.h, _capi.dptr(out)), self.h)
        return out

    def rhs(self, t: float, dt_lin: float, lin: np.ndarray, mf: np.ndarray, want_linop: bool = True):
        lin = np.ascontiguousarray(lin, dtype=np.complex128)
        mf = np.ascontiguousarray(mf, dtype=np.complex128)
        F = np.empty_like(lin)
        Fm = np.empty_like(mf)
        Lop = np.empty(lin.shape) if want_linop else None
        _capi.check(self.L.qlgpu_rhs(self.h, float(t), float(dt_lin), _capi.dptr(lin), _capi.dptr(mf),
                                     _capi.dptr(F), _capi.dptr(Fm), None if Lop is None else _capi.dptr(Lop)),
                    self.h)
        return F, Fm, Lop

    def adjoint_maxwell(self, t0: float, lin0: np.ndarray, mf0: np.ndarray, kx0: np.ndarray | None, nsteps: int,
                        checkpoint_every: int = 100):
        """J = mean over nsteps steps of the fluctuation Maxwell stress, and dJ/d lin0, dJ/d mf0
        (qlgpu_adjoint_maxwell).  Returns (J, grad_lin, grad_mf)."""
        lin0 = np.ascontiguousarray(lin0, dtype=np.complex128)
        mf0 = np.ascontiguousarray(mf0, dtype=np.complex128)
        k = None
        if kx0 is not None:
            kx0 = np.ascontiguousarray(kx0, dtype=np.float64)
            k = _capi.dptr(kx0)
        J = ctypes.c_double()
        gl = np.empty_like(lin0)
        gm = np.empty_like(mf0)
        _capi.check(self.L.qlgpu_adjoint_maxwell(self.h, float(t0), _capi.dptr(lin0), _capi.dptr(mf0), k, int(nsteps),
                                                 int(checkpoint_every), ctypes.byref(J), _capi.dptr(gl),
                                                 _capi.dptr(gm)), self.h)
        return J.value, gl, gm

    @staticmethod
    def adjoint_maxwell_batch(solvers, t0: float, lin0s, mf0s, kx0s, nsteps: int, checkpoint_every: int = 100):
        """qlgpu_adjoint_maxwell for several initial states at once, one solver (handle and
        stream) per seed; the seeds' sweeps run concurrently.  Returns (J[n], grad_lin[n], grad_mf[n])."""
        n = len(solvers)
        lin = np.ascontiguousarray(np.stack(lin0s), dtype=np.complex128)
        mf = np.ascontiguousarray(np.stack(mf0s), dtype=np.complex128)
        k = None
        if kx0s is not None:
            kx = np.ascontiguousarray(np.stack(kx0s), dtype=np.float64)
            k = _capi.dptr(kx)
        hs = (ctypes.c_void_p * n)(*[s.h.value for s in solvers])
        J = np.zeros(n)
        gl = np.empty_like(lin)
        gm = np.empty_like(mf)
        L = solvers[0].L
        _capi.check(L.qlgpu_adjoint_maxwell_batch(hs, n, float(t0), _capi.dptr(lin), _capi.dptr(mf), k, int(nsteps),
                                                  int(checkpoint_every), _capi.dptr(J), _capi.dptr(gl),
                                                  _capi.dptr(gm)), solvers[0].h)
        return J, gl, gm

    def launch_info(self) -> dict:
        a = (ctypes.c_int * 8)()
        _capi.check(self.L.qlgpu_launch_info(self.h, a), self.h)
        keys = ["grid", "block", "smem", "ctas_per_sm", "tmem_cols", "threads_per_transform", "modes", "warps"]
        return dict(zip(keys, list(a)))

    def kernel_attrs(self) -> dict:
        a = (ctypes.c_int * 8)()
        _capi.check(self.L.qlgpu_kernel_attrs(self.h, a), self.h)
        keys = ["regs", "static_smem", "local_bytes", "max_threads", "ctas_per_sm_no_dyn_smem",
                "ctas_per_sm", "max_dyn_smem", "carveout"]
        return dict(zip(keys, list(a)))

    def status(self) -> int:
        s = ctypes.c_int()
        _capi.check(self.L.qlgpu_status(self.h, ctypes.byref(s)), self.h)
        return s.value

    def time(self) -> float:
        t = ctypes.c_double()
        _capi.check(self.L.qlgpu_time(self.h, ctypes.byref(t)), self.h)
        return t.value

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _capi.check(self.L.qlgpu_stream(self.h, ctypes.byref(s)), self.h)
        return s.value or 0


# ---------------------------------------------------------------------------
# Reference-named mirrors
# ---------------------------------------------------------------------------
class solution:
    """Host-side solution container (QL_DNS/solution.h:23-49)."""

    def __init__(self, model: "_Model"):
        p = model.p
        self.lin = np.zeros((p.nxy, 4, p.nz), dtype=np.complex128)
        self.mf = np.zeros((p.nmf, p.nz), dtype=np.complex128)

    def pLin(self, i: int, V: int) -> np.ndarray:
        return self.lin[i, V]

    def pMF(self, i: int) -> np.ndarray:
        return self.mf[i]


class _Model:
    equations_name = ""
    model_id = MODEL_BQLIN

    def __init__(self, p: QLParams):
        self.p = p.replace(model=self.model_id)
        self._solver = None

    def _ensure(self):
        if self._solver is None:
            self._solver = QLSolver(self.p)
        return self._solver

    def Dimxy(self):
        return self.p.nxy

    def Dimxy_full(self):
        return self.p.nxy

    def NZ(self):
        return self.p.nz

    def NZfull(self):
        return self.p.NZ

    def num_MFs(self):
        return self.p.nmf

    def num_Lin(self):
        return 4

    def rhs(self, t, dt_lin, SolIn: solution, SolOut: solution, linOpFluct=None):
        F, Fm, Lop = self._ensure().rhs(t, dt_lin, SolIn.lin, SolIn.mf, want_linop=linOpFluct is not None)
        SolOut.lin[...] = F
        SolOut.mf[...] = Fm
        if linOpFluct is not None:
            linOpFluct[...] = Lop

    def Calc_Energy_AM_Diss(self, t, sol: solution, kx0=None):
        s = self._ensure()
        s.set_state(t, sol.lin, sol.mf, kx0)
        return s.diagnostics()


class MHD_BQlin(_Model):
    equations_name = "MHD_BQlin"
    model_id = MODEL_BQLIN


class MHD_FullQlin(_Model):
    equations_name = "MHD_FullQlin"
    model_id = MODEL_FULLQLIN


class _Integrator:
    integ_id = INTEGRATOR_RK3_EXP

    def __init__(self, t0: float, p: QLParams, model: _Model):
        self.p = model.p.replace(integrator=self.integ_id, dt=p.dt)
        self.solver = QLSolver(self.p)
        self.t0 = t0
        self._bound = None
        self.step_count = 0

    def Step(self, t: float, sol: solution) -> float:
        """Advance sol by one step from time t (state stays on the device
        between calls with the same solution object)."""
        if self._bound is not sol or abs(self.solver.time() - t) > 0:
            self.solver.set_state(t, sol.lin, sol.mf)
            self._bound = sol
        self.solver.step(1)
        _, sol.lin[...], sol.mf[...], _ = self.solver.get_state()
        self.step_count += 1
        return self.p.dt

    def mean_time_step(self) -> float:
        return self.p.dt


class RK3CN_Elin(_Integrator):
    integ_id = INTEGRATOR_RK3_EXP


class RK3CN(_Integrator):
    integ_id = INTEGRATOR_RK3_CN


def main(argv=None):
    """One case through the single-case path:

        python -m ql_dns_b200.solver [--case production|small] [--steps 20] [--diag-every 0]

    production: 64x64 modes x NZ=128 (Re=Rm=8000, dt=0.005, seed 1); small: 16x16 x NZ=32
    (Re=Rm=2000, dt=0.01, seed 0).  Prints the device time per step (CUDA events of the
    three stage kernels) and the last diagnostic record as JSON."""
    import argparse
    import json
    from .initial import initial_state
    from .params import mri_16x16_nz32, mri_64x64_nz128
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="production", choices=["production", "small"])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--diag-every", type=int, default=0)
    a = ap.parse_args(argv)
    p, seed = (mri_64x64_nz128(), 1) if a.case == "production" else (mri_16x16_nz32(), 0)
    lin, mf, kx0 = initial_state(p, seed, sigma=1e-3)
    with QLSolver(p) as s:
        s.set_state(0.0, lin, mf, kx0)
        ms = np.zeros(3)
        for _ in range(a.steps):
            ms += s.step_timed()
        rec = s.step(a.diag_every, diag_every=1) if a.diag_every else s.diagnostics()[None]
        print(json.dumps({"case": a.case, "steps": a.steps, "ms_per_step": float(ms.sum() / max(a.steps, 1)),
                          "stage_ms": list(ms / max(a.steps, 1)), "launch": s.launch_info(),
                          "last_record": list(rec[-1])}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
