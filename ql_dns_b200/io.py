"""Output and restart files in the reference's layouts (include/qlgpu_io.h).

* ``TimeVariables``: the binary ``energy.dat``, ``angular_momentum.dat``,
  ``dissipation.dat``, ``reynolds_stress.dat``, ``time_vec.dat`` and
  ``mean_fields.dat`` files of QL_DNS/Auxiliary/TimeVariables.cpp, written from
  the diagnostic records of a step call.
* ``save_solution`` / ``load_solution``: the groups of
  QL_DNS/Auxiliary/FullSave_Load.cpp (``/t=<t>`` with ``Ind j: kx a ky b``,
  ``Mean`` and ``kx`` datasets, float32) in a raw binary container, since HDF5
  is not available to this build.

Host-only: no GPU is needed.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from .params import MODEL_BQLIN, QLParams

# Model::num_reynolds_saves (MHD_BQlin.h:41; MHD_FullQlin.cpp:56-58 without full stresses)
NUM_REYNOLDS = {MODEL_BQLIN: 5, 1: 4}


class TimeVariables:
    def __init__(self, directory: str, p: QLParams, append: bool = False):
        self.L = _capi.load()
        self.p = p
        h = ctypes.c_void_p()
        _capi.check_io(self.L.qlgpu_timevars_open(directory.encode(), p.nmf, p.NZ, NUM_REYNOLDS[p.model],
                                                  1 if append else 0, ctypes.byref(h)))
        self.h = h

    def save_data(self, rec15: np.ndarray):
        r = np.ascontiguousarray(rec15, dtype=np.float64)
        assert r.shape == (15,)
        _capi.check_io(self.L.qlgpu_timevars_save_data(self.h, _capi.dptr(r)))

    def save_mean_fields(self, mf: np.ndarray):
        m = np.ascontiguousarray(mf, dtype=np.complex128)
        assert m.shape == (self.p.nmf, self.p.nz)
        _capi.check_io(self.L.qlgpu_timevars_save_mean_fields(self.h, _capi.dptr(m), self.p.nz))

    def close(self):
        if getattr(self, "h", None):
            self.L.qlgpu_timevars_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def save_solution(path: str, p: QLParams, t: float, lin: np.ndarray, mf: np.ndarray, kx0: np.ndarray):
    L = _capi.load()
    cp = _capi.to_c(p)
    lin = np.ascontiguousarray(lin, dtype=np.complex128)
    mf = np.ascontiguousarray(mf, dtype=np.complex128)
    kx0 = np.ascontiguousarray(kx0, dtype=np.float64)
    _capi.check_io(L.qlgpu_fullsave_write(path.encode(), ctypes.byref(cp), float(t), _capi.dptr(lin),
                                          _capi.dptr(mf), _capi.dptr(kx0)))


def load_solution(path: str, p: QLParams):
    """The latest saved group: (t, lin, mf, kx0)."""
    L = _capi.load()
    cp = _capi.to_c(p)
    lin = np.empty((p.nxy, 4, p.nz), dtype=np.complex128)
    mf = np.empty((p.nmf, p.nz), dtype=np.complex128)
    kx0 = np.empty(p.nxy)
    t = ctypes.c_double()
    _capi.check_io(L.qlgpu_fullsave_read_latest(path.encode(), ctypes.byref(cp), ctypes.byref(t), _capi.dptr(lin),
                                                _capi.dptr(mf), _capi.dptr(kx0)))
    return t.value, lin, mf, kx0


def saved_times(path: str) -> list[float]:
    L = _capi.load()
    n = ctypes.c_int()
    _capi.check_io(L.qlgpu_fullsave_times(path.encode(), None, 0, ctypes.byref(n)))
    ts = np.zeros(max(n.value, 1))
    _capi.check_io(L.qlgpu_fullsave_times(path.encode(), _capi.dptr(ts), n.value, ctypes.byref(n)))
    return list(ts[: n.value])
