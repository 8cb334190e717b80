"""ctypes binding of the C ABI declared in include/qlgpu.h (libqlgpu.so).

The library is loaded from the package's ``_lib`` directory.  There is no CPU
fallback: if the library or a CUDA device is missing every call fails loudly.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libqlgpu.so")
# QLGPU_DEBUG=1: the -DQLGPU_DEBUG build (device bounds checks, canary-guarded buffers)
DEBUG_LIB_PATH = os.path.join(HERE, "_lib", "libqlgpu_debug.so")

QLGPU_OK = 0
ERRORS = {1: "QLGPU_ERR_ARG", 2: "QLGPU_ERR_UNSUPPORTED", 3: "QLGPU_ERR_CUDA", 4: "QLGPU_ERR_STATUS",
          5: "QLGPU_ERR_NODEVICE"}

# Every symbol include/qlgpu.h declares.
EXPORTS = ["qlgpu_create", "qlgpu_destroy", "qlgpu_dims", "qlgpu_set_state", "qlgpu_get_state",
           "qlgpu_set_state_device", "qlgpu_get_state_device", "qlgpu_step", "qlgpu_step_timed", "qlgpu_diagnostics",
           "qlgpu_rhs", "qlgpu_rhs_noalloc", "qlgpu_status", "qlgpu_time", "qlgpu_trace", "qlgpu_launch_info", "qlgpu_kernel_attrs",
           "qlgpu_stream",
           "qlgpu_last_error",
           "qlgpu_version",
           "qlgpu_adjoint_maxwell",
           "qlgpu_batch_create", "qlgpu_batch_destroy", "qlgpu_batch_dims", "qlgpu_batch_set_state",
           "qlgpu_batch_get_state", "qlgpu_batch_diagnostics", "qlgpu_batch_step", "qlgpu_batch_step_timed",
           "qlgpu_batch_step_async", "qlgpu_batch_step_collect",
           "qlgpu_batch_tune", "qlgpu_batch_mapping", "qlgpu_batch_set_mapping", "qlgpu_batch_status",
           "qlgpu_batch_set_wait", "qlgpu_batch_debug_drop_item", "qlgpu_batch_stream",
           "qlgpu_batch_last_error", "qlgpu_batch_set_engine", "qlgpu_batch_engine", "qlgpu_batch_set_chunks",
           "qlgpu_batch_queue_trace",
           "qlgpu_batch_set_states", "qlgpu_batch_get_states", "qlgpu_batch_chunks",
           "qlgpu_timevars_open", "qlgpu_timevars_save_data", "qlgpu_timevars_save_mean_fields",
           "qlgpu_timevars_close", "qlgpu_fullsave_write", "qlgpu_fullsave_read_latest", "qlgpu_fullsave_times",
           "qlgpu_io_last_error",
           "qlgpu_dns_create", "qlgpu_dns_destroy", "qlgpu_dns_dims", "qlgpu_dns_set_state", "qlgpu_dns_get_state",
           "qlgpu_dns_step", "qlgpu_dns_diagnostics", "qlgpu_dns_rhs", "qlgpu_dns_status", "qlgpu_dns_last_error",
           "qlgpu_dns_step_timed", "qlgpu_dns_stream", "qlgpu_fp64_peak",
           "qlgpu_set_noise", "qlgpu_set_cfl", "qlgpu_mean_time_step", "qlgpu_adjoint_maxwell_batch",
           "qlgpu_batch_cost_model", "qlgpu_set_noise_fields", "qlgpu_batch_set_noise", "qlgpu_debug_build",
           "qlgpu_debug_guard_poke", "qlgpu_batch_debug_guard_poke"]


class qlgpu_params(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int), ("integrator", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("NZ", ctypes.c_int),
        ("L", ctypes.c_double * 3),
        ("q", ctypes.c_double), ("omega", ctypes.c_double),
        ("nu", ctypes.c_double), ("eta", ctypes.c_double), ("B0z", ctypes.c_double),
        ("viscosity_order", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("remap", ctypes.c_int), ("quasilinear", ctypes.c_int),
    ]


class qlgpu_dns_params(ctypes.Structure):
    _fields_ = [
        ("integrator", ctypes.c_int), ("Mx", ctypes.c_int), ("My", ctypes.c_int), ("NZ", ctypes.c_int),
        ("L", ctypes.c_double * 3),
        ("q", ctypes.c_double), ("omega", ctypes.c_double),
        ("nu", ctypes.c_double), ("eta", ctypes.c_double), ("B0z", ctypes.c_double),
        ("viscosity_order", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("remap", ctypes.c_int), ("dealias_xy", ctypes.c_int),
    ]


class QLGPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load(path: str | None = None):
    """Load libqlgpu.so, or libqlgpu_debug.so when QLGPU_DEBUG=1 (raises if it is
    missing; there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if path is None:
        path = DEBUG_LIB_PATH if os.environ.get("QLGPU_DEBUG") == "1" else LIB_PATH
    if not os.path.exists(path):
        raise QLGPUError(5, f"{path} not built (python -m ql_dns_b200.build)")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    L.qlgpu_create.argtypes = [ctypes.POINTER(qlgpu_params), ctypes.c_int, ctypes.POINTER(vp)]
    L.qlgpu_destroy.argtypes = [vp]
    L.qlgpu_dims.argtypes = [vp, ip, ip, ip, ip]
    L.qlgpu_set_state.argtypes = [vp, ctypes.c_double, dp, dp, dp]
    L.qlgpu_get_state.argtypes = [vp, dp, dp, dp, dp]
    L.qlgpu_set_state_device.argtypes = [vp, ctypes.c_double, vp, vp, vp]
    L.qlgpu_get_state_device.argtypes = [vp, dp, vp, vp, vp]
    L.qlgpu_step.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ip]
    L.qlgpu_step_timed.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.qlgpu_diagnostics.argtypes = [vp, dp]
    L.qlgpu_rhs.argtypes = [vp, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp, dp]
    L.qlgpu_rhs_noalloc.argtypes = [ctypes.POINTER(qlgpu_params), ctypes.c_double, ctypes.c_double,
                                    vp, vp, vp, vp, vp, vp, vp]
    L.qlgpu_status.argtypes = [vp, ip]
    L.qlgpu_time.argtypes = [vp, dp]
    L.qlgpu_trace.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    L.qlgpu_launch_info.argtypes = [vp, ip]
    L.qlgpu_kernel_attrs.argtypes = [vp, ip]
    L.qlgpu_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.qlgpu_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    L.qlgpu_version.restype = ctypes.c_char_p
    L.qlgpu_adjoint_maxwell.argtypes = [vp, ctypes.c_double, dp, dp, dp, ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.qlgpu_batch_create.argtypes = [ctypes.POINTER(qlgpu_params), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.qlgpu_batch_destroy.argtypes = [vp]
    L.qlgpu_batch_dims.argtypes = [vp, ctypes.c_int, ip, ip, ip]
    L.qlgpu_batch_set_state.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp, dp, dp]
    L.qlgpu_batch_get_state.argtypes = [vp, ctypes.c_int, dp, dp, dp, dp]
    L.qlgpu_batch_diagnostics.argtypes = [vp, ctypes.c_int, dp]
    L.qlgpu_batch_step.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ip]
    L.qlgpu_batch_step_timed.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.qlgpu_batch_step_async.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.qlgpu_batch_step_collect.argtypes = [vp, dp, ctypes.c_int, ip]
    L.qlgpu_batch_tune.argtypes = [vp, ctypes.c_int, dp]
    L.qlgpu_batch_mapping.argtypes = [vp, ip, ip]
    L.qlgpu_batch_set_mapping.argtypes = [vp, ctypes.c_int, ip]
    L.qlgpu_batch_status.argtypes = [vp, ip, ip]
    L.qlgpu_batch_set_wait.argtypes = [vp, ctypes.c_double]
    L.qlgpu_batch_debug_drop_item.argtypes = [vp, ctypes.c_int]
    L.qlgpu_batch_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.qlgpu_batch_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    L.qlgpu_batch_set_engine.argtypes = [vp, ctypes.c_int]
    L.qlgpu_batch_engine.argtypes = [vp, ip]
    L.qlgpu_batch_set_chunks.argtypes = [vp, ip]
    L.qlgpu_batch_chunks.argtypes = [vp, ip]
    L.qlgpu_batch_queue_trace.argtypes = [vp, dp]
    dpp = ctypes.POINTER(dp)
    L.qlgpu_batch_set_states.argtypes = [vp, ctypes.c_double, dpp, dpp, dpp]
    L.qlgpu_batch_get_states.argtypes = [vp, dp, dpp, dpp, dpp]
    L.qlgpu_timevars_open.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(vp)]
    L.qlgpu_timevars_save_data.argtypes = [vp, dp]
    L.qlgpu_timevars_save_mean_fields.argtypes = [vp, dp, ctypes.c_int]
    L.qlgpu_timevars_close.argtypes = [vp]
    L.qlgpu_fullsave_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(qlgpu_params), ctypes.c_double, dp, dp, dp]
    L.qlgpu_fullsave_read_latest.argtypes = [ctypes.c_char_p, ctypes.POINTER(qlgpu_params), dp, dp, dp, dp]
    L.qlgpu_fullsave_times.argtypes = [ctypes.c_char_p, dp, ctypes.c_int, ip]
    L.qlgpu_io_last_error.argtypes = [ctypes.c_char_p, ctypes.c_int]
    L.qlgpu_dns_create.argtypes = [ctypes.POINTER(qlgpu_dns_params), ctypes.c_int, ctypes.POINTER(vp)]
    L.qlgpu_dns_destroy.argtypes = [vp]
    L.qlgpu_dns_dims.argtypes = [vp, ip, ip, ip, ip]
    L.qlgpu_dns_set_state.argtypes = [vp, ctypes.c_double, dp, dp]
    L.qlgpu_dns_get_state.argtypes = [vp, dp, dp, dp]
    L.qlgpu_dns_step.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ip]
    L.qlgpu_dns_diagnostics.argtypes = [vp, dp]
    L.qlgpu_dns_rhs.argtypes = [vp, ctypes.c_double, dp]
    L.qlgpu_dns_status.argtypes = [vp, ip]
    L.qlgpu_dns_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    L.qlgpu_dns_step_timed.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.qlgpu_dns_stream.argtypes = [vp]
    L.qlgpu_dns_stream.restype = vp
    L.qlgpu_fp64_peak.argtypes = [ctypes.c_int, dp]
    L.qlgpu_set_noise.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong]
    L.qlgpu_set_noise_fields.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.qlgpu_debug_build.argtypes = []
    L.qlgpu_debug_guard_poke.argtypes = [vp, ctypes.c_int]
    L.qlgpu_batch_debug_guard_poke.argtypes = [vp, ctypes.c_int]
    L.qlgpu_batch_set_noise.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int]
    L.qlgpu_set_cfl.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    L.qlgpu_mean_time_step.argtypes = [vp, dp]
    L.qlgpu_batch_cost_model.argtypes = [vp, dp]
    L.qlgpu_adjoint_maxwell_batch.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_double, dp, dp, dp,
                                              ctypes.c_int, ctypes.c_int, dp, dp, dp]
    for name in EXPORTS:
        if name not in ("qlgpu_version", "qlgpu_dns_stream"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def to_c(p) -> qlgpu_params:
    return qlgpu_params(p.model, p.integrator, p.nx, p.ny, p.NZ, (ctypes.c_double * 3)(*p.L), p.q, p.omega,
                        p.nu, p.eta, p.B0z, p.viscosity_order, p.dt, p.remap, p.quasilinear)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def check(rc: int, h=None):
    if rc != QLGPU_OK:
        L = load()
        buf = ctypes.create_string_buffer(512)
        L.qlgpu_last_error(h, buf, 512)
        raise QLGPUError(rc, buf.value.decode(errors="replace"))


def check_batch(rc: int, b=None):
    """As check() for the qlgpu_batch_* entry points (their own error message)."""
    if rc != QLGPU_OK:
        L = load()
        buf = ctypes.create_string_buffer(512)
        L.qlgpu_batch_last_error(b, buf, 512)
        raise QLGPUError(rc, buf.value.decode(errors="replace"))


def to_c_dns(p) -> qlgpu_dns_params:
    return qlgpu_dns_params(p.integrator, p.Mx, p.My, p.NZ, (ctypes.c_double * 3)(*p.L), p.q, p.omega, p.nu, p.eta,
                            p.B0z, p.viscosity_order, p.dt, p.remap, p.dealias_xy)


def check_dns(rc: int, h=None):
    """As check() for the qlgpu_dns_* entry points (include/qlgpu_dns.h)."""
    if rc != QLGPU_OK:
        L = load()
        buf = ctypes.create_string_buffer(512)
        L.qlgpu_dns_last_error(h, buf, 512)
        raise QLGPUError(rc, buf.value.decode(errors="replace"))


def check_io(rc: int):
    """As check() for the file entry points of include/qlgpu_io.h."""
    if rc != QLGPU_OK:
        L = load()
        buf = ctypes.create_string_buffer(512)
        L.qlgpu_io_last_error(buf, 512)
        raise QLGPUError(rc, buf.value.decode(errors="replace"))
