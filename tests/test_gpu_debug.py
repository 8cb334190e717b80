"""The QLGPU_DEBUG build (libqlgpu_debug.so) on the GPU: every kernel family
(single-case stage kernels of both models and integrators, both batch engines
with per-case noise, the DNS step, the adjoint of both integrators) runs its
tiny-grid parity cases with the device index checks and the canary guard zones
on, and matches the oracle as the release build does; a guard zone overwritten
from the host is reported by the next call.  Each case runs in a child process
with QLGPU_DEBUG=1 (tests/debug_cases.py)."""
import os
import subprocess
import sys

import pytest

from gpu_util import require_gpu

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", ["debug_library", "single", "batch", "dns", "adjoint", "canary"])
def test_debug_build_case(name):
    require_gpu()
    env = dict(os.environ, QLGPU_DEBUG="1")
    r = subprocess.run([sys.executable, os.path.join(HERE, "debug_cases.py"), name], env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0 and f"ok {name}" in r.stdout, (r.stdout[-2000:], r.stderr[-4000:])
