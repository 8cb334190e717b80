"""Cases run in a child process with QLGPU_DEBUG=1, so that the Python binding
loads libqlgpu_debug.so (device index checks and canary guard zones checked
after every call that launches kernels).  `python debug_cases.py NAME` prints
"ok NAME" when the case passed.  Used by test_gpu_debug.py; the bars are the
release tests' bars (relative L2 <= 1e-10 against the oracle)."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

from gpu_util import rel  # noqa: E402
from oracle import oracle as O  # noqa: E402
from ql_dns_b200 import _capi  # noqa: E402
from ql_dns_b200.initial import initial_state  # noqa: E402
from ql_dns_b200.params import QLParams  # noqa: E402

TOL = 1e-10


def case_debug_library():
    L = _capi.load()
    assert os.path.basename(L._name) == "libqlgpu_debug.so", L._name
    assert L.qlgpu_debug_build() == 1


def case_single():
    from ql_dns_b200.solver import QLSolver
    for model in (0, 1):
        for integ in (0, 1):
            for NZ in (16, 32, 64, 128):
                p = QLParams(model=model, integrator=integ, nx=8, ny=6, NZ=NZ, dt=0.01, B0z=0.01 if model else 0.0,
                             omega=0.9)
                st = initial_state(p, 3, sigma=0.2, B0=0.05, mean_u=0.01 if model else 0.0)
                with QLSolver(p) as s:
                    s.set_state(0.0, *st)
                    d = s.step(6, diag_every=2)
                    t, lo, mo, ko = s.get_state()
                t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, *st, 6, diag_every=2)
                assert t == t2 and rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (model, integ, NZ)


def case_batch():
    from ql_dns_b200.batch import QLBatch
    cases = [QLParams(nx=8, ny=6, NZ=16, dt=0.01), QLParams(nx=10, ny=8, NZ=32, dt=0.01),
             QLParams(nx=6, ny=8, NZ=64, dt=0.01), QLParams(nx=8, ny=8, NZ=128, dt=0.01)]
    sts = [initial_state(p, 20 + i, sigma=0.2, B0=0.04) for i, p in enumerate(cases)]
    for engine in ("queue", "items"):
        with QLBatch(cases) as b:
            b.set_engine(engine)
            for c, st in enumerate(sts):
                b.set_state(c, 0.0, *st)
            b.set_noise(1, 0.05, 0.5, 40.0, 9)
            b.step(5, diag_every=1)
            for c, (p, st) in enumerate(zip(cases, sts)):
                t, lo, mo, ko = b.get_state(c)
                if c == 1:
                    t2, lo2, mo2, _, _, _ = O.run_forced(p, 0.0, *st, 5, f_noise=0.05, k_lo=0.5, k_hi=40.0, seed=9)
                else:
                    t2, lo2, mo2, _, _ = O.run(p, 0.0, *st, 5)
                assert t == t2 and rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (engine, c)


def case_dns():
    from oracle.dns_oracle import DNSOracle
    from ql_dns_b200.dns import QLDns
    from ql_dns_b200.initial import dns_initial_state
    from ql_dns_b200.params import DNSParams
    pd = DNSParams(Mx=16, My=32, NZ=16, dt=0.01)
    ld, kd = dns_initial_state(pd, 0, sigma=0.2, B0=0.1)
    with QLDns(pd) as g:
        g.set_state(0.0, ld, kd)
        g.step(1)
        _, lg, _ = g.get_state()
    _, lgo, _, _ = DNSOracle(pd).step(0.0, ld, kd)
    assert rel(lg, lgo) < TOL


def case_adjoint():
    from ql_dns_b200.params import mri_16x16_nz32
    from ql_dns_b200.solver import QLSolver
    for integ in (0, 1):
        p = mri_16x16_nz32(nx=8, ny=8, NZ=32, integrator=integ)
        lin, mf, kx0 = initial_state(p, 7, sigma=0.2)
        n = 8
        with QLSolver(p) as s:
            J, g, _ = s.adjoint_maxwell(0.0, lin, mf, kx0, n, checkpoint_every=3)
        rng = np.random.default_rng(5)
        d = rng.normal(size=lin.shape) + 1j * rng.normal(size=lin.shape)
        Jo, dJ = O.tlm_maxwell(p, 0.0, lin, mf, kx0, d, None, n)
        assert abs(J - Jo) <= 1e-10 * abs(Jo)
        adj = float(np.real(np.vdot(g, d)))
        assert abs(adj - dJ) <= 1e-8 * abs(dJ), (integ, adj, dJ)


def case_canary():
    # a byte written into a guard zone from the host is reported by the next call
    from ql_dns_b200._capi import QLGPUError
    from ql_dns_b200.batch import QLBatch
    from ql_dns_b200.solver import QLSolver
    L = _capi.load()
    p = QLParams(nx=8, ny=6, NZ=32, dt=0.01)
    st = initial_state(p, 1, sigma=0.2)
    with QLSolver(p) as s:
        s.set_state(0.0, *st)
        s.step(1)
        assert L.qlgpu_debug_guard_poke(s.h, 0) == 0
        try:
            s.step(1)
            raise AssertionError("the overwritten guard zone was not reported")
        except QLGPUError as e:
            assert e.code == 4 and "guard zone" in str(e), e
    with QLBatch([p, QLParams(nx=6, ny=8, NZ=64, dt=0.01)]) as b:
        b.set_state(0, 0.0, *st)
        b.step(1)
        assert L.qlgpu_batch_debug_guard_poke(b.b, 3) == 0
        try:
            b.step(1)
            raise AssertionError("the overwritten guard zone was not reported")
        except QLGPUError as e:
            assert e.code == 4 and "guard zone" in str(e), e


if __name__ == "__main__":
    name = sys.argv[1]
    globals()["case_" + name]()
    print("ok", name)
