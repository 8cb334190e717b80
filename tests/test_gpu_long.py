"""Parity at the workloads' own horizons (the MRI is linearly unstable, so the
relative error of a long run is what the 1e-10 bar is about):

* the production single case, 64x64 modes x NZ=128, Re=Rm=8000, dt=0.005,
  seed 1, for all 2000 steps (QL_DNS/main.cpp:108-154 loop);
* every case of the 48-case batched ensemble for 100 steps (both engines'
  default: the chunk-queue engine);
* the 64x128x64 DNS for 100 steps against its numpy oracle.

The QL oracle is the strict FP64 build with OpenMP over modes (the order of the
stress sums over modes differs from the serial build by round-off only)."""
import os

import numpy as np
import pytest

from gpu_util import rel, require_gpu
from oracle import oracle as O
from ql_dns_b200.initial import initial_state
from ql_dns_b200.params import mri_64x64_nz128
from ql_dns_b200.solver import QLSolver

pytestmark = pytest.mark.gpu
TOL = 1e-10
THREADS = os.cpu_count() or 1


def series_rel(dg, do):
    errs = []
    for c in range(1, 13):
        scale = np.abs(do[:, c]).max()
        if scale > 0:
            errs.append(np.abs(dg[:, c] - do[:, c]).max() / scale)
    return max(errs)


def test_production_single_case_2000_steps():
    require_gpu()
    p = mri_64x64_nz128()
    lin, mf, kx0 = initial_state(p, 1, sigma=1e-3)
    n = 2000
    with QLSolver(p) as s:
        s.set_state(0.0, lin, mf, kx0)
        d0 = s.diagnostics()
        d = s.step(n, diag_every=10)
        t, lo, mo, ko = s.get_state()
    t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, n, diag_every=10, kind="strict_omp", nthreads=THREADS)
    assert abs(t - t2) < 1e-12 and np.array_equal(ko, ko2)
    assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (rel(lo, lo2), rel(mo, mo2))
    assert series_rel(np.vstack([d0[None], d]), d2) < TOL


def test_ensemble_every_case_100_steps():
    require_gpu()
    from ql_dns_b200.batch import QLBatch, mri_ensemble
    cases, b0s, seeds = mri_ensemble()
    sts = [initial_state(p, s, sigma=1e-3, B0=b0) for p, b0, s in zip(cases, b0s, seeds)]
    n = 100
    with QLBatch(cases) as b:
        assert b.engine() == "queue"
        b.set_states(0.0, sts)
        recs = b.step(n, diag_every=5)
        outs = b.get_states()
    for c, (p, (lin, mf, kx0)) in enumerate(zip(cases, sts)):
        t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, n, diag_every=5, kind="strict_omp", nthreads=THREADS)
        t, lo, mo, ko = outs[c]
        assert abs(t - t2) < 1e-12 and np.array_equal(ko, ko2), c
        assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (c, rel(lo, lo2), rel(mo, mo2))
        assert series_rel(recs[c], d2[1:]) < TOL, c


def test_dns_production_grid_100_steps():
    require_gpu()
    from oracle.dns_oracle import DNSOracle
    from ql_dns_b200.dns import QLDns
    from ql_dns_b200.initial import dns_initial_state
    from ql_dns_b200.params import dns_64x128x64
    p = dns_64x128x64()
    lin, kx0 = dns_initial_state(p, 2, sigma=1e-2, B0=0.05)
    n = 100
    D = DNSOracle(p)
    t2, lo, ko, d2 = D.run(0.0, lin, kx0, n, diag_every=10)
    with QLDns(p) as g:
        g.set_state(0.0, lin, kx0)
        d = g.step(n, diag_every=10)
        t, lg, kg = g.get_state()
    assert np.array_equal(kg, ko)
    assert rel(lg, lo) < TOL, rel(lg, lo)
    # every column of the DNS record (15 values, MHD_FullQlin.cpp:487-717 order)
    assert max(np.abs(d[:, c] - d2[:, c]).max() / max(np.abs(d2[:, c]).max(), 1e-300) for c in range(1, 15)) < TOL
