"""Generate the golden fixtures in tests/golden/ (run from the repo root:
``python tests/golden/make_golden.py``).

Each case is a seeded initial state advanced by the CPU oracle
(oracle/ql_oracle.cpp, strict build) and, for the first step, cross-checked
against the independent numpy restatement (tests/numpy_ref.py).  The reference
itself cannot be built here, so these fixtures pin this repository's oracle,
not the reference's binary.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from numpy_ref import NumpyQL  # noqa: E402
from oracle import oracle as O  # noqa: E402
from ql_dns_b200.initial import initial_state  # noqa: E402
from ql_dns_b200.params import mri_16x16_nz32  # noqa: E402

CASES = {
    # name: (params kwargs, seed, sigma, mean_u, nsteps)
    "bqlin_exp": (dict(nx=8, ny=8, NZ=16), 11, 0.3, 0.0, 20),
    "bqlin_cn": (dict(nx=8, ny=8, NZ=16, integrator=1), 12, 0.3, 0.0, 20),
    "fullqlin_exp": (dict(nx=8, ny=8, NZ=16, model=1, B0z=0.02, omega=1.0, viscosity_order=2), 13, 0.3, 0.03, 20),
    "fullqlin_cn_hyper": (dict(nx=8, ny=8, NZ=16, model=1, integrator=1, B0z=0.01, omega=0.9,
                               viscosity_order=4, nu=1e-5, eta=2e-5), 14, 0.3, 0.03, 20),
    "bqlin_remap": (dict(nx=8, ny=8, NZ=32, dt=0.05), 15, 0.1, 0.0, 30),
    "mri16_sigma0p1": (dict(), 0, 0.1, 0.0, 60),
}


def make(name):
    kw, seed, sigma, mean_u, n = CASES[name]
    p = mri_16x16_nz32(**kw)
    lin, mf, kx0 = initial_state(p, seed, sigma=sigma, mean_u=mean_u)
    R = NumpyQL(p)
    l1, m1, _ = R.step(0.0, lin, mf, kx0)
    _, l2, m2, _, _ = O.run(p, 0.0, lin, mf, kx0, 1)
    assert np.linalg.norm(l2 - l1) <= 1e-13 * np.linalg.norm(l1)
    t, lo, mo, ko, d = O.run(p, 0.0, lin, mf, kx0, n, diag_every=1)
    fields = dict(model=p.model, integrator=p.integrator, nx=p.nx, ny=p.ny, NZ=p.NZ, L=np.array(p.L),
                  q=p.q, omega=p.omega, nu=p.nu, eta=p.eta, B0z=p.B0z, viscosity_order=p.viscosity_order,
                  dt=p.dt, remap=p.remap, quasilinear=p.quasilinear, seed=seed, sigma=sigma, mean_u=mean_u,
                  nsteps=n, lin0=lin, mf0=mf, kx00=kx0, t=t, lin=lo, mf=mo, kx0=ko, diag=d)
    path = os.path.join(ROOT, "tests", "golden", name + ".npz")
    np.savez_compressed(path, **fields)
    print(name, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    for c in CASES:
        make(c)
