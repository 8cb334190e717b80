"""Generate the DNS golden fixtures in tests/golden/ (run from the repo root:
``python tests/golden/make_dns_golden.py``).

Each case is a seeded DNS initial state (ql_dns_b200.initial.dns_initial_state)
advanced by the numpy DNS oracle (oracle/dns_oracle.py).  Before saving, the
oracle's QL projection is checked against the MHD_FullQlin oracle on the same
parameters (the pin of test_dns_oracle.py).  There is no reference DNS: the
fixtures freeze this repository's restatement and its initial-condition law.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle.dns_oracle import DNSOracle, from_ql, to_ql  # noqa: E402
from ql_dns_b200.initial import dns_initial_state, initial_state  # noqa: E402
from ql_dns_b200.ktables import ktables  # noqa: E402
from ql_dns_b200.params import DNSParams  # noqa: E402

CASES = {
    # name: (params kwargs, seed, sigma, B0, nsteps)
    "dns_exp": (dict(Mx=16, My=32, NZ=16, dt=0.01, B0z=0.02), 21, 0.3, 0.1, 15),
    "dns_cn_hyper": (dict(Mx=16, My=16, NZ=32, dt=0.01, integrator=1, viscosity_order=4, nu=1e-5, eta=2e-5,
                          omega=0.9), 22, 0.3, 0.1, 15),
}


def ql_pin(p):
    q = p.ql()
    lin, mf, kx0 = initial_state(q, 5, sigma=0.3, B0=0.1, mean_u=0.05)
    lin[ktables(q)["ky_index"] == 0] = 0.0
    _, lo, mo, ko, _ = O.run(q, 0.0, lin, mf, kx0, 5)
    t, l6, kx, _ = DNSOracle(p).run(0.0, from_ql(p, 0.0, lin, mf, kx0), kx0, 5, ql=True)
    l4, m4 = to_ql(p, t, l6, kx)
    assert np.linalg.norm(l4 - lo) <= 1e-13 * np.linalg.norm(lo)


def make(name):
    kw, seed, sigma, B0, n = CASES[name]
    p = DNSParams(**kw)
    ql_pin(p)
    lin, kx0 = dns_initial_state(p, seed, sigma=sigma, B0=B0)
    t, lo, ko, d = DNSOracle(p).run(0.0, lin, kx0, n, diag_every=1)
    fields = dict(integrator=p.integrator, Mx=p.Mx, My=p.My, NZ=p.NZ, L=np.array(p.L), q=p.q, omega=p.omega,
                  nu=p.nu, eta=p.eta, B0z=p.B0z, viscosity_order=p.viscosity_order, dt=p.dt, remap=p.remap,
                  dealias_xy=p.dealias_xy, seed=seed, sigma=sigma, B0=B0, nsteps=n, lin0=lin, kx00=kx0, t=t,
                  lin=lo, kx0=ko, diag=d)
    path = os.path.join(ROOT, "tests", "golden", name + ".npz")
    np.savez_compressed(path, **fields)
    print(name, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    for c in CASES:
        make(c)
