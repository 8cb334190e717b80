"""Adjoint run of the QL MRI at 32x32 modes x NZ=64 (Re=Rm=4000, dt=0.01).

    python -m ql_dns_b200.adjoint_run [--seeds 16] [--steps 2000] [--checkpoint 100] [--fd-dirs 8]

For every seed: J = the fluctuation Maxwell stress averaged over the steps and
dJ/d lin0 from qlgpu_adjoint_maxwell (checkpoints every --checkpoint steps,
stages recomputed per window), checked along --fd-dirs random unit directions
(unit in the norm of lin0, so eps is a relative perturbation of the initial
state) against central finite differences of the GPU forward run with step eps
and eps/2.  Per direction it reports the relative error |adj - fd| / |fd| and
the error relative to |grad| |d|, which stays meaningful for directions nearly
orthogonal to the gradient.  The
adjoint's wall time is compared with the forward run's (both include the
host-device copies of one call).  Seeds run one after another on one GPU.
Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .initial import initial_state
from .params import adjoint_32x32_nz64
from .solver import QLSolver


def forward_J(s: QLSolver, lin, mf, kx0, n):
    s.set_state(0.0, lin, mf, kx0)
    d = s.step(n, diag_every=1)
    return float(d[:, 8].mean())


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--checkpoint", type=int, default=100)
    ap.add_argument("--fd-dirs", type=int, default=8)
    ap.add_argument("--eps", type=float, default=1e-6)
    a = ap.parse_args(argv)
    p = adjoint_32x32_nz64()
    out = {"workload": f"MHD_BQlin + RK3CN_Elin, {p.nx}x{p.ny} modes x NZ={p.NZ}, Re=Rm={1 / p.nu:.0f}, "
                       f"dt={p.dt}, {a.steps} steps, checkpoint every {a.checkpoint}",
           "eps": a.eps, "seeds": []}
    with QLSolver(p) as s:
        for seed in range(a.seeds):
            lin, mf, kx0 = initial_state(p, seed, sigma=1e-3)
            forward_J(s, lin, mf, kx0, 3)  # warm-up
            t0 = time.perf_counter()
            J = forward_J(s, lin, mf, kx0, a.steps)
            t_fwd = time.perf_counter() - t0
            t0 = time.perf_counter()
            Ja, g, _ = s.adjoint_maxwell(0.0, lin, mf, kx0, a.steps, a.checkpoint)
            t_adj = time.perf_counter() - t0
            rng = np.random.default_rng(1000 + seed)
            gnorm = float(np.linalg.norm(g))
            dirs = []
            for _ in range(a.fd_dirs):
                d = rng.normal(size=lin.shape) + 1j * rng.normal(size=lin.shape)
                d *= np.linalg.norm(lin) / np.linalg.norm(d)
                adj = float(np.real(np.vdot(g, d)))
                fd = []
                for eps in (a.eps, a.eps / 2):
                    fd.append((forward_J(s, lin + eps * d, mf, kx0, a.steps) -
                               forward_J(s, lin - eps * d, mf, kx0, a.steps)) / (2 * eps))
                scale = gnorm * float(np.linalg.norm(d))
                dirs.append({"adjoint": adj, "fd_eps": fd[0], "fd_eps_half": fd[1],
                             "cos": adj / scale,  # directional derivative / (|grad| |d|)
                             "rel_err": abs(adj - fd[0]) / abs(fd[0]),
                             "norm_err": abs(adj - fd[0]) / scale})  # error / (|grad| |d|)
            out["seeds"].append({"seed": seed, "J": Ja, "J_forward": J, "grad_norm": gnorm, "dirs": dirs,
                                 "forward_s": t_fwd, "adjoint_s": t_adj, "adjoint_over_forward": t_adj / t_fwd})
    sd = out["seeds"]
    out["adjoint_over_forward_median"] = float(np.median([x["adjoint_over_forward"] for x in sd]))
    out["adjoint_over_forward_max"] = float(np.max([x["adjoint_over_forward"] for x in sd]))
    alld = [d for x in sd for d in x["dirs"]]
    if alld:
        out["fd_rel_err_max"] = max(d["rel_err"] for d in alld)
        out["fd_rel_err_median"] = float(np.median([d["rel_err"] for d in alld]))
        out["fd_norm_err_max"] = max(d["norm_err"] for d in alld)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
