"""Adjoint run of the QL MRI at 32x32 modes x NZ=64 (Re=Rm=4000, dt=0.01).

    python -m ql_dns_b200.adjoint_run [--seeds 16] [--steps 2000] [--checkpoint 100] [--fd-dirs 8] [--reps 2]
                                      [--integrator 0|1]

All seeds run together: J = the fluctuation Maxwell stress averaged over the
steps and dJ/d lin0 come from one qlgpu_adjoint_maxwell_batch call (one handle
and stream per seed, checkpoints every --checkpoint steps, stages recomputed
per window).  The forward cost it is compared with is the same seeds' forward
run with a record every step through the batched ensemble (one persistent
launch for all seeds, QLBatch), with the batch's default engine (the chunk
queue, which the adjoint's forward sweep also uses) and with the work-item
engine (which its window recompute uses: that engine records the stage inputs).
--integrator 1 runs RK3CN (Crank-Nicolson) instead of RK3CN_Elin.  Gradients are checked along --fd-dirs random
directions per seed (scaled to |lin0|, so eps is a relative perturbation)
against central finite differences of the batched forward run with step eps
and eps/2.  Per direction: the relative error |adj - fd| / |fd| and the error
relative to |grad| |d|, which stays meaningful for directions nearly
orthogonal to the gradient.  The batched forward and adjoint calls are timed
by the wall clock --reps times each (the adjoint call includes its device
allocations); the minimum is reported.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .batch import QLBatch
from .initial import initial_state
from .params import adjoint_32x32_nz64
from .solver import QLSolver


def batch_J(b: QLBatch, states, n):
    for c, (lin, mf, kx0) in enumerate(states):
        b.set_state(c, 0.0, lin, mf, kx0)
    recs = b.step(n, diag_every=1)
    return np.array([float(r[:, 8].mean()) for r in recs])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--checkpoint", type=int, default=100)
    ap.add_argument("--fd-dirs", type=int, default=8)
    ap.add_argument("--eps", type=float, default=1e-6)
    ap.add_argument("--reps", type=int, default=2, help="timed repetitions; the minimum is reported")
    ap.add_argument("--integrator", type=int, default=0, choices=[0, 1])
    a = ap.parse_args(argv)
    p = adjoint_32x32_nz64(integrator=a.integrator)
    S = a.seeds
    states = [initial_state(p, seed, sigma=1e-3) for seed in range(S)]
    integ = "RK3CN_Elin" if a.integrator == 0 else "RK3CN"
    out = {"workload": f"MHD_BQlin + {integ}, {p.nx}x{p.ny} modes x NZ={p.NZ}, Re=Rm={1 / p.nu:.0f}, "
                       f"dt={p.dt}, {a.steps} steps, checkpoint every {a.checkpoint}, {S} seeds together",
           "eps": a.eps}
    with QLBatch([p] * S) as b:
        batch_J(b, states, 3)  # warm-up
        t_fwds, t_adjs = [], []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            Jf = batch_J(b, states, a.steps)
            t_fwds.append(time.perf_counter() - t0)
        t_fwd = min(t_fwds)
        engine = b.engine()
        b.set_engine("items")
        batch_J(b, states, 3)
        t_items = []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            batch_J(b, states, a.steps)
            t_items.append(time.perf_counter() - t0)
        t_fwd_items = min(t_items)
        b.set_engine("auto")
        solvers = [QLSolver(p) for _ in range(S)]
        try:
            QLSolver.adjoint_maxwell_batch(solvers, 0.0, [s[0] for s in states], [s[1] for s in states],
                                           [s[2] for s in states], 3, 3)  # warm-up
            for _ in range(a.reps):
                t0 = time.perf_counter()
                Ja, G, _ = QLSolver.adjoint_maxwell_batch(solvers, 0.0, [s[0] for s in states],
                                                          [s[1] for s in states], [s[2] for s in states], a.steps,
                                                          a.checkpoint)
                t_adjs.append(time.perf_counter() - t0)
            t_adj = min(t_adjs)
            t0 = time.perf_counter()
            solvers[0].adjoint_maxwell(0.0, *states[0], a.steps, a.checkpoint)
            t_adj1 = time.perf_counter() - t0
            t0 = time.perf_counter()
            solvers[0].set_state(0.0, *states[0])
            solvers[0].step(a.steps, diag_every=1)
            t_fwd1 = time.perf_counter() - t0
        finally:
            for s in solvers:
                s.close()
        rng = np.random.default_rng(1000)
        dirs = []
        for _ in range(a.fd_dirs):
            ds = []
            for lin, _, _ in states:
                d = rng.normal(size=lin.shape) + 1j * rng.normal(size=lin.shape)
                ds.append(d * (np.linalg.norm(lin) / np.linalg.norm(d)))
            fd = []
            for eps in (a.eps, a.eps / 2):
                Jp = batch_J(b, [(lin + eps * d, mf, kx0) for (lin, mf, kx0), d in zip(states, ds)], a.steps)
                Jm = batch_J(b, [(lin - eps * d, mf, kx0) for (lin, mf, kx0), d in zip(states, ds)], a.steps)
                fd.append((Jp - Jm) / (2 * eps))
            for k in range(S):
                adj = float(np.real(np.vdot(G[k], ds[k])))
                scale = float(np.linalg.norm(G[k]) * np.linalg.norm(ds[k]))
                dirs.append({"seed": k, "adjoint": adj, "fd_eps": float(fd[0][k]), "fd_eps_half": float(fd[1][k]),
                             "cos": adj / scale, "rel_err": abs(adj - fd[0][k]) / abs(fd[0][k]),
                             "norm_err": abs(adj - fd[0][k]) / scale})
    out.update({"J_adjoint": Ja.tolist(), "J_forward": Jf.tolist(),
                "J_rel_diff_max": float(np.max(np.abs(Ja - Jf) / np.abs(Jf))),
                "forward_batch_s": t_fwd, "adjoint_batch_s": t_adj,
                "forward_batch_s_all": t_fwds, "adjoint_batch_s_all": t_adjs,
                "adjoint_over_forward": t_adj / t_fwd, "forward_engine": engine,
                "forward_batch_items_s": t_fwd_items, "adjoint_over_forward_items": t_adj / t_fwd_items,
                "single_seed": {"forward_s": t_fwd1, "adjoint_s": t_adj1, "adjoint_over_forward": t_adj1 / t_fwd1},
                "batch_speedup_vs_sequential_adjoint": S * t_adj1 / t_adj})
    if dirs:
        out["fd_rel_err_median"] = float(np.median([d["rel_err"] for d in dirs]))
        out["fd_rel_err_max"] = max(d["rel_err"] for d in dirs)
        out["fd_norm_err_max"] = max(d["norm_err"] for d in dirs)
        out["directions"] = len(dirs)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
