"""Command-line driver of the batched QL MRI ensemble.

    python -m ql_dns_b200.ensemble [--cases 48] [--steps 100] [--tune] [--diag-every 0] [--nz 32 64]
                                   [--engine auto|queue|items] [--chunks P16 P32 P64 P128]

Builds the ensemble of ``batch.mri_ensemble`` (mode grids {16, 32, 48, 64}^2,
NZ {32, 64, 128}, Rm log-uniform in [500, 16000], Pm {1, 2, 4}, B0 in
[0.01, 0.1]; initial-condition seed c for case c), optionally runs the
autotuner, advances every case by --steps steps in one persistent launch and
prints the device time, the mapping and each case's last energy / stress
record.  Used as the command of the batch-kernel profiles.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from .batch import QLBatch, mri_ensemble
from .initial import initial_state


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=48)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--tune", action="store_true")
    ap.add_argument("--diag-every", type=int, default=0)
    ap.add_argument("--nz", type=int, nargs="*", default=None, help="keep only the cases with these NZ")
    ap.add_argument("--engine", choices=["auto", "queue", "items"], default="auto")
    ap.add_argument("--chunks", type=int, nargs=4, default=None, help="queue engine: passes per chunk, NZ 16..128")
    a = ap.parse_args(argv)
    cases, b0s, seeds = mri_ensemble(a.cases)
    if a.nz:
        keep = [i for i, p in enumerate(cases) if p.NZ in a.nz]
        cases, b0s, seeds = [cases[i] for i in keep], [b0s[i] for i in keep], [seeds[i] for i in keep]
    with QLBatch(cases) as b:
        b.set_engine(a.engine)
        if a.chunks:
            b.set_chunks(a.chunks)
        for c, (p, b0, s) in enumerate(zip(cases, b0s, seeds)):
            lin, mf, kx0 = initial_state(p, s, sigma=1e-3, B0=b0)
            b.set_state(c, 0.0, lin, mf, kx0)
        if a.tune:
            b.tune(3)
        # one untimed launch first (kernel set-up), then the initial state again
        b.step_timed(1)
        for c, (p, b0, s) in enumerate(zip(cases, b0s, seeds)):
            lin, mf, kx0 = initial_state(p, s, sigma=1e-3, B0=b0)
            b.set_state(c, 0.0, lin, mf, kx0)
        if a.diag_every > 0:
            recs = b.step(a.steps, diag_every=a.diag_every)
            last = [r[-1].tolist() if len(r) else None for r in recs]
            ms = None
        else:
            ms = b.step_timed(a.steps)
            last = None
        out = {"cases": len(cases), "steps": a.steps, "modes": int(sum(p.nxy for p in cases)),
               "engine": b.engine(), "device_ms": ms, "mapping": b.mapping()}
        if ms:
            out["mode_steps_per_s"] = out["modes"] * a.steps / (ms / 1e3)
            if os.environ.get("QLGPU_TRACE") == "1" and b.engine() == "queue":
                out["queue_trace"] = b.queue_trace()
        if last:
            out["last_records"] = last
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
