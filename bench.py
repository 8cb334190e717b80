"""Benchmark of the quasi-linear shearing-box RK3 step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one full RK3 step, three fused stage kernels, of every
(kx,ky) mode): QL MRI plain FP64 at production size, MHD_BQlin with
RK3CN_Elin, 64x64 (kx,ky) modes (2016 mode columns) x NZ=128 (85 dealiased kz),
Lx=1, Ly=pi, Lz=1, q=1.5, Re=Rm=8000, dt=0.005, seeded initial condition
(seed 1, sigma=1e-3 |k|^-2, By = 0.05 sin(2 pi z)).  The data are synthetic
(the reference ships no data sets).

Metric: mode-steps/s = (mode columns advanced by one full step) / second,
whole job over all ranks.  N > 1 runs independent replicas of the workload,
one per GPU (the step has no cross-GPU exchange at this size), so scaling is
weak.  The timed region is bracketed by a barrier and device synchronisation;
the time per rank is the sum of CUDA-event durations on the solver's stream,
and the job time is the max over ranks.  L2 is flushed (a 512 MiB write)
before every timed step because the 2016-mode working set (~45 MB) would
otherwise stay resident in the 126 MB L2.

--impl reference times the CPU restatement of the reference's step (the
oracle, OpenMP over modes, -O3 -ffast-math -march=native like the reference's
SConstruct) on the host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mode-steps/s on 1 B200, batched vs plain per-case, rel err ≤1e-10 vs FP64 CPU"
UNIT = "mode-steps/s"
WORKLOAD = ("QL MRI plain FP64 MHD_BQlin + RK3CN_Elin, 64x64 (kx,ky) modes (2016 columns) x NZ=128 "
            "(nz=85), Re=Rm=8000, dt=0.005, seed 1")
FALLBACK_HBM_GBS = 6650.0


def workload_params():
    from ql_dns_b200.params import config1
    return config1()


def algorithmic_bytes_per_step(p) -> float:
    # 2N-storage minimum per mode-step: 10 * nLin * nz * 16 B (stage 1: read u,
    # write u, F1; stage 2: read u, F1, write u, F2; stage 3: read u, F2, write u)
    return 10.0 * 4 * p.nz * 16 * p.nxy


def stage_bytes(p):
    unit = 4 * p.nz * 16 * p.nxy
    return [3 * unit, 4 * unit, 3 * unit]


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def read_traffic():
    """DRAM bytes per stage-kernel launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_cfg1.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(backend: str = "nccl"):
    """One process per GPU (torchrun env); N > 1 runs independent replicas."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, x: float) -> float:
    """Job time = the slowest rank's device time (outside the timed region)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_plan(ws: int, rank: int, p):
    """Weak scaling: every rank advances its own replica of the workload (no
    data-path collective); returns (seed, mode columns of this rank, job total)."""
    return 1 + rank, p.nxy, p.nxy * ws


# ---------------------------------------------------------------------------
# CPU reference arm: the oracle restatement of the reference step
# ---------------------------------------------------------------------------
def cpu_oracle_time(p, steps: int, threads: int):
    """Time `steps` RK3 steps of the workload on the host with the fast oracle."""
    from oracle import oracle as O
    from ql_dns_b200.initial import initial_state
    kind = "native"
    try:
        O.build(native=True)
    except Exception:
        kind = "fast"
    lin, mf, kx0 = initial_state(p, 1, sigma=1e-3)
    O.run(p, 0.0, lin, mf, kx0, 1, kind=kind, nthreads=threads)  # warm-up (page-in, OpenMP pool)
    t0 = time.perf_counter()
    O.run(p, 0.0, lin, mf, kx0, steps, kind=kind, nthreads=threads)
    dt = time.perf_counter() - t0
    return p.nxy * steps / dt, dt, kind


def cpu_baseline(p, budget_s: float = 15.0, threads: int | None = None):
    threads = threads or os.cpu_count() or 1
    # size the sample: one timed step first, then as many as fit the budget
    rate1, dt1, kind = cpu_oracle_time(p, 1, threads)
    steps = max(1, min(200, int(budget_s / max(dt1, 1e-6))))
    rate, dt, kind = cpu_oracle_time(p, steps, threads)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} RK3 steps of the full 2016-mode x NZ=128 workload ({dt:.1f} s), "
                      f"oracle build '{kind}', OpenMP over modes"}


def run_reference(args):
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return 0
    p = workload_params()
    threads = os.cpu_count() or 1
    vals = []
    # each "step" of this arm is a bounded sample (a few RK3 steps on all cores),
    # sized so the whole run stays near 60 s of CPU work
    rate1, dt1, kind = cpu_oracle_time(p, 1, threads)
    per = max(1, min(50, int(60.0 / (max(args.steps, 1) * max(dt1, 1e-6)))))
    for _ in range(args.warmup):
        cpu_oracle_time(p, 1, threads)
    total_t = 0.0
    for _ in range(args.steps):
        r, dt, kind = cpu_oracle_time(p, per, threads)
        vals.append(r)
        total_t += dt
    value = p.nxy * per * args.steps / total_t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_t / (args.steps * per),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": "host cores (OpenMP over modes)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{per} RK3 steps per timed step, oracle build '{kind}'"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from ql_dns_b200.initial import initial_state
    from ql_dns_b200.solver import QLSolver
    p = workload_params()
    seed, my_modes, job_modes = replica_plan(ws, rank, p)
    lin, mf, kx0 = initial_state(p, seed, sigma=1e-3)
    solver = QLSolver(p, device=local)
    solver.set_state(0.0, lin, mf, kx0)
    ext = torch.cuda.ExternalStream(solver.stream())
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def flush_l2():
        with torch.cuda.stream(ext):
            flush.fill_(1.0)

    for _ in range(args.warmup):
        solver.step_timed()
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    stage_ms = np.zeros(3)
    step_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush_l2()
            with torch.cuda.stream(ext):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(ext)
            st = solver.step_timed()  # synchronises on its last event
            e1.record(ext)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            stage_ms += st
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    my_total_ms = float(sum(step_ms))
    job_ms = max_over_ranks(ws, my_total_ms)
    value = job_modes * args.steps / (job_ms / 1e3)
    launches = 3 * args.steps

    # roofline of the stage kernel: algorithmic bytes / event-timed duration
    peak, peak_kind = hbm_peak()
    sb = stage_bytes(p)
    achieved = sum(sb) * args.steps / (stage_ms.sum() / 1e3) / 1e9
    traffic = read_traffic()

    # end to end through the C ABI with pinned host buffers: set_state (H2D),
    # K steps with a diagnostic record per step (D2H of the step's metrics),
    # get_state (D2H)
    lin_h = torch.empty(lin.shape, dtype=torch.complex128, pin_memory=True).numpy()
    mf_h = torch.empty(mf.shape, dtype=torch.complex128, pin_memory=True).numpy()
    lin_h[...] = lin
    mf_h[...] = mf
    torch.cuda.synchronize()
    barrier(ws)
    flush_l2()
    torch.cuda.synchronize()
    ee0 = torch.cuda.Event(enable_timing=True)
    ee1 = torch.cuda.Event(enable_timing=True)
    ee0.record(ext)
    solver.set_state(0.0, lin_h, mf_h, kx0)
    solver.step(args.steps, diag_every=1)
    t_out, lo, mo, ko = solver.get_state()
    ee1.record(ext)
    ee1.synchronize()
    e2e_ms = max_over_ranks(ws, ee0.elapsed_time(ee1))
    state_bytes = lin.nbytes + mf.nbytes + kx0.nbytes
    e2e = {"value": job_modes * args.steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": 15 * 8 + state_bytes / args.steps}
    assert np.isfinite(lo).all() and np.isfinite(mo).all()

    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": job_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "flushed (512 MiB write) before every timed step",
                       "mode_columns": p.nxy, "NZ": p.NZ, "nz": p.nz},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "stage_kernel<128,MHD_BQlin,RK3CN_Elin>",
                         "algorithmic_bytes_per_launch": sum(sb) / 3,
                         "avg_launch_ms": float(stage_ms.sum() / launches)},
            "e2e": e2e,
            "gpu_launches": launches,
        }
        out["clocks"] = clk.summary()
    solver.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if not args.no_cpu_baseline and ws == 1:
            out["cpu_baseline"] = cpu_baseline(p, budget_s=args.cpu_budget)
        print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
