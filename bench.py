"""Benchmark of the quasi-linear shearing-box RK3 step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload: the batched QL MRI ensemble.  48 independent MHD_BQlin
cases stepped with RK3CN_Elin at dt = 0.01, drawn with numpy seed 12345: per
case a square (kx,ky) mode grid from {16, 32, 48, 64}^2, NZ from {32, 64,
128}, Rm log-uniform in [500, 16000], Pm from {1, 2, 4} (eta = 1/Rm,
nu = Pm/Rm) and a mean-field amplitude B0 uniform in [0.01, 0.1]; case c
starts from the seeded initial condition with seed c (sigma = 1e-3 |k|^-2,
By = B0 sin(2 pi z)).  The data are synthetic (the reference ships no data
sets).  One "step" = one full RK3 step of every mode of every case.  All 48
cases run in ONE persistent cooperative launch per call (K steps), with the
CTA mapping chosen by the autotuner before the warm-up.

Metric: mode-steps/s = (mode columns advanced by one full step) / second,
whole job over all ranks.  The same ensemble run case after case through the
plain single-case path is reported beside it ("plain_per_case"), and so is
the single-case production workload (64x64 modes x NZ=128, Re=Rm=8000,
dt=0.005, seed 1; "single_case").  N > 1 runs independent replicas of the
ensemble, one per GPU (rank r uses initial-condition seeds 48 r + c), so
scaling is weak.  The timed region is bracketed by a barrier and device
synchronisation and timed with CUDA events on the batch's stream; the job
time is the max over ranks.  The ensemble's state (about 0.5 GB with its RK
buffers) is larger than the 126 MB L2, so no flush is needed between steps;
the single-case workload (45 MB) is timed with an L2 flush before every step.

--impl reference times the CPU restatement of the reference's step (the
oracle, OpenMP over modes, -O3 -ffast-math -march=native like the reference's
SConstruct) on the host cores on a bounded sample of the same ensemble.
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
WORKLOAD = ("batched QL MRI ensemble: 48 MHD_BQlin cases (RK3CN_Elin, dt=0.01), mode grids {16,32,48,64}^2, "
            "NZ {32,64,128}, Rm log-uniform [500,16000], Pm {1,2,4}, B0 U[0.01,0.1], draw seed 12345, "
            "IC seeds 0..47, one persistent launch")
SINGLE_WORKLOAD = ("QL MRI plain FP64 MHD_BQlin + RK3CN_Elin, 64x64 (kx,ky) modes (2016 columns) x NZ=128 "
                   "(nz=85), Re=Rm=8000, dt=0.005, seed 1")
NCASES = 48
FALLBACK_HBM_GBS = 6650.0
KERNEL_NAME = {"queue": "ens_kernel<MHD_BQlin,RK3CN_Elin> (chunk-queue engine, one launch of K steps)",
               "items": "batch_kernel<MHD_BQlin,RK3CN_Elin> (work-item engine, one launch of K steps)"}
KERNEL_PROFILE = {"queue": "ens_kernel_mri_ensemble48.md", "items": "batch_kernel_mri_ensemble48.md"}


def single_params():
    from ql_dns_b200.params import mri_64x64_nz128
    return mri_64x64_nz128()


def ensemble(rank: int = 0):
    """Cases, mean-field amplitudes and initial-condition seeds of one replica."""
    from ql_dns_b200.batch import mri_ensemble
    cases, b0s, seeds = mri_ensemble(NCASES)
    return cases, b0s, [NCASES * rank + s for s in seeds]


def ensemble_states(cases, b0s, seeds):
    from ql_dns_b200.initial import initial_state
    return [initial_state(p, s, sigma=1e-3, B0=b0) for p, b0, s in zip(cases, b0s, seeds)]


def algorithmic_bytes_per_step(p) -> float:
    # 2N-storage minimum per mode-step: 10 * nLin * nz * 16 B (stage 1: read u,
    # write u, F1; stage 2: read u, F1, write u, F2; stage 3: read u, F2, write u)
    return 10.0 * 4 * p.nz * 16 * p.nxy


def reference_flops_per_step(p) -> float:
    """FP64 flops of one mode-step in the reference's formulation of MHD_BQlin: 3 rhs per
    step x (15 inverse + 7 forward) length-NZ transforms x 5 NZ log2 NZ, per mode column."""
    import math
    return p.nxy * 3 * (15 + 7) * 5 * p.NZ * math.log2(p.NZ)


def own_transform_flops_per_step(p) -> float:
    """FP64 flops of the transforms this build runs per mode-step: 3 stages x (9 inverse +
    5 forward) length-NZ transforms x 5 NZ log2 NZ (qlgpu_ens.cuh)."""
    import math
    return p.nxy * 3 * 14 * 5 * p.NZ * math.log2(p.NZ)


def fp64_peak(local) -> float:
    import ctypes
    from ql_dns_b200 import _capi
    v = ctypes.c_double()
    _capi.check(_capi.load().qlgpu_fp64_peak(local, ctypes.byref(v)))
    return v.value


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


def read_traffic(name: str):
    """DRAM bytes per launch (per step for the batch kernel) from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:") or line.startswith("traffic_bytes_per_step:"):
                return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region: NVML read
    every ~2 ms in a thread (read-only queries), else nvidia-smi every 200 ms."""

    HW_SLOWDOWN, SW_POWER_CAP, SW_THERMAL, HW_THERMAL = 0x8, 0x4, 0x20, 0x40

    def __init__(self, index: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        self.index = int(ids[index]) if index < len(ids) and ids[index].isdigit() else index
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

            def loop():
                while not self.stop.is_set():
                    try:
                        self.samples.append((float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)),
                                             float(smax), int(get_reasons(h))))
                    except Exception:
                        pass
                    time.sleep(0.002)

            self.nvml = pynvml
            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            # the thread is sampling before the timed region starts; only the samples taken
            # from here on (inside the region) are kept
            t_end = time.time() + 0.5
            while not self.samples and time.time() < t_end:
                time.sleep(0.0005)
            self.samples.clear()
            return self
        except Exception:
            self.nvml = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read_smi(self):
        names = [self.HW_SLOWDOWN, self.HW_THERMAL, self.SW_THERMAL, self.SW_POWER_CAP]
        for ln in self.proc.stdout:
            f = [x.strip() for x in ln.strip().split(",")]
            if len(f) < 9:
                continue
            try:
                bits = sum(b for b, v in zip(names, f[5:9]) if v.lower().startswith("active"))
                self.samples.append((float(f[1]), float(f[2]), bits))
            except ValueError:
                continue

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        elif self.nvml:
            self.thread.join(timeout=1)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        names = {self.HW_SLOWDOWN: "hw_slowdown", self.HW_THERMAL: "hw_thermal_slowdown",
                 self.SW_THERMAL: "sw_thermal_slowdown", self.SW_POWER_CAP: "sw_power_cap"}
        reasons = sorted({n for b, n in names.items() for s in self.samples if s[2] & b})
        return {"sm_mhz": statistics.median(s[0] for s in self.samples), "sm_max_mhz": self.samples[-1][1],
                "reasons": reasons, "samples": len(self.samples),
                "source": "NVML, ~2 ms period" if self.nvml else "nvidia-smi, 200 ms period"}


def dist_setup(backend: str = "nccl", timeout_s: float = 120.0):
    """One process per GPU (torchrun env); N > 1 runs independent replicas.  A rank
    that dies or never arrives ends the others' next collective with an error within
    timeout_s instead of a hang."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
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


def replica_plan(ws: int, rank: int, modes: int):
    """Weak scaling: every rank advances its own replica of the ensemble (no
    data-path collective); returns (first initial-condition seed of this rank,
    mode columns of this rank, job total)."""
    return NCASES * rank, modes, modes * ws


# ---------------------------------------------------------------------------
# CPU reference arm: the oracle restatement of the reference step
# ---------------------------------------------------------------------------
def _oracle_kind():
    from oracle import oracle as O
    try:
        O.build(native=True)
        return "native"
    except Exception:
        return "fast"


def cpu_ensemble_time(cases, sts, steps: int, threads: int, kind: str):
    """`steps` RK3 steps of every case of the ensemble with the oracle; (mode-steps/s, seconds)."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    for p, (lin, mf, kx0) in zip(cases, sts):
        O.run(p, 0.0, lin, mf, kx0, steps, kind=kind, nthreads=threads)
    dt = time.perf_counter() - t0
    return sum(p.nxy for p in cases) * steps / dt, dt


def cpu_baseline(budget_s: float = 15.0, threads: int | None = None):
    threads = threads or os.cpu_count() or 1
    cases, b0s, seeds = ensemble(0)
    sts = ensemble_states(cases, b0s, seeds)
    kind = _oracle_kind()
    cpu_ensemble_time(cases, sts, 1, threads, kind)  # warm-up (page-in, OpenMP pool)
    r1, dt1 = cpu_ensemble_time(cases, sts, 1, threads, kind)
    steps = max(1, min(200, int(budget_s / max(dt1, 1e-6))))
    rate, dt = cpu_ensemble_time(cases, sts, steps, threads, kind)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} RK3 steps of all 48 ensemble cases ({dt:.1f} s), oracle build '{kind}', "
                      f"OpenMP over modes"}


def run_reference(args):
    ws, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    cases, b0s, seeds = ensemble(0)
    sts = ensemble_states(cases, b0s, seeds)
    kind = _oracle_kind()
    # each "step" of this arm is a bounded sample (RK3 steps of all cases on all
    # cores), sized so the whole run stays near 60 s of CPU work
    r1, dt1 = cpu_ensemble_time(cases, sts, 1, threads, kind)
    per = max(1, min(50, int(60.0 / (max(args.steps, 1) * max(dt1, 1e-6)))))
    for _ in range(args.warmup):
        cpu_ensemble_time(cases, sts, 1, threads, kind)
    total_t = 0.0
    for _ in range(args.steps):
        r, dt = cpu_ensemble_time(cases, sts, per, threads, kind)
        total_t += dt
    modes = sum(p.nxy for p in cases)
    value = modes * per * args.steps / total_t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_t / (args.steps * per),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": "host cores (OpenMP over modes)", "mode_columns": modes},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{per} RK3 steps of all 48 cases per timed step, oracle build '{kind}'"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_single(args, ext_stream_of, local):
    """The single-case production workload through the plain path (L2 flushed before each step)."""
    import torch
    from ql_dns_b200.initial import initial_state
    from ql_dns_b200.solver import QLSolver
    p = single_params()
    lin, mf, kx0 = initial_state(p, 1, sigma=1e-3)
    steps = max(1, min(args.steps, 500))
    with QLSolver(p, device=local) as solver:
        solver.set_state(0.0, lin, mf, kx0)
        ext = ext_stream_of(solver.stream())
        flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        for _ in range(args.warmup):
            solver.step_timed()
        stage_ms = np.zeros(3)
        for _ in range(steps):
            with torch.cuda.stream(ext):
                flush.fill_(1.0)
            stage_ms += solver.step_timed()
        del flush
    # the same case as a batch of one on the chunk-queue engine: all K steps in one persistent
    # launch, its ~45 MB working set staying in L2 between steps as in a run
    from ql_dns_b200.batch import QLBatch
    with QLBatch([p], device=local) as b:
        b.set_engine("queue")
        b.set_chunks([2, 2, 2, 2])  # 84 chunks of 24 modes: one wave over the SMs
        b.set_state(0, 0.0, lin, mf, kx0)
        b.step_timed(max(args.warmup, 1))
        b.set_state(0, 0.0, lin, mf, kx0)
        pms = b.step_timed(steps)
    peak, _ = hbm_peak()
    sb = stage_bytes(p)
    achieved = sum(sb) * steps / (stage_ms.sum() / 1e3) / 1e9
    p_ach = sum(sb) * steps / (pms / 1e3) / 1e9
    persistent = {"path": "QLBatch of one case, chunk-queue engine, K steps in one launch", "value":
                  p.nxy * steps / (pms / 1e3), "unit": UNIT, "ms_per_step": pms / steps,
                  "l2": "not flushed: the working set stays in L2 across the steps of the launch",
                  "roofline": {"bound": "hbm", "achieved": p_ach, "peak": peak, "unit": "GB/s", "frac": p_ach / peak,
                               "kernel": "ens_kernel<RK3CN_Elin>"}}
    return {"workload": SINGLE_WORKLOAD, "value": p.nxy * steps / (stage_ms.sum() / 1e3), "unit": UNIT,
            "persistent": persistent,
            "steps": steps, "ms_per_step": float(stage_ms.sum() / steps),
            "l2": "flushed (512 MiB write) before every timed step",
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "kernel": "stage_kernel<128,MHD_BQlin,RK3CN_Elin>",
                         "traffic": read_traffic("stage_kernel_mri_64x64_nz128.md"),
                         "algorithmic_bytes_per_launch": sum(sb) / 3,
                         "avg_launch_ms": float(stage_ms.sum() / (3 * steps))}}


def run_plain_per_case(cases, sts, local, steps_per_case: int = 10):
    """The ensemble case after case through the plain single-case path (device time)."""
    from ql_dns_b200.solver import QLSolver
    tot = 0.0
    for p, (lin, mf, kx0) in zip(cases, sts):
        with QLSolver(p, device=local) as s:
            s.set_state(0.0, lin, mf, kx0)
            for _ in range(3):
                s.step_timed()
            t = 0.0
            for _ in range(steps_per_case):
                t += float(s.step_timed().sum())
            tot += t / steps_per_case
    modes = sum(p.nxy for p in cases)
    return {"value": modes / (tot / 1e3), "unit": UNIT, "ms_per_step": tot,
            "sample": f"{steps_per_case} steps of each case, one case after another, 3 stage launches per step"}


DNS_WORKLOAD = ("full 3-D DNS MRI, MHD shearing box 64x128x64 grid (2/3 dealiased in x, y, z; 1849 (kx,ky) columns x "
                "nz=43), Re=Rm=4000, dt=0.005, RK3CN_Elin, mean By = 0.05 sin(2 pi z), sigma=1e-2 k^-2 "
                "divergence-free fluctuations, seed 2")


def dns_flops_per_step(p, nxy, Kyn) -> float:
    """FP64 flops of the transforms of one DNS step, 5 N log2 N per complex transform
    (6 inverse and 9 forward fields per stage; two real y lines per complex transform)."""
    import math
    fz = 5 * p.NZ * math.log2(p.NZ)
    fx = 5 * p.Mx * math.log2(p.Mx)
    fy = 5 * p.My * math.log2(p.My)
    per_rhs = 15 * nxy * fz + 15 * Kyn * p.NZ * fx + 8 * p.Mx * p.NZ * fy
    return 3 * per_rhs


def run_dns(args, local):
    """The 64x128x64 DNS through QLDns: K steps timed with CUDA events on the handle's stream."""
    from ql_dns_b200.dns import QLDns
    from ql_dns_b200.initial import dns_initial_state
    from ql_dns_b200.params import dns_64x128x64
    p = dns_64x128x64()
    lin, kx0 = dns_initial_state(p, 2, sigma=1e-2, B0=0.05)
    steps = max(1, min(args.steps, 1000))
    with QLDns(p, device=local) as d:
        d.set_state(0.0, lin, kx0)
        d.step(args.warmup)
        d.set_state(0.0, lin, kx0)
        ms = d.step_timed(steps)
        rec = d.diagnostics()
        nxy = d.nxy
        Kyn = d.ny // 2
    pk = fp64_peak(local)
    flops = dns_flops_per_step(p, nxy, Kyn)
    achieved = flops * steps / (ms / 1e3) / 1e12
    out = {"workload": DNS_WORKLOAD, "value": nxy * steps / (ms / 1e3), "unit": UNIT, "steps": steps,
           "ms_per_step": ms / steps, "grid_points_per_s": p.Mx * p.My * p.NZ * steps / (ms / 1e3),
           "l2": "not flushed: the DNS state and transform scratch (~75 MB) stay in L2 across steps, as in a run",
           "roofline": {"bound": "fp64", "achieved": achieved, "peak": pk, "unit": "TFLOP/s",
                        "frac": achieved / pk, "peak_source": "measured FP64 FMA loop (qlgpu_fp64_peak)",
                        "flops_per_step": flops,
                        "kernels": "dns_inv_zx<64,64>, dns_phys<128>, dns_fwd_xz<64,64>, dns_update (x3 per step)"},
           "energy_at_end": {"t": rec[0], "E_u": rec[3], "E_b": rec[4], "E_By_mean": rec[2]},
           "gpu_launches_per_step": 14}
    if not args.no_cpu_baseline:
        from oracle.dns_oracle import DNSOracle
        D = DNSOracle(p)
        D.step(0.0, lin, kx0)  # warm-up
        n = 2
        t0 = time.perf_counter()
        t, l, k = 0.0, lin, kx0
        for _ in range(n):
            t, l, k, _ = D.step(t, l, k)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": nxy * n / dt, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"{n} steps of the same DNS with the numpy oracle ({dt:.1f} s)"}
    return out


def ensemble_parity(cases, sts, recs_e2e, outs_e2e, timed_out, args):
    """Every case of the timed ensemble against the CPU oracle (strict FP64 build, OpenMP over
    modes) from the same initial state: the end-to-end run's state and energy / stress /
    dissipation series after K steps, and the device-timed run's state after W + K steps."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()

    def rel(a, b):
        nb = np.linalg.norm(b)
        return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))

    err_e2e = err_e2e_mf = err_series = err_timed = err_timed_mf = 0.0
    for c, (p, (lin, mf, kx0)) in enumerate(zip(cases, sts)):
        t1, l1, m1, k1, d1 = O.run(p, 0.0, lin, mf, kx0, args.steps, diag_every=1, kind="strict_omp",
                                   nthreads=threads)
        err_e2e = max(err_e2e, rel(outs_e2e[c][1], l1))
        err_e2e_mf = max(err_e2e_mf, rel(outs_e2e[c][2], m1))
        dg = np.vstack(recs_e2e[c])
        d1 = d1[1:]  # the oracle's series starts with the initial record
        for col in range(1, 13):
            scale = np.abs(d1[:, col]).max()
            if scale > 0:
                err_series = max(err_series, float(np.abs(dg[:, col] - d1[:, col]).max() / scale))
        t2, l2, m2, k2, _ = O.run(p, t1, l1, m1, k1, args.warmup, kind="strict_omp", nthreads=threads)
        err_timed = max(err_timed, rel(timed_out[c][1], l2))
        err_timed_mf = max(err_timed_mf, rel(timed_out[c][2], m2))
    return {"against": "CPU oracle, strict FP64 build (-O2 -ffp-contract=off), OpenMP over modes",
            "cases": len(cases), "tolerance": 1e-10,
            "e2e_run": {"steps": args.steps, "max_rel_err_state": err_e2e, "max_rel_err_mean_field": err_e2e_mf,
                        "max_rel_err_series": err_series},
            "timed_run": {"steps": args.steps + args.warmup, "max_rel_err_state": err_timed,
                          "max_rel_err_mean_field": err_timed_mf},
            "oracle_s": time.perf_counter() - t0}


def run_gpu(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from ql_dns_b200.batch import QLBatch
    cases, b0s, _ = ensemble(0)
    modes = sum(p.nxy for p in cases)
    seed0, my_modes, job_modes = replica_plan(ws, rank, modes)
    seeds = [seed0 + c for c in range(NCASES)]
    sts = ensemble_states(cases, b0s, seeds)
    batch = QLBatch(cases, device=local)
    for c, (lin, mf, kx0) in enumerate(sts):
        batch.set_state(c, 0.0, lin, mf, kx0)
    tune_ms = batch.tune(3)
    batch.step_timed(args.warmup)
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms = batch.step_timed(args.steps)  # one persistent launch of K steps, CUDA events on the batch stream
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    job_ms = max_over_ranks(ws, ms)
    value = job_modes * args.steps / (job_ms / 1e3)
    st, ls = batch.status()
    assert ls == 0 and not any(st), (st, ls)
    mapping = batch.mapping()
    cost = batch.cost_model()
    engine = batch.engine()
    # the state after the W warm-up and K timed steps, for the parity check below
    timed_out = [batch.get_state(c) for c in range(NCASES)]

    peak, peak_kind = hbm_peak()
    alg_step = sum(algorithmic_bytes_per_step(p) for p in cases)
    achieved = alg_step * args.steps / (ms / 1e3) / 1e9
    flops_step = sum(reference_flops_per_step(p) for p in cases)
    fp64_pk = fp64_peak(local)
    fp64_ach = flops_step * args.steps / (ms / 1e3) / 1e12
    own_flops_step = sum(own_transform_flops_per_step(p) for p in cases)
    own_ach = own_flops_step * args.steps / (ms / 1e3) / 1e12

    # end to end through the batch C ABI: H2D of every case's state from pinned
    # host memory, then per step one call that advances all cases and reads the
    # 48 diagnostic records (energy / stress / dissipation) back to the host,
    # then D2H of every case's state
    def pinned_like(a):
        return torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.complex128,
                           pin_memory=True).numpy()

    pin_in, pin_out = [], []
    for lin, mf, kx0 in sts:
        lh, mh, kh = pinned_like(lin), pinned_like(mf), pinned_like(kx0)
        lh[...], mh[...], kh[...] = lin, mf, kx0
        pin_in.append((lh, mh, kh))
        pin_out.append((pinned_like(lin), pinned_like(mf), pinned_like(kx0)))
    ext = torch.cuda.ExternalStream(batch.stream())

    def e2e_run(per_step):
        """State of all cases in from pinned host memory, K steps with the energy / stress /
        dissipation record of every step read back, state of all cases out.  per_step: "async"
        (one call per step, each step's records collected while the next step runs), "sync"
        (one call per step that returns its records) or False (one call for the K steps)."""
        torch.cuda.synchronize()
        barrier(ws)
        ee0 = torch.cuda.Event(enable_timing=True)
        ee1 = torch.cuda.Event(enable_timing=True)
        ee0.record(ext)
        h0 = time.perf_counter()
        batch.set_states(0.0, pin_in)
        h1 = time.perf_counter()
        recs_all = [[] for _ in range(NCASES)]
        if per_step == "async":
            batch.step_async(1, diag_every=1)
            for s in range(args.steps):
                if s + 1 < args.steps:
                    batch.step_async(1, diag_every=1)
                for c, r in enumerate(batch.step_collect()):
                    recs_all[c].append(r)
        elif per_step == "sync":
            for _ in range(args.steps):
                for c, r in enumerate(batch.step(1, diag_every=1)):
                    recs_all[c].append(r)
        else:
            for c, r in enumerate(batch.step(args.steps, diag_every=1)):
                recs_all[c].append(r)
        h2 = time.perf_counter()
        outs = batch.get_states(pin_out)
        ee1.record(ext)
        ee1.synchronize()
        h3 = time.perf_counter()
        ms = max_over_ranks(ws, ee0.elapsed_time(ee1))
        assert sum(len(r) for rr in recs_all for r in rr) == NCASES * args.steps
        assert all(np.isfinite(o[1]).all() and np.isfinite(o[2]).all() for o in outs)
        outs = [(o[0], o[1].copy(), o[2].copy(), o[3].copy()) for o in outs]
        return ms, recs_all, outs, {"set_states_ms": 1e3 * (h1 - h0), "steps_ms": 1e3 * (h2 - h1),
                                    "get_states_ms": 1e3 * (h3 - h2)}

    def e2e_roundtrip():
        """Every step a full host round trip: the state of all cases in from pinned memory, one
        step with its records read back, the state out (a caller that keeps the state on the host)."""
        torch.cuda.synchronize()
        barrier(ws)
        ee0 = torch.cuda.Event(enable_timing=True)
        ee1 = torch.cuda.Event(enable_timing=True)
        ee0.record(ext)
        cur, nxt = pin_in, pin_out  # the last e2e use of pin_in: it is overwritten here
        for _ in range(args.steps):
            batch.set_states(0.0, cur)
            batch.step(1, diag_every=1)
            batch.get_states(nxt)
            cur, nxt = nxt, cur
        ee1.record(ext)
        ee1.synchronize()
        return max_over_ranks(ws, ee0.elapsed_time(ee1))

    e2e_run("async")  # warm-up of the one-step graph
    e2e_ms, recs_all, outs, phases = e2e_run("async")
    sync_ms, _, _, sync_phases = e2e_run("sync")
    e2e_run(False)  # warm-up: the K-step graph with records is captured and uploaded here
    one_ms, _, _, one_phases = e2e_run(False)
    rt_ms = e2e_roundtrip()
    state_bytes = sum(lin.nbytes + mf.nbytes + kx0.nbytes for lin, mf, kx0 in sts)
    e2e = {"value": job_modes * args.steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": NCASES * 15 * 8 + state_bytes / args.steps,
           "path": "QLBatch.set_states (pinned, all 48 cases), K x QLBatch.step_async(1, diag_every=1) (one "
                   "launch per step; the 48 records of each step read back by QLBatch.step_collect while the "
                   "next step runs), QLBatch.get_states (pinned)",
           "phases_host_ms": phases,
           "per_step_sync": {"value": job_modes * args.steps / (sync_ms / 1e3), "unit": UNIT,
                             "path": "as above with K x QLBatch.step(1, diag_every=1), each call waiting for its "
                                     "step and records", "phases_host_ms": sync_phases},
           "one_call": {"value": job_modes * args.steps / (one_ms / 1e3), "unit": UNIT,
                        "path": "as above with one QLBatch.step(K, diag_every=1): one launch, every step's 48 "
                                "records read back after it", "phases_host_ms": one_phases},
           "state_roundtrip_every_step": {
               "value": job_modes * args.steps / (rt_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": NCASES * 15 * 8 + state_bytes,
               "path": "every step: QLBatch.set_states (pinned) of all cases, QLBatch.step(1, diag_every=1), "
                       "QLBatch.get_states (pinned); for a caller that keeps the state in host memory"}}
    batch.close()

    parity = ensemble_parity(cases, sts, recs_all, outs, timed_out, args) if rank == 0 else None
    plain = run_plain_per_case(cases, sts, local) if rank == 0 else None
    single = run_single(args, torch.cuda.ExternalStream, local) if rank == 0 else None
    dns = run_dns(args, local) if rank == 0 else None

    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": job_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "not flushed: the ensemble state (~0.5 GB with RK buffers) exceeds the 126 MB L2",
                       "cases": NCASES, "mode_columns": modes, "mapping": mapping, "tune_probe_ms": tune_ms,
                       "cost_model": cost},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": read_traffic(KERNEL_PROFILE[engine]),
                         "kernel": KERNEL_NAME[engine], "engine": engine,
                         "algorithmic_bytes_per_step": alg_step, "avg_launch_ms": ms,
                         "fp64": {"achieved": fp64_ach, "peak": fp64_pk, "unit": "TFLOP/s", "frac": fp64_ach / fp64_pk,
                                  "flops_per_step": flops_step,
                                  "count": "reference formulation: 3 x (15 + 7) transforms x 5 NZ log2 NZ per "
                                           "mode-step; peak: measured FP64 FMA loop (qlgpu_fp64_peak)",
                                  "hbm_roofline_needs_fp64_frac": flops_step / (alg_step / (peak * 1e9)) / 1e12
                                  / fp64_pk,
                                  "actual": {"achieved": own_ach, "frac": own_ach / fp64_pk,
                                             "flops_per_step": own_flops_step,
                                             "count": "this kernel's transforms: 3 x 14 length-NZ transforms x "
                                                      "5 NZ log2 NZ per mode-step (pointwise work not counted)",
                                             "hbm_roofline_needs_fp64_frac":
                                                 own_flops_step / (alg_step / (peak * 1e9)) / 1e12 / fp64_pk}}},
            "parity": parity,
            "plain_per_case": plain,
            "speedup_vs_plain_per_case": value / plain["value"],
            "single_case": single,
            "dns": dns,
            "e2e": e2e,
            "gpu_launches": 2,
        }
        out["clocks"] = clk.summary()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if not args.no_cpu_baseline and ws == 1:
            out["cpu_baseline"] = cpu_baseline(budget_s=args.cpu_budget)
            out["cpu_baseline_1thread"] = cpu_baseline(budget_s=min(args.cpu_budget, 10.0), threads=1)
        print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
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
