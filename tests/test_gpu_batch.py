"""Batched ensemble (one persistent cooperative launch for many cases) against
the CPU oracle, case by case, through the C ABI (qlgpu_batch_*).

Tolerance: relative L2 error <= 1e-10 for every case's state after N steps and
for its energy / stress / dissipation series, as for the single-case step.
"""
import numpy as np
import pytest

from gpu_util import rel, require_gpu
from oracle import oracle as O
from ql_dns_b200.batch import QLBatch, mri_ensemble
from ql_dns_b200.initial import initial_state
from ql_dns_b200.params import QLParams
from ql_dns_b200.solver import QLSolver

pytestmark = pytest.mark.gpu
TOL = 1e-10


def series_rel(dg, do):
    errs = []
    for c in range(1, 13):
        scale = np.abs(do[:, c]).max()
        if scale > 0:
            errs.append(np.abs(dg[:, c] - do[:, c]).max() / scale)
    return max(errs)


def mixed_cases(model=0, integ=0):
    """Uneven mode counts, every NZ, different nu / eta / mean fields."""
    specs = [(8, 6, 16, 1 / 700), (16, 16, 32, 1 / 2000), (8, 8, 64, 1 / 3000), (12, 10, 32, 1 / 1500),
             (6, 8, 128, 1 / 5000), (10, 4, 256, 1 / 9000), (20, 20, 64, 1 / 4000)]
    cases = []
    for i, (nx, ny, NZ, eta) in enumerate(specs):
        cases.append(QLParams(model=model, integrator=integ, nx=nx, ny=ny, NZ=NZ, nu=eta * (1 + i % 3), eta=eta,
                              dt=0.01, B0z=0.02 if model else 0.0, omega=0.9))
    return cases


def states(cases, sigma=0.2):
    out = []
    for i, p in enumerate(cases):
        out.append(initial_state(p, 100 + i, sigma=sigma, B0=0.03 + 0.01 * i, mean_u=0.01 if p.model else 0.0))
    return out


def bq_cases(integ=0):
    """MHD_BQlin cases of every NZ the chunk-queue engine takes (16 ... 128), uneven mode counts."""
    specs = [(8, 6, 16, 1 / 700), (16, 16, 32, 1 / 2000), (8, 8, 64, 1 / 3000), (12, 10, 32, 1 / 1500),
             (6, 8, 128, 1 / 5000), (20, 20, 64, 1 / 4000), (18, 14, 128, 1 / 6000), (34, 30, 32, 1 / 800)]
    return [QLParams(integrator=integ, nx=nx, ny=ny, NZ=NZ, nu=eta * (1 + i % 3), eta=eta, dt=0.01)
            for i, (nx, ny, NZ, eta) in enumerate(specs)]


def run_batch(cases, sts, n, diag_every=1, mapping=None, tune=0, engine=None, chunks=None, noise=None):
    require_gpu()
    res = []
    with QLBatch(cases) as b:
        for c, args in (noise or {}).items():
            b.set_noise(c, *args[:4], **args[4] if len(args) > 4 else {})
        if engine is not None:
            b.set_engine(engine)
            assert b.engine() == engine
        if chunks is not None:
            b.set_chunks(chunks)
        if mapping is not None:
            b.set_mapping(*mapping)
        for c, (lin, mf, kx0) in enumerate(sts):
            b.set_state(c, 0.0, lin, mf, kx0)
        if tune:
            b.tune(tune)
        d0 = [b.diagnostics(c) for c in range(len(cases))]
        d = b.step(n, diag_every=diag_every)
        for c in range(len(cases)):
            t, lo, mo, ko = b.get_state(c)
            res.append((t, lo, mo, ko, np.vstack([d0[c][None], d[c]]) if diag_every else None))
        st, ls = b.status()
        assert ls == 0 and all(s == 0 for s in st)
        m = b.mapping()
    return res, m


@pytest.mark.parametrize("model", [0, 1])
@pytest.mark.parametrize("integ", [0, 1])
def test_batch_matches_oracle(model, integ):
    cases = mixed_cases(model, integ)
    sts = states(cases)
    n = 30
    res, m = run_batch(cases, sts, n)
    for p, (lin, mf, kx0), (t, lo, mo, ko, d) in zip(cases, sts, res):
        t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, n, diag_every=1)
        assert t == t2 and np.array_equal(ko, ko2)
        assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (p, rel(lo, lo2), rel(mo, mo2))
        assert d.shape == d2.shape and series_rel(d, d2) < TOL


def test_batch_equals_single_case_path_bitwise():
    # With the same CTA count and width as the single-case handle, a case's sums
    # run in the same order: the batch reproduces the single-case step exactly.
    cases = [c for c in mixed_cases() if c.NZ <= 64] + [QLParams(nx=32, ny=32, NZ=64, dt=0.01),
                                                         QLParams(nx=24, ny=16, NZ=32, dt=0.01)]
    sts = states(cases)
    groups = {}
    for p, st in zip(cases, sts):
        with QLSolver(p) as s:
            info = s.launch_info()
            s.set_state(0.0, *st)
            s.step(12)
            groups.setdefault(info["warps"], []).append((p, st, info["grid"], s.get_state()))
    compared = 0
    for w, items in groups.items():
        cs = [it[0] for it in items]
        res, m = run_batch(cs, [it[1] for it in items], 12, diag_every=0, mapping=(w, [it[2] for it in items]))
        assert m["warps"] == w
        for (t, lo, mo, ko, _), it in zip(res, items):
            t2, lo2, mo2, ko2 = it[3]
            assert t == t2
            assert np.array_equal(lo, lo2) and np.array_equal(mo, mo2) and np.array_equal(ko, ko2)
            compared += 1
    assert compared >= 2


def test_batch_mapping_and_width_independent():
    # different CTA counts / widths / packing change only the order of sums over CTAs
    cases = mixed_cases()
    sts = states(cases)
    a, _ = run_batch(cases, sts, 20, diag_every=0, mapping=(6, [1] * len(cases)))
    b, mb = run_batch(cases, sts, 20, diag_every=0, mapping=(3, [2, 3, 2, 4, 1, 2, 5]))
    assert mb["warps"] == 3
    for x, y in zip(a, b):
        assert rel(x[1], y[1]) < 1e-12 and rel(x[2], y[2]) < 1e-12


def test_batch_tune_keeps_state_and_parity():
    cases = mixed_cases()
    sts = states(cases)
    require_gpu()
    with QLBatch(cases) as b:
        for c, (lin, mf, kx0) in enumerate(sts):
            b.set_state(c, 0.0, lin, mf, kx0)
        ms = b.tune(2)
        assert ms > 0
        for c, (lin, mf, kx0) in enumerate(sts):
            t, lo, mo, ko = b.get_state(c)
            assert t == 0.0 and np.array_equal(lo, lin) and np.array_equal(mo, mf) and np.array_equal(ko, kx0)
        b.step(7)
        b.step(6)  # two launches: the lin buffer parity carries over
        for p, (lin, mf, kx0), c in zip(cases, sts, range(len(cases))):
            t, lo, mo, ko = b.get_state(c)
            t2, lo2, mo2, ko2, _ = O.run(p, 0.0, lin, mf, kx0, 13)
            assert abs(t - t2) < 1e-15 and rel(lo, lo2) < TOL and rel(mo, mo2) < TOL


def test_batch_without_graph(monkeypatch):
    monkeypatch.setenv("QLGPU_BATCH_GRAPH", "0")
    cases = mixed_cases()[:3]
    sts = states(cases)
    res, _ = run_batch(cases, sts, 9)
    for p, (lin, mf, kx0), (t, lo, mo, ko, d) in zip(cases, sts, res):
        t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 9, diag_every=1)
        assert rel(lo, lo2) < TOL and series_rel(d, d2) < TOL


def test_batch_ensemble_law_short():
    # the 48-case MRI ensemble (mode grids 16..64 squared, NZ 32..128) for a few steps
    cases, b0s, seeds = mri_ensemble()
    sts = [initial_state(p, s, sigma=1e-3, B0=b0) for p, b0, s in zip(cases, b0s, seeds)]
    res, m = run_batch(cases, sts, 3, diag_every=1, tune=2)
    assert 1 <= m["grid"] <= 2 * 148
    for c in (0, 17, 47):
        p = cases[c]
        lin, mf, kx0 = sts[c]
        t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 3, diag_every=1)
        assert rel(res[c][1], lo2) < TOL and rel(res[c][2], mo2) < TOL
        assert series_rel(res[c][4], d2) < TOL


def test_batch_wait_bound_reports_timeout():
    # A case loses one of its work items, so its other CTAs wait for a stage that
    # never completes: the bounded wait ends the launch with a status, and the
    # batch is usable again after a new mapping and state.
    from ql_dns_b200._capi import QLGPUError
    cases = mixed_cases()[:3]
    sts = states(cases)
    require_gpu()
    with QLBatch(cases) as b:
        b.set_mapping(6, [2, 2, 1])
        for c, (lin, mf, kx0) in enumerate(sts):
            b.set_state(c, 0.0, lin, mf, kx0)
        b.set_wait(0.2)
        b.debug_drop_item(0)
        with pytest.raises(QLGPUError) as ei:
            b.step(2)
        assert ei.value.code == 4 and "waiting" in str(ei.value)
        st, ls = b.status()
        assert ls & 8
        b.set_mapping(6, [2, 2, 1])
        for c, (lin, mf, kx0) in enumerate(sts):
            b.set_state(c, 0.0, lin, mf, kx0)
        b.step(4)
        st, ls = b.status()
        assert ls == 0
        for p, (lin, mf, kx0), c in zip(cases, sts, range(3)):
            t, lo, mo, ko = b.get_state(c)
            t2, lo2, mo2, ko2, _ = O.run(p, 0.0, lin, mf, kx0, 4)
            assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL


def test_batch_of_tiny_and_ragged_cases():
    # one-column, ky = 0 only and odd-sized mode grids next to a regular case, and a batch of one
    shapes = [(2, 2), (4, 2), (2, 4), (6, 10), (4, 18), (16, 16)]
    cases = [QLParams(nx=nx, ny=ny, NZ=32, dt=0.02, nu=1 / 1500, eta=1 / 1500) for nx, ny in shapes]
    sts = [initial_state(p, 50 + i, sigma=0.3, B0=0.05) for i, p in enumerate(cases)]
    for sub in (cases, cases[3:4]):
        idx = [cases.index(p) for p in sub]
        res, m = run_batch(sub, [sts[i] for i in idx], 8)
        for p, i, (t, lo, mo, ko, d) in zip(sub, idx, res):
            t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, *sts[i], 8, diag_every=1)
            assert np.array_equal(ko, ko2)
            assert (np.linalg.norm(lo2) == 0 and np.abs(lo).max() == 0) or rel(lo, lo2) < TOL
            assert rel(mo, mo2) < TOL and series_rel(d, d2) < TOL


# ---------------------------------------------------------------------------
# Chunk-queue engine (MHD_BQlin, NZ <= 128): the default for such batches
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("integ", [0, 1])
def test_queue_engine_matches_oracle(integ):
    cases = bq_cases(integ)
    sts = states(cases)
    n = 30
    res, m = run_batch(cases, sts, n, engine="queue")
    assert m["warps"] == 12
    for p, (lin, mf, kx0), (t, lo, mo, ko, d) in zip(cases, sts, res):
        t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, n, diag_every=1)
        assert t == t2 and np.array_equal(ko, ko2)
        assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (p, rel(lo, lo2), rel(mo, mo2))
        assert d.shape == d2.shape and series_rel(d, d2) < TOL


def test_queue_engine_is_the_default_and_chunking_independent():
    # chunk sizes change only which CTA steps which modes and how many chunk sums there are
    cases = bq_cases()
    sts = states(cases)
    with QLBatch(cases) as b:
        assert b.engine() == "queue"
    a, ma = run_batch(cases, sts, 20, diag_every=0, chunks=[1, 1, 1, 1])
    c, mc = run_batch(cases, sts, 20, diag_every=0, chunks=[3, 2, 5, 1])
    assert ma["ncta"] != mc["ncta"]
    for x, y in zip(a, c):
        assert rel(x[1], y[1]) < 1e-12 and rel(x[2], y[2]) < 1e-12
    # the same chunking twice is bit for bit the same
    c2, _ = run_batch(cases, sts, 20, diag_every=0, chunks=[3, 2, 5, 1])
    for x, y in zip(c, c2):
        assert np.array_equal(x[1], y[1]) and np.array_equal(x[2], y[2])


def test_queue_engine_matches_item_engine():
    cases = bq_cases()
    sts = states(cases)
    a, _ = run_batch(cases, sts, 25, diag_every=5, engine="queue")
    b, _ = run_batch(cases, sts, 25, diag_every=5, engine="items")
    for x, y in zip(a, b):
        assert np.array_equal(x[3], y[3])
        assert rel(x[1], y[1]) < 1e-12 and rel(x[2], y[2]) < 1e-12 and series_rel(x[4], y[4]) < 1e-12


def test_queue_engine_tune_keeps_state_and_parity():
    cases = bq_cases()
    sts = states(cases)
    require_gpu()
    with QLBatch(cases) as b:
        for c, (lin, mf, kx0) in enumerate(sts):
            b.set_state(c, 0.0, lin, mf, kx0)
        assert b.tune(2) > 0 and b.engine() == "queue"
        for c, (lin, mf, kx0) in enumerate(sts):
            t, lo, mo, ko = b.get_state(c)
            assert t == 0.0 and np.array_equal(lo, lin) and np.array_equal(mo, mf)
        b.step(5)
        b.step(4)
        for p, (lin, mf, kx0), c in zip(cases, sts, range(len(cases))):
            t, lo, mo, ko = b.get_state(c)
            t2, lo2, mo2, ko2, _ = O.run(p, 0.0, lin, mf, kx0, 9)
            assert abs(t - t2) < 1e-15 and rel(lo, lo2) < TOL and rel(mo, mo2) < TOL


def test_queue_engine_wait_bound_reports_timeout():
    # one chunk of case 1 is left out of every stage: the case's next stage never
    # becomes ready, the bounded wait ends the launch with a status, and the batch
    # is usable again after set_engine and set_state
    from ql_dns_b200._capi import QLGPUError
    cases = bq_cases()[:4]
    sts = states(cases)
    require_gpu()
    with QLBatch(cases) as b:
        b.set_chunks([1, 1, 1, 1])
        for c, (lin, mf, kx0) in enumerate(sts):
            b.set_state(c, 0.0, lin, mf, kx0)
        b.set_wait(0.2)
        b.debug_drop_item(1)
        with pytest.raises(QLGPUError) as ei:
            b.step(2)
        assert ei.value.code == 4 and "waiting" in str(ei.value)
        st, ls = b.status()
        assert ls & 8
        b.set_engine("queue")
        for c, (lin, mf, kx0) in enumerate(sts):
            b.set_state(c, 0.0, lin, mf, kx0)
        b.step(4)
        st, ls = b.status()
        assert ls == 0
        for p, (lin, mf, kx0), c in zip(cases, sts, range(4)):
            t, lo, mo, ko = b.get_state(c)
            t2, lo2, mo2, ko2, _ = O.run(p, 0.0, lin, mf, kx0, 4)
            assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL


@pytest.mark.parametrize("engine", ["queue", "items"])
def test_set_states_get_states_match_per_case_calls(engine):
    # every case in one call (some with their own kx0, some with the default table) and out
    # again in one call, against the per-case entry points
    cases = bq_cases()
    base = states(cases)  # kx0 of initial_state is the default table
    sts = [(lin, mf, kx0 + 0.5 * (2 * np.pi / p.L[0]) if c % 2 else None)
           for c, (p, (lin, mf, kx0)) in enumerate(zip(cases, base))]
    require_gpu()
    with QLBatch(cases) as b:
        b.set_engine(engine)
        b.set_states(0.25, sts)
        b.step(6)
        a = b.get_states()
        for c, (lin, mf, kx0) in enumerate(sts):
            b.set_state(c, 0.25, lin, mf, kx0)
        b.step(6)
        for c in range(len(cases)):
            t, lo, mo, ko = b.get_state(c)
            assert a[c][0] == t and np.array_equal(a[c][1], lo) and np.array_equal(a[c][2], mo)
            assert np.array_equal(a[c][3], ko)
    for p, (lin, mf, kx0), (_, _, k_default), (t, lo, mo, ko) in zip(cases, sts, base, a):
        t2, lo2, mo2, ko2, _ = O.run(p, 0.25, lin, mf, k_default if kx0 is None else kx0, 6)
        assert abs(t - t2) < 1e-15 and rel(lo, lo2) < TOL and np.array_equal(ko, ko2)


@pytest.mark.parametrize("engine", ["queue", "items"])
def test_step_async_matches_step(engine):
    # two outstanding one-step calls at a time, every step's records collected while the next
    # step runs: the same records and state as one synchronous call per step
    from ql_dns_b200._capi import QLGPUError
    cases = bq_cases()[:5]
    sts = states(cases)
    require_gpu()
    with QLBatch(cases) as b:
        b.set_engine(engine)
        b.set_states(0.0, sts)
        sync = [b.step(1, diag_every=1) for _ in range(5)]
        a = b.get_states()
        b.set_states(0.0, sts)
        got = []
        b.step_async(1, diag_every=1)
        for _ in range(4):
            b.step_async(1, diag_every=1)
            with pytest.raises(QLGPUError):
                b.step_async(1, diag_every=1)  # a third outstanding call
            with pytest.raises(QLGPUError):
                b.get_states()  # state moves wait for the outstanding steps
            got.append(b.step_collect())
        got.append(b.step_collect())
        with pytest.raises(QLGPUError):
            b.step_collect()  # nothing outstanding
        g = b.get_states()
    for rs, rg in zip(sync, got):
        for x, y in zip(rs, rg):
            assert x.shape == (1, 15) and np.array_equal(x, y)
    for x, y in zip(a, g):
        assert x[0] == y[0] and np.array_equal(x[1], y[1]) and np.array_equal(x[2], y[2])


@pytest.mark.parametrize("engine", ["queue", "items"])
def test_batch_noise_per_case_matches_oracle(engine):
    # Model::DrivingNoise inside the batch step (main.cpp:111-113): each case its own
    # f_noise, band and seed, or none; the counter restarts with the case's state
    cases = bq_cases()[:6]
    sts = states(cases, sigma=1e-3)
    n = 12
    noise = {0: (0.05, 0.5, 40.0, 11), 2: (0.02, 1.0, 80.0, 12), 4: (0.08, 0.0, 30.0, 13),
             5: (0.03, 0.5, 50.0, 14)}
    res, _ = run_batch(cases, sts, n, diag_every=3, engine=engine, noise=noise)
    for c, (p, (lin, mf, kx0), (t, lo, mo, ko, d)) in enumerate(zip(cases, sts, res)):
        if c in noise:
            f, klo, khi, seed = noise[c]
            t2, lo2, mo2, ko2, d2, _ = O.run_forced(p, 0.0, lin, mf, kx0, n, diag_every=3, f_noise=f, k_lo=klo,
                                                    k_hi=khi, seed=seed)
        else:
            t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, n, diag_every=3)
        assert t == t2 and np.array_equal(ko, ko2)
        assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (c, rel(lo, lo2), rel(mo, mo2))
        assert d.shape == d2.shape and series_rel(d, d2) < TOL


def test_batch_fullqlin_noise_matches_oracle():
    # MHD_FullQlin cases (work-item engine) with the ky = 0 conjugate pairs and the
    # drive_only_* switches (MHD_FullQlin.cpp:21-22,786-1045)
    cases = [c for c in mixed_cases(model=1) if c.NZ <= 128][:4]
    sts = states(cases, sigma=1e-3)
    n = 10
    noise = {0: (0.05, 0.5, 40.0, 21), 1: (0.04, 0.5, 60.0, 22, {"drive_only_velocity": True}),
             3: (0.06, 0.0, 50.0, 23, {"drive_only_magnetic": True})}
    res, _ = run_batch(cases, sts, n, diag_every=5, engine="items", noise=noise)
    for c, (p, (lin, mf, kx0), (t, lo, mo, ko, d)) in enumerate(zip(cases, sts, res)):
        if c in noise:
            a = noise[c]
            kw = a[4] if len(a) > 4 else {}
            t2, lo2, mo2, ko2, d2, _ = O.run_forced(p, 0.0, lin, mf, kx0, n, diag_every=5, f_noise=a[0], k_lo=a[1],
                                                    k_hi=a[2], seed=a[3], **kw)
        else:
            t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, n, diag_every=5)
        assert t == t2 and np.array_equal(ko, ko2)
        assert rel(lo, lo2) < TOL and rel(mo, mo2) < TOL, (c, rel(lo, lo2), rel(mo, mo2))
        assert d.shape == d2.shape and series_rel(d, d2) < TOL


def test_default_chunk_passes_give_every_sm_a_chunk():
    # sixteen 32x32-mode NZ=64 cases (the adjoint workload): four CTA passes per chunk would
    # make 64 chunks for 148 SMs, so the default takes fewer; the 48-case ensemble keeps four
    require_gpu()
    small = [QLParams(nx=32, ny=32, NZ=64, dt=0.01) for _ in range(16)]
    with QLBatch(small) as b:
        b.set_engine("queue")
        m = b.mapping()
        assert m["chunk_passes"][64] < 4
        assert sum(m["ncta"]) >= 100, m["ncta"]
    cases, _, _ = mri_ensemble(48)
    with QLBatch(cases) as b:
        b.set_engine("queue")
        assert all(v == 4 for v in b.mapping()["chunk_passes"].values())
