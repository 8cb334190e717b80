"""The N > 1 path of bench.py on CPU ranks (gloo, world size 2): replica
planning, barrier and the max-over-ranks job time.  No GPU needed."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import bench
    w, r, _ = bench.dist_setup("gloo")
    assert (w, r) == (ws, rank)
    cases, _, _ = bench.ensemble(r)
    modes = sum(p.nxy for p in cases)
    seed, mine, total = bench.replica_plan(w, r, modes)
    bench.barrier(w)
    t = bench.max_over_ranks(w, 10.0 + r)
    out[rank] = (seed, mine, total, t)
    import torch.distributed as dist
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_and_max_time():
    ws, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(ws, port, out), nprocs=ws, join=True, start_method="spawn")
    assert out[0][3] == out[1][3] == 11.0          # slowest rank's time on every rank
    assert out[0][2] == out[1][2] == 2 * out[0][1]  # job total = sum of replicas
    assert {out[0][0], out[1][0]} == {0, 48}        # disjoint initial-condition seed ranges


def _dying_worker(rank, ws, port, out, mode):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import time

    import bench
    w, r, _ = bench.dist_setup("gloo", timeout_s=5.0)
    if r == 1:
        if mode == "exit":
            os._exit(3)      # the rank dies between steps, with no collective in flight
        time.sleep(30)       # "hang": the rank never reaches its next collective
        os._exit(0)
    t0 = time.time()
    try:
        bench.barrier(w)
        bench.max_over_ranks(w, 1.0)
        out[rank] = ("ok", time.time() - t0)
    except Exception as e:  # the surviving rank learns of the failure on the host
        out[rank] = ("error:" + type(e).__name__, time.time() - t0)
    os._exit(0)


@pytest.mark.parametrize("mode", ["exit", "hang"])
def test_failed_rank_ends_the_other_ranks_collective_with_an_error(mode):
    # host-side failure injection: rank 1 exits, or stops answering, after the rendezvous;
    # rank 0's next collective must fail (connection loss or the 5 s process-group
    # timeout) rather than wait for good
    import multiprocessing as mpx
    ws, port = 2, _free_port()
    ctx = mpx.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_dying_worker, args=(r, ws, port, out, mode)) for r in range(ws)]
    for p_ in procs:
        p_.start()
    procs[0].join(60)
    alive = procs[0].is_alive()
    for p_ in procs:
        if p_.is_alive():
            p_.kill()
        p_.join(10)
    assert not alive, "rank 0 hung on a dead peer"
    status, waited = out[0]
    assert status.startswith("error:"), status
    assert waited < 40
    if mode == "exit":
        assert procs[1].exitcode == 3
