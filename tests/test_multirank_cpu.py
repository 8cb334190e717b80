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
