"""Multi-process plumbing of bench.py on CPU (gloo, world size 2): case sharding and the
max-over-ranks timing.  No GPU: the same code paths run under torchrun with NCCL on B200s."""
import importlib
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def worker(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    bench = importlib.import_module("bench")
    from datetime import timedelta
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    serve = importlib.import_module("3d_aero_lab_b200.serve")
    reqs = serve.requests(1, 64)
    mine = reqs[rank::ws]
    obj = [None] * ws
    dist.all_gather_object(obj, [(r["type"], r["cells"], r["M"]) for r in mine])
    t = bench.max_over_ranks(1.0 + rank, ws)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, obj, t, [(r["type"], r["cells"], r["M"]) for r in reqs]))


def test_case_list_shards_disjointly_and_timing_takes_the_max():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in range(ws)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, shards, t, full in out:
        assert t == 2.0                                   # max over ranks
        union = [x for s in shards for x in s]
        assert sorted(union) == sorted(full) and len(union) == 64   # disjoint cover of the case list
