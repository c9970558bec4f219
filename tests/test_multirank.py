"""Host logic of `bench.py --gpus N` on two CPU ranks (gloo): every rank builds
its own planetesimal (independent instances, weak scaling), and the whole-job
number is the sum of every rank's marker updates over the slowest rank's time.
No GPU is involved."""
import hashlib
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        inst = bench.build_instance("micro", rank)
        digest = hashlib.sha256(inst.x.tobytes()).hexdigest()
        # rank r "processed" (r + 1) * 1000 units in 10 * (r + 1) ms
        units, ms = bench.reduce_job((rank + 1) * 1000, 10.0 * (rank + 1), "cpu")
        seen = [None] * ws
        dist.all_gather_object(seen, (digest, inst.marknum))
        q.put((rank, units, ms, seen))
    finally:
        dist.destroy_process_group()


def test_two_ranks_independent_instances_and_job_reduction():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, units, ms, seen in out:
        assert units == 3000.0 and ms == 20.0
        digests = [d for d, _ in seen]
        assert len(set(digests)) == ws            # each rank has its own instance
        assert len({n for _, n in seen}) == 1     # of the same size (weak scaling)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert not dist.is_initialized()
    assert bench.reduce_job(5, 7.5, "cpu") == (5.0, 7.5)
