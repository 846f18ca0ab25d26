"""The N > 1 path of bench.py on CPU: two ranks in a gloo process group on
127.0.0.1 (one process per GPU on the B200 node, one per CPU rank here).

The path shards with no data-path collective: each rank generates its own
seeded shard of the full workload size (weak scaling), the job's time is the
max over ranks (one all-reduce of a scalar), and the reference arm runs on
rank 0 alone while the other ranks exit 0 without work."""
import contextlib
import io
import os
import socket
import sys
from datetime import timedelta

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench

        cpu = torch.device("cpu")
        # the job's time: the slowest rank's
        t = bench.max_over_ranks_of(1.5 + rank, world, cpu)
        # each rank's own shard: same size, different seeded operands
        wl = bench.AxpyWorkload("axpy_r256", False, 256, 2048, 0x5EED1)
        a, x, y = wl.make_host(rank)
        digest = float(np.frombuffer(x.tobytes(), dtype=np.uint32).astype(np.float64).sum())
        sums = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(sums, torch.tensor([digest], dtype=torch.float64))
        # the reference arm: ranks other than 0 return at once, printing nothing
        printed = ""
        rc = None
        if rank != 0:
            buf = io.StringIO()
            with contextlib.redirect_stdout(buf):
                rc = bench.run_reference(type("A", (), {"workload": "axpy_r256", "steps": 1, "warmup": 0, "gpus": world})())
            printed = buf.getvalue()
        dist.barrier()
        out.put((rank, t, [float(s.item()) for s in sums], x.shape, rc, printed))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        rank, t, sums, shape, rc, printed = q.get(timeout=240)
        res[rank] = (t, sums, shape, rc, printed)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # max over ranks seen identically by both
    assert res[0][0] == res[1][0] == 2.5
    # the same shard size on every rank, different operands
    assert res[0][2] == res[1][2]
    assert res[0][1] == res[1][1] and res[0][1][0] != res[0][1][1]
    # rank 1 skips the reference arm without output
    assert res[1][3] == 0 and res[1][4] == ""
    assert bench_shard_seed_is_distinct()


def bench_shard_seed_is_distinct():
    sys.path.insert(0, ROOT)
    import bench

    seeds = {bench.shard_seed(0x5EED1, r) for r in range(8)}
    return len(seeds) == 8
