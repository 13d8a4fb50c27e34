"""The multi-GPU path is replicas only: every rank scores its own batch
(weak scaling), device times are reduced with a max over ranks and pose
counts with a sum, and the reference arm runs on rank 0 alone.  This host
logic of bench.py runs here as two gloo ranks on the CPU."""

import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes, seeds = bench.workload_sizes("uniform64x150", rank)
        usizes, useeds = bench.workload_sizes("uneven256", rank)
        bench.barrier(world)
        res = {
            "max": bench.max_over_ranks(10.0 * (rank + 1), world),
            "sum": bench.sum_over_ranks(len(sizes), world),
            "seeds": seeds[:3],
            "useeds": useeds[:3],
            "usizes": list(usizes[:5]),
        }

        class Args:
            workload = "uniform64x150"
            steps = 1
            warmup = 1
            gpus = world

        # the reference arm: ranks other than 0 do no work and exit cleanly
        if rank != 0:
            res["ref_rc"] = bench.run_reference(Args, world, rank)
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0]["max"] == got[1]["max"] == 20.0
    assert got[0]["sum"] == got[1]["sum"] == 128
    # each rank scores its own poses: weak scaling
    assert set(got[0]["seeds"]).isdisjoint(got[1]["seeds"])
    assert set(got[0]["useeds"]).isdisjoint(got[1]["useeds"])
    assert got[0]["usizes"] != got[1]["usizes"]
    assert got[1]["ref_rc"] == 0
