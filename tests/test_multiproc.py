"""Multi-process (world_size 2, gloo, CPU) checks of the replica path of bench.py:
each rank advances its own independent member with no data exchange, and the
job throughput is all ranks' steps over the slowest rank's time."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    from oracle import oracle as orc
    # one independent member per rank (seed 1 + rank), small grid
    ng, nz = 16, 3
    q3, d3, g3 = bench.initial_fields(ng, nz, 1 + rank, orc.vstrip)
    sp, st = orc.initial_state(ng, nz, q3, d3, g3)
    status, _, _ = orc.advance(sp, st, ggen=True)
    t_local = 1.0 + rank  # pretend rank 1 is slower
    value = bench.replica_throughput(3, t_local, world)
    tmax = bench.max_over_ranks(t_local, world)
    q.put((rank, status, value, tmax, float(np.abs(st.f["qs"]).sum())))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, v0, m0, q0), (r1, s1, v1, m1, q1) = res
    assert s0 == 0 and s1 == 0
    assert m0 == m1 == 2.0                 # max over ranks
    assert v0 == v1 == pytest.approx(2 * 3 / 2.0)
    assert q0 != q1                        # different seeds: independent members


def test_bench_gpus_flag_starts_the_ranks():
    """`python bench.py --gpus 2` with no torchrun environment starts two ranks
    itself (torch.distributed.run on 127.0.0.1), each with its rank and the world
    size; --rank-check keeps it to the launch (gloo, no GPU work)."""
    import json
    import subprocess
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                             "MASTER_PORT")}
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--rank-check"],
                         env=env, capture_output=True, text=True, timeout=240)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    assert lines[0]["world_size"] == 2 and lines[0]["ranks"] == [0, 1]
