"""Multi-rank paths on CPU (gloo, world size 2): the timing/count reduction
the bench uses under torchrun, and the sharding of independent meshes."""
import os
import socket

import numpy as np
import pytest

from trinity_b200.dist import shard_meshes


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from trinity_b200.dist import reduce_stats
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # [triangles, round time, wall time]: rank r did (r+1)*1000 triangles in (r+1)*10 ms
        out = reduce_stats([(rank + 1) * 1000.0, (rank + 1) * 10.0, 5.0 + rank], [0], [1, 2])
        q.put((rank, out.tolist()))
    finally:
        dist.destroy_process_group()


def test_reduce_stats_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert res[r] == [3000.0, 20.0, 6.0]


def test_reduce_stats_single_process_is_identity():
    from trinity_b200.dist import reduce_stats
    assert reduce_stats([1.0, 2.0], [0], [1]).tolist() == [1.0, 2.0]


def test_shard_meshes_balanced_and_complete():
    from trinity_b200 import meshgen
    sizes = [2 * s * s for s, _, _ in meshgen.batch_specs()]
    for world in (1, 2, 4, 8):
        sh = shard_meshes(sizes, world)
        flat = sorted(i for lst in sh for i in lst)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in lst) for lst in sh]
        assert max(loads) - min(loads) <= max(sizes)
        assert sh == shard_meshes(sizes, world)


def test_reference_arm_only_rank0_prints():
    """Under torchrun the reference arm runs on rank 0 only: another rank
    exits 0 at once and prints nothing."""
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, os.path.join(repo, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-500:]
    assert r.stdout.strip() == ""
