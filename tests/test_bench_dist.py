"""The multi-rank harness of bench.py on the CPU: replicas exchange nothing
but their timings (MAX over ranks) and work counts (SUM), checked with two
`gloo` ranks; and under torchrun with two ranks the reference arm prints one
line from rank 0 while the other rank exits without work."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.reduce_over_ranks(dist, 10.0 * (rank + 1), dist.ReduceOp.MAX, "cpu")
        n = bench.reduce_over_ranks(dist, 8.0, dist.ReduceOp.SUM, "cpu")
        q.put((rank, t, n))
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_gloo_world2():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29650 + os.getpid() % 200
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps)
    out = sorted(q.get(timeout=10) for _ in range(2))
    # every rank sees the slowest rank's time and the total work
    assert out == [(0, 20.0, 16.0), (1, 20.0, 16.0)]


def test_reduce_over_ranks_without_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(None, 3.5, None, "cpu") == 3.5


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_driver")),
                    reason="oracle/_ref not built")
def test_reference_arm_under_torchrun_two_ranks():
    port = 29850 + os.getpid() % 100
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port),
                        os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--ref-iter-cap", "10", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
