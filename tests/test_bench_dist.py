"""bench.py's multi-rank path on CPU (gloo, two ranks): the slowest rank's
time sets the whole-job throughput of the replicas, and only rank 0 runs the
CPU reference arm."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    # rank r spends r + 1 seconds on 10 units each
    v = bench.replica_value(10, float(rank + 1), world)
    out.put((rank, v, bench._allreduce_max(float(rank), world)))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_value_uses_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # 2 ranks x 10 units over the slowest rank's 2 s
    assert [g[1] for g in got] == [10.0, 10.0]
    assert [g[2] for g in got] == [1.0, 1.0]


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r1 = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                         "--warmup", "3"], capture_output=True, text=True, env=env, timeout=300)
    assert r1.returncode == 0 and r1.stdout.strip() == ""
    env = dict(os.environ, WORLD_SIZE="2", RANK="0", LOCAL_RANK="0")
    r0 = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                         "--warmup", "3"], capture_output=True, text=True, env=env, timeout=300)
    assert r0.returncode == 0
    import json
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["n_gpus"] == 2
