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


def test_reference_arm_maps_no_engine_code():
    """The reference arm draws its instance with the pure-Python generator and
    times the CPU restatement: the engine's library is never loaded."""
    code = ("import sys, types; sys.path.insert(0, %r); import bench; "
            "args = types.SimpleNamespace(steps=1, warmup=1); bench.run_reference(args, 1); "
            "maps = open('/proc/self/maps').read(); "
            "print('ENGINE' if 'libvfb_b200' in maps else 'CLEAN', 'ORACLE' if 'libvfb_oracle' in maps else '')"
            % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    last = r.stdout.strip().splitlines()[-1]
    assert last.split() == ["CLEAN", "ORACLE"], last


def test_scope_byte_model():
    """The per-candidate byte model: block counts of a level add up to the
    canonical candidate count, and a level tested without being stored moves
    only its operand rows."""
    sys.path.insert(0, ROOT)
    import bench
    from vfb_b200 import synth
    rows = [8, 32, 172, 1270, 8187, 58822]
    counts = synth.formula_counts(8, 7)
    for k in range(2, 7):
        full = sum(bench.level_blocks(rows, k, 1 << 62))
        # with every row of the smaller levels distinct, the canonical count
        # is the formula count of the numbering with those rows as operands
        un = rows[k - 2]
        com = sum(rows[i - 1] * rows[k - 2 - i] for i in range(1, (k - 1) // 2 + 1))
        ncom = sum(rows[i - 1] * rows[k - 2 - i] for i in range(1, k - 1))
        assert full == 4 * un + 2 * com + ncom
    assert counts[2][7] == 4 * 8
    nu, nb, nU = bench.level_blocks(rows, 7, 100)
    assert (nu, nb, nU) == (100, 0, 0)           # the ~ block comes first
    t = 63
    b = bench.scope_bytes(t, rows + [0], [8, 32, 320, 1712, 13656, 95404, 1000], tile_rows=16)
    assert abs(b[7] - 1000 * 8 * t) < 1e-6      # level 7 not stored: 1000 unary operand reads
