"""The N-process path of bench.py on CPU: two gloo ranks (world size 2).

The B200 run launches bench.py once per GPU under torch.distributed with NCCL;
the plumbing is the same with gloo on the host: a barrier around the timed
region, the job's time is the slowest rank's, the aggregate counts every
rank's units, and only rank 0 prints.  The reference arm under N > 1 runs on
rank 0 alone; the other ranks return without work."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r'''
import datetime, io, json, os, sys, contextlib
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank=int(sys.argv[1]),
                        world_size=2, timeout=datetime.timedelta(seconds=60))
R = bench.Replicas(dist, "cpu")
r = R.rank
R.barrier()
t = R.max_over_ranks(10.0 + 5.0 * r)            # per-rank times 10 and 15 ms
agg = R.aggregate(100.0, 10.0 + 5.0 * r)        # 100 units per rank
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    printed = R.emit({{"rank": r, "value": agg}})

class Args: steps = 1; warmup = 0; gpus = 2
ran = []
bench.problem = lambda M: ran.append(1) or (_ for _ in ()).throw(SystemExit(0))
if r != 0:
    bench.run_reference_arm(Args, r)              # must return without touching the workload
world = R.world
dist.barrier()
dist.destroy_process_group()
print(json.dumps({{"rank": r, "world": world, "max": t, "agg": agg, "printed": printed,
                  "out": buf.getvalue(), "ran": len(ran)}}))
'''


def test_two_gloo_ranks(tmp_path):
    port = 29500 + (os.getpid() % 1000)
    src = tmp_path / "worker.py"
    src.write_text(WORKER.format(root=ROOT, port=port))
    env = dict(os.environ, MASTER_ADDR="127.0.0.1")
    procs = [subprocess.Popen([sys.executable, str(src), str(r)], stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True, env=env) for r in (0, 1)]
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2 and o["max"] == 15.0
        assert abs(o["agg"] - 200.0 / 0.015) < 1e-6      # all units over the slowest time
    assert outs[0]["printed"] and json.loads(outs[0]["out"])["rank"] == 0
    assert not outs[1]["printed"] and outs[1]["out"] == ""
    assert outs[1]["ran"] == 0


def test_shard_systems_and_block_diag(M):
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    systems, (n, rp, ci, v, off) = M.graph_batch(64, 1000, 8192, 8.0, 32.0, 1e-2, seed=3)
    # the block-diagonal matrix of all systems is the generator's own
    A = bench.block_diag(systems, list(range(len(systems))))
    assert A[0] == n and np.array_equal(A[1], rp) and np.array_equal(A[2], ci)
    assert np.array_equal(A[3], v) and np.array_equal(A[4], off)
    work = [len(sy[2]) for sy in systems]
    for world in (1, 2, 3, 8):
        parts = bench.shard_systems(work, world)
        assert sorted(s for p in parts for s in p) == list(range(len(systems)))
        loads = [sum(work[s] for s in p) for p in parts]
        assert max(loads) - min(loads) <= max(work)          # greedy bound


SHARD_WORKER = r'''
import datetime, json, os, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, os.path.join({root!r}, "mtl4-mirror_b200", "python"))
import torch.distributed as dist
import bench, mtlgpu as M
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank=int(sys.argv[1]),
                        world_size=2, timeout=datetime.timedelta(seconds=60))
R = bench.Replicas(dist, "cpu")
def fake_solve(A, rhs):      # stands in for the device solve: work-proportional time
    n, rp, ci, v, off = A
    assert len(rhs) == n and len(off) >= 1
    return len(ci) / 1e6, [1] * (len(off) - 1)
out = bench.batched_sharded(M, R, fake_solve)
dist.barrier()
dist.destroy_process_group()
print(json.dumps(out))
'''


def test_batched_sharded_two_gloo_ranks(tmp_path):
    # config 4 split over two ranks: every system solved once, loads balanced,
    # the job's time the slowest rank's, the same summary on both ranks
    port = 30500 + (os.getpid() % 1000)
    src = tmp_path / "shard_worker.py"
    src.write_text(SHARD_WORKER.format(root=ROOT, port=port))
    env = dict(os.environ, MASTER_ADDR="127.0.0.1")
    procs = [subprocess.Popen([sys.executable, str(src), str(r)], stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True, env=env) for r in (0, 1)]
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=300)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    assert outs[0] == outs[1]
    o = outs[0]
    assert o["ranks"] == 2 and o["all_systems_once"] and sum(o["per_rank_systems"]) == 512
    assert o["ms"] == max(o["per_rank_ms"])
    assert max(o["per_rank_ms"]) <= 1.01 * min(o["per_rank_ms"])


def test_sell_index_bytes_follows_the_library_rule(M, monkeypatch):
    # The bench counts 2 bytes of column index per entry where the library's
    # SELL-32 copies hold 16-bit offsets (every entry within 32,767 of its
    # row, MTLGPU_SELL_INDEX not 32), else 4.
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    n, rp, ci, v = M.laplacian3d(16)
    assert bench.sell_index_bytes(rp, ci) == 2
    rp2 = np.array([0, 2, 3], np.int32)
    assert bench.sell_index_bytes(rp2, np.array([0, 1, 1], np.int32)) == 2
    # 32,769 rows: one entry in row 0, one in row 32,768 on its own column
    far_rp = np.array([0, 1] + [1] * 32767 + [2], np.int32)
    assert bench.sell_index_bytes(far_rp, np.array([32767, 32768], np.int32)) == 2
    assert bench.sell_index_bytes(far_rp, np.array([32768, 32768], np.int32)) == 4
    monkeypatch.setenv("MTLGPU_SELL_INDEX", "32")
    assert bench.sell_index_bytes(rp, ci) == 4
