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
