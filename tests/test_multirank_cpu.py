"""The N > 1 path of the benchmark is replicas: each rank runs its own
instance, no collective on the data path, timing is the max over ranks and
only rank 0 prints.  Checked here with two gloo ranks on the CPU (the
reference arm, which runs on the host cores)."""
import json
import os
import subprocess
import sys

import pytest

from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not ref.ref_available(), reason="oracle/_ref not built")
def test_reference_arm_two_gloo_ranks():
    env = dict(os.environ, ASG_BENCH_GLOO="1", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", "29517",
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "3", "--warmup", "3", "--cells", "20000"]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def test_max_over_ranks_gloo():
    code = r'''
import os, sys
sys.path.insert(0, %r)
import torch.distributed as dist
import bench
dist.init_process_group("gloo")
r = int(os.environ["RANK"])
v = bench.max_over_ranks(dist, 1.5 + r)
assert v == 2.5, v
dist.barrier()
dist.destroy_process_group()
print("ok", r)
''' % ROOT
    import tempfile
    fd, script = tempfile.mkstemp(suffix=".py")
    with os.fdopen(fd, "w") as f:
        f.write(code)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", "29518", script]
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    finally:
        os.unlink(script)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.count("ok") == 2
