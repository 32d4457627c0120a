"""bench.py's multi-GPU launcher on CPU: `--gpus 2` outside a launcher
starts two ranks itself (torch.distributed.run, gloo without a GPU), each
rank takes its shard of the physics blocks, and rank 0 reports n_gpus = 2
with the max over ranks of a per-rank value."""
import json
import os
import subprocess
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _run(*extra):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                           "MASTER_PORT")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--dry-run", *extra], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    return json.loads(lines[0])


def test_gpus_2_starts_two_ranks():
    rec = _run("--gpus", "2")
    assert rec["n_gpus"] == 2
    assert rec["ranks_seen"] == 0b11          # both ranks joined the reduction
    assert rec["max_over_ranks"] == 2.0       # rank 1's value: the max, not rank 0's
    assert rec["config"]["parallelism"] == "block shards x2"
    assert 0 < rec["rank0_columns"] < 884736


def test_default_is_one_rank():
    rec = _run()
    assert rec["n_gpus"] == 1 and rec["ranks_seen"] == 1
    assert rec["rank0_columns"] == 884736
