"""bench.py's multi-rank launch path on CPU: without WORLD_SIZE, --gpus 2
re-launches the script as two ranks under torch.distributed.run; the dry run
replaces the solve by a stand-in dose but keeps the spot partition, the SUM
all-reduce of the total dose (gloo) and the max-over-ranks timing."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gpus_2_dry_run_launches_two_ranks():
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    env.pop("RANK", None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--dry-run", "--gpus", "2", "--steps", "1"],
                         capture_output=True, text=True, timeout=180, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = lines[0]
    assert d["n_gpus"] == 2 and d["dry_run"]
    # 16 stand-in spots over 2 ranks: rank 0 holds 8; the reduced total covers all 16
    assert d["spots_rank0"] == 8
    assert d["total_dose_sum"] > 0


def test_single_rank_dry_run():
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--dry-run", "--steps", "1"],
                         capture_output=True, text=True, timeout=120, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][0])
    assert d["n_gpus"] == 1 and d["spots_rank0"] == 16
