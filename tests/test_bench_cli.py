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


def test_workload_configs():
    # the config dicts both arms print, for the 2D and 3D workloads
    sys.path.insert(0, ROOT)
    import bench

    c = bench.solve_config(bench.WORKLOADS["bug"], iterations=29695)
    assert c["cells"] == 200 * 200 and c["moments"] == 900 and c["rank_cap"] == 80
    assert c["loop_iterations"] == 29695
    w3 = bench.three_d_workload(bench.WORKLOADS["pn3d"], 0)
    c3 = bench.solve_config(w3)
    assert c3["cells"] == 96 ** 3 and c3["moments"] == 196 and "rank_cap" not in c3
    w64 = bench.three_d_workload(bench.WORKLOADS["bug3d"], 64)
    assert w64["Nx"] == 65 and "64cube" in w64["name"]
    assert bench.solve_config(w64)["rank_cap"] == 40
    # the size option leaves 2D workloads alone
    assert bench.three_d_workload(bench.WORKLOADS["bug"], 64) is bench.WORKLOADS["bug"]


def test_cost_of_history_ignores_single_sample_nodes():
    sys.path.insert(0, ROOT)
    import bench

    by_rank = {2: [1.0, 1.0], 8: [3.0, 3.0], 40: [100.0]}
    # rank 10 takes rank 8's time (nearest node), not an interpolation towards rank 40
    total, direct = bench._cost_of_history(by_rank, [2, 8, 10, 40])
    assert total == 1.0 + 3.0 + 3.0 + 100.0
    assert direct == 0.75
    # rank 5 interpolates between the nodes 2 and 8
    assert bench._cost_of_history(by_rank, [5])[0] == 2.0
