"""Rank history of the benchmark solve, for the CPU baseline's cost model.

Runs the benchmark problem (seeded 200 x 200 phantom, P29, rank cap 80, BUG
with rejection, the whole 5 MeV -> 1 keV sweep) once on the GPU and stores the
rank entering every loop iteration in ``phantom200_P29_bug_ranks.npz`` beside
this script. The CPU baseline (``bench.py --impl reference`` and the
``cpu_baseline`` leg) times the FP64 oracle per iteration at the ranks it
meets in bounded windows and sums that cost over this history; it cannot run
the 29 695-iteration sweep itself within a benchmark run. Needs a CUDA GPU:

    python tests/golden/make_rank_history.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main() -> None:
    from titus_b200 import Settings, SolverCSD, _lib

    g = SolverCSD(Settings(201, 201, 80, "csdPhantom", nPN=29), team_ctas=148)
    out = g.run(_lib.TITUS_BUG_ADAPTIVE)
    it = int(out["steps"])
    ranks = out["rank_history"][:it].astype(np.int8)
    assert (ranks > 0).all()
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "phantom200_P29_bug_ranks.npz")
    np.savez_compressed(dst, ranks=ranks, iters=np.int32(it), final_rank=np.int32(out["rank"]))
    vals, cnt = np.unique(ranks, return_counts=True)
    print("wrote", dst, "iterations", it, "rank counts", dict(zip(vals.tolist(), cnt.tolist())))


if __name__ == "__main__":
    main()
