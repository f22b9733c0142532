"""Oracle fixture for the benchmark's accuracy check.

Runs the FP64 oracle's BUG-rejection integrator (SolverCSD.jl:2011-2374) on the
benchmark problem -- the seeded 200 x 200 water/lung/bone phantom, P29 (900
moments), rank cap 80, 5 MeV electrons at tau-CFL 0.5 -- for its first 200 loop
iterations, and stores the dose, the rank of every iteration and the final
psi in ``phantom200_P29_bug200.npz`` beside this script. ``bench.py`` runs the
same 200 iterations on the GPU after its timed region and reports the relative
L2 error of the dose against this file (``dose_rel_err_vs_oracle``).

    python tests/golden/make_bench_fixture.py      # about a minute on 8 cores
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

ITERS = 200
NX, NPN, CAP = 201, 29, 80


def main() -> None:
    from oracle.settings import Settings
    from oracle.solver import SolverCSD, solve_dlr_bug

    o = solve_dlr_bug(SolverCSD(Settings(NX, NX, CAP, "csdPhantom", nPN=NPN)), max_steps=ITERS)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "phantom200_P29_bug200.npz")
    np.savez_compressed(dst, dose=o[4], ranks=o[5][1].astype(np.int32), iters=np.int32(ITERS),
                        nx=np.int32(NX), npn=np.int32(NPN), cap=np.int32(CAP))
    print("wrote", dst, "final rank", int(o[5][1][-1]))


if __name__ == "__main__":
    main()
