"""Per-spot tables of batched pencil-beam solves against the oracle (CPU).

A spot is the base problem with its own beam energy (eMax) and entry point
(y0): its energy grid (CSD.jl:47-89) and PsiBeam boundary values
(SolverCSD.jl:240-276) must match what the oracle's SolverCSD builds for those
settings.
"""
import numpy as np
import pytest

from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver
from titus_b200 import Settings, SolverCSD


@pytest.mark.parametrize("energy,y0", [(0.05, 0.3), (0.2, 0.62), (1.5, 0.45)])
def test_spot_tables_match_oracle(energy, y0):
    g = SolverCSD(Settings(31, 31, 12, "csdPhantom", nPN=5))
    nE, dE, S, bce, sig, bcs = g.beam_tables(energy, y0)
    os_ = OSettings(31, 31, 12, "csdPhantom", nPN=5)
    os_.eMax, os_.y0 = energy, y0
    o = OSolver(os_)
    assert nE == o.csd.eTrafo.size
    assert dE == pytest.approx(o.csd.eTrafo[1] - o.csd.eTrafo[0], rel=1e-14)
    np.testing.assert_allclose(S, o.csd.S, rtol=1e-13)
    np.testing.assert_allclose(sig[0], o.csd.sigma_at_energy(o.csd.eGrid[0]), rtol=1e-14)
    ny = os_.NCellsY
    for k in (0, nE // 2, nE - 1):
        for c in (0, 7, ny // 2, 2 * ny + ny - 1):
            i, j = divmod(c, ny)
            for kq in g.idxBeam[:3]:
                ref = o.psi_beam(o.Q_points[kq:kq + 1], o.csd.eGrid[k], os_.xMid[i], os_.yMid[j], k + 1)[0]
                ang = np.exp(-os_.sigmaO1Inv * (os_.Omega1 - g.Q_points[kq, 0]) ** 2) * \
                    np.exp(-os_.sigmaO3Inv * (os_.Omega3 - g.Q_points[kq, 2]) ** 2)
                assert bce[k] * bcs[c] * ang == pytest.approx(ref, rel=1e-12, abs=1e-300)
