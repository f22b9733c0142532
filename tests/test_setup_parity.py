"""Product host setup (titus_b200.physics / solver) against the oracle's restatement.

Both build the data of ``SolverCSD(settings)`` (``code/SolverCSD.jl:63-146``)
independently; the arrays handed to the device must agree.
"""
import numpy as np
import pytest

from oracle import pn as opn
from oracle import quadrature as oq
from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver
from titus_b200 import physics as ph
from titus_b200.settings import Settings
from titus_b200.solver import SolverCSD


@pytest.mark.parametrize("npn", [1, 3, 7, 13, 21])
def test_flux_matrices(npn):
    Ax, _, Az = opn.setup_system_matrices(npn)
    Px, Pz = ph.flux_matrices(npn)
    assert np.array_equal(Ax, Px) and np.array_equal(Az, Pz)
    for A, P in ((Ax, Px), (Az, Pz)):
        ref = opn.roe_abs(A).toarray()
        got = ph.roe(P)
        assert np.abs(ref - got).max() < 1e-12


@pytest.mark.parametrize("npn", [3, 7, 21])
def test_quadrature(npn):
    q = npn + 1
    O, M = oq.compute_trafo_matrices(q, npn)
    pts, w = oq.standard_points(q)
    P, Wt, O2, M2 = ph.quadrature(q, npn)
    assert np.abs(pts - P).max() < 1e-15
    assert np.abs(w - Wt).max() < 1e-15
    assert np.abs(O - O2).max() < 1e-12
    assert np.abs(M - M2).max() < 1e-12


def test_csr_roundtrip():
    Ax, Az = ph.flux_matrices(5)
    for A in (Ax, Az, ph.roe(Ax)):
        rp, ci, v = ph.to_csr(A)
        B = np.zeros_like(A)
        for m in range(A.shape[0]):
            B[m, ci[rp[m]:rp[m + 1]]] = v[rp[m]:rp[m + 1]]
        assert np.array_equal(A, B)


@pytest.mark.parametrize("problem,nx,npn", [("csdWaterBeam", 21, 5), ("csdPhantom", 31, 7), ("csdWaterBeam", 101, 21)])
def test_solver_data(problem, nx, npn):
    os_ = OSettings(nx, nx, 8, problem, nPN=npn)
    o = OSolver(os_)
    psi = o.setup_directions()
    s = Settings(nx, nx, 8, problem, nPN=npn)
    p = SolverCSD(s)
    assert np.array_equal(s.density, os_.density)
    assert s.dx == os_.dx and s.dy == os_.dy
    assert np.array_equal(p.eTrafo, o.csd.eTrafo)
    assert np.abs(p.eGrid - o.csd.eGrid).max() < 1e-14
    assert np.abs(p.S - o.csd.S).max() < 1e-14
    assert np.array_equal(p.idxBeam, o.idxBeam)
    assert np.abs(p.MReduced - o.MReduced).max() < 1e-12
    assert np.array_equal(p.x_completion, o.x_completion)
    assert np.array_equal(p.w_completion, o.w_completion)
    # separable PsiBeam equals the oracle's PsiBeam on all boundary cells, 3 energies
    nyc = s.NCellsY
    for kE in (0, 1, p.nE // 2):
        ps = np.zeros_like(psi)
        o.apply_bc(ps, o.csd.eGrid[kE], kE + 1)
        for c in np.unique(p.boundaryIdx):
            i, j = divmod(c, nyc)
            ref = ps[i, j, :]
            got = p.bc_energy[kE] * p.bc_space[c] * p.bc_angle
            assert np.allclose(got, ref, rtol=1e-13, atol=0.0)


def test_sweep_restore_quirk_ragged():
    # nx != ny: the linear-index quirk restores ordinate 0 at the transposed cells
    s = Settings(13, 9, 4, "csdWaterBeam", nPN=3)
    p = SolverCSD(s)
    nx, ny = s.NCellsX, s.NCellsY
    L = p.boundaryIdx
    expect = set(((L % nx) * ny + L // nx).tolist())
    assert set(p.sweep_restore.tolist()) == expect
    assert any(not (c // ny in (0, nx - 1) or c % ny in (0, ny - 1)) for c in expect)
