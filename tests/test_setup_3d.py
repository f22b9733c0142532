"""Host-side tables of the 3D problems (titus_b200.SolverCSD3D, uploaded by
titus_create_3d) against the oracle's 3D solver data (oracle/three_d.py): the
z pair Ay / |Ay|, the reduced ordinates, the inflow factors, the boundary
cells, the sweep's restore cells and the completion candidates. No GPU."""
import numpy as np
import scipy.sparse as sp

from oracle.three_d import Settings3D as OSettings3D
from oracle.three_d import SolverCSD3D as OSolver3D
from titus_b200 import Settings3D, SolverCSD3D


def _pair(**kw):
    s, o = Settings3D(**kw), OSettings3D(**kw)
    for t in (s, o):
        t.sigmaO1Inv = t.sigmaO2Inv = t.sigmaO3Inv = 1.0 / (2 * 0.2**2)
        t.y0, t.z0 = 0.4 * kw["L"], 0.6 * kw["L"]
    return SolverCSD3D(s), OSolver3D(o)


def _csr(op, N):
    rp, ci, v = op
    return sp.csr_matrix((v, ci, rp), shape=(N, N)).toarray()


def test_tables_match_oracle():
    g, o = _pair(Nx=9, Ny=8, Nz=7, nPN=4, L=1.0)
    o.setup_directions()
    assert np.array_equal(g.idxBeam, o.idxBeam)
    assert np.array_equal(g.density, o.densityVec)
    assert np.array_equal(g.boundaryIdx, o.boundaryIdx)
    assert np.array_equal(g.x_completion, o.x_completion)
    # the z pair
    assert np.abs(_csr(g.ops3[0], g.N) - o.Ay.toarray()).max() == 0.0
    assert np.abs(_csr(g.ops3[1], g.N) - o.AbsAy.toarray()).max() <= 1e-14
    # PsiBeam: spatial profile and the inflow factor at energy index 3 (csd.S[n-1] = S[2])
    assert np.abs(g.bc_space - o.spatial_profile()).max() <= 1e-15
    f_g = g.bc_energy[3] / g.S[3] * g.S[2] * g.bc_angle
    f_o = o.inflow_factor(o.csd.eGrid[3], 3)
    assert np.abs(f_g - f_o).max() <= 1e-14 * np.abs(f_o).max()
    # restore cells: the 2D positions (L % nx, L // nx) in every z layer
    nz, nx, ny = 6, 8, 7
    a, b = o.restore_ab
    want = np.unique((np.arange(nz)[:, None] * nx * ny + (a * ny + b)[None, :]).ravel())
    assert np.array_equal(np.unique(g.sweep_restore), want)


def test_proton_problem_sizes():
    s = Settings3D()
    assert (s.NCellsX, s.NCellsY, s.NCellsZ) == (96, 96, 96)
    assert abs(s.dx - 0.1) < 1e-15 and abs(s.dz - 0.1) < 1e-15
    g = SolverCSD3D(s)
    assert g.N == 196 and g.n == 96 ** 3
    assert g.nE == 1337
    assert 1 <= g.q <= 24
    # the stopping power is positive down to the 1 MeV cutoff
    assert np.all(g.S > 0)
