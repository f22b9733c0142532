"""The 3D extension of the oracle (oracle/three_d.py), pinned by reduction to
the 2D oracle: a three-layer extrusion with dz = 1e30 evolves its middle layer
as the 2D problem, for the full-rank P_N loop (SolverCSD.jl:465-586) and the
rank-adaptive BUG loop (SolverCSD.jl:2011-2374)."""
import numpy as np
import pytest

from oracle import pn
from oracle import quadrature as qd
from oracle.full_rank import solve_pn_full
from oracle.settings import Settings
from oracle.solver import SolverCSD, solve_dlr_bug
from oracle.three_d import Settings3D, SolverCSD3D, solve_pn_full_3d


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_ay_is_the_omega_y_projection():
    # z streams with Ay: it must be M diag(Omega_y) O, as Ax and Az are for x and z
    npn = 6
    Ax, Ay, Az = pn.setup_system_matrices(npn)
    pts, _ = qd.standard_points(npn + 1)
    O, M = qd.compute_trafo_matrices(npn + 1, npn)
    assert np.abs(M @ np.diag(pts[:, 1]) @ O - Ay).max() < 1e-14
    assert np.abs(Ay - Ay.T).max() == 0.0


def test_stencils_z_rows():
    # L1z / L2z rows follow stencils.jl with dz and the z neighbours' densities
    s = Settings3D(Nx=7, Ny=6, Nz=8, nPN=1)
    s.sigmaO1Inv = s.sigmaO2Inv = s.sigmaO3Inv = 1.0
    sv = SolverCSD3D(s)
    nz, nx, ny = s.NCellsZ, s.NCellsX, s.NCellsY
    rho = s.density
    f = np.random.default_rng(1).standard_normal((nz, nx, ny))
    l2 = (sv.stencil.L2z @ f.ravel()).reshape(f.shape)
    l1 = (sv.stencil.L1z @ f.ravel()).reshape(f.shape)
    g = f / rho
    e2 = (g[2:, 1:-1, 1:-1] - g[:-2, 1:-1, 1:-1]) / (2 * s.dz)
    e1 = (2 * g[1:-1, 1:-1, 1:-1] - g[2:, 1:-1, 1:-1] - g[:-2, 1:-1, 1:-1]) / (2 * s.dz)
    assert np.allclose(l2[1:-1, 1:-1, 1:-1], e2, rtol=1e-14, atol=1e-13)
    assert np.allclose(l1[1:-1, 1:-1, 1:-1], e1, rtol=1e-14, atol=1e-13)
    assert not l2[sv.face].any() and not l1[sv.face].any()


def _extruded_pair(problem, nx, npn, r):
    s2 = Settings(nx, nx, r, problem, nPN=npn)
    s3 = Settings3D.extrude(Settings(nx, nx, r, problem, nPN=npn), nz=3)
    return SolverCSD(s2), SolverCSD3D(s3), (nx - 1) * (nx - 1)


def test_full_rank_reduces_to_2d():
    o2, o3, n2 = _extruded_pair("csdPhantom", 17, 3, 4)
    u2, d2, _ = solve_pn_full(o2, max_steps=40)
    u3, d3, _ = solve_pn_full_3d(o3, max_steps=40)
    assert _rel(d3[n2:2 * n2], d2) < 1e-13
    assert _rel(u3[n2:2 * n2], u2) < 1e-13


def test_bug_reduces_to_2d():
    # the smoke case of the 2D BUG loop (well conditioned: ranks exact)
    o2, o3, n2 = _extruded_pair("csdWaterBeam", 23, 3, 8)
    r2 = solve_dlr_bug(o2, max_steps=40)
    r3 = solve_dlr_bug(o3, max_steps=40)
    nx = 22
    i, j = np.divmod(np.arange(n2), nx)
    inner = (i > 0) & (j > 0) & (i < nx - 1) & (j < nx - 1)
    assert np.array_equal(r2[5][1], r3[5][1])
    assert _rel(r3[4][n2:2 * n2][inner], r2[4][inner]) < 1e-10


@pytest.mark.parametrize("npn", [3])
def test_z_mirror_symmetry(npn):
    # a problem symmetric under z -> -z (density mirrored, beam centred in z)
    # gives a z-mirrored dose: the quadrature is symmetric under Omega_y -> -Omega_y
    s = Settings3D(Nx=11, Ny=11, Nz=11, r=6, nPN=npn, L=1.0)
    s.sigmaXInv = s.sigmaYInv = s.sigmaZInv = 1.0 / (2 * 0.1**2)
    # a wide angular profile: at P_3 no ordinate lies within 0.01 rad of +x
    s.sigmaO1Inv = s.sigmaO2Inv = s.sigmaO3Inv = 1.0 / (2 * 0.3**2)
    s.density = 0.5 * (s.density + s.density[::-1])
    s.z0 = 0.5
    sv = SolverCSD3D(s)
    _, d, _ = solve_pn_full_3d(sv, max_steps=30)
    d = d.reshape(s.NCellsZ, s.NCellsX, s.NCellsY)
    assert np.abs(d).max() > 0
    assert np.abs(d - d[::-1]).max() <= 1e-12 * np.abs(d).max()
