"""Result files in the reference's formats (main.jl:189-193 VTK rectilinear
grid; SolverCSD.jl:878 writedlm text): exact FP64 round trips."""
import math

import numpy as np
import pytest

from titus_b200.output import read_vtr, write_dlm, write_dose_vtk, write_vtr
from titus_b200.settings import Settings


def test_vtr_round_trip(tmp_path):
    x = np.linspace(0.0, 1.0, 7)
    y = np.linspace(-0.5, 0.5, 5)
    rng = np.random.default_rng(0)
    a = rng.standard_normal(35) * 1e-300   # subnormal-range values survive too
    b = rng.standard_normal(35)
    p = write_vtr(str(tmp_path / "g"), x, y, {"a": a, "b": b})
    assert p.endswith(".vtr")
    x2, y2, d = read_vtr(p)
    assert np.array_equal(x2, x) and np.array_equal(y2, y)
    assert np.array_equal(d["a"], a) and np.array_equal(d["b"], b)
    head = open(p).read(200)
    assert 'type="RectilinearGrid"' in head and 'WholeExtent="0 6 0 4 0 0"' in head
    with pytest.raises(ValueError, match="grid points"):
        write_vtr(str(tmp_path / "bad"), x, y, {"a": a[:-1]})


def test_dose_vtk_fields(tmp_path):
    s = Settings(21, 21, 8, "csdWaterBeam", nPN=3)
    n = s.NCellsX * s.NCellsY
    rng = np.random.default_rng(1)
    dose = np.abs(rng.standard_normal(n))
    u = rng.standard_normal(n)
    gamma0 = 2.0
    p = write_dose_vtk(s, dose, u, gamma0, outdir=str(tmp_path))
    assert p.endswith(f"dose_csd_nx{s.NCellsX}ny{s.NCellsY}.vtr")
    x, y, d = read_vtr(p)
    assert np.array_equal(x, s.xMid) and np.array_equal(y, s.yMid)
    assert np.array_equal(d["dose"], dose)
    assert np.array_equal(d["dose_normalized"], dose / dose.max())
    assert np.array_equal(d["u"], u / 0.5 / math.sqrt(gamma0))


def test_dlm_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    W = rng.standard_normal((9, 4))
    p = write_dlm(str(tmp_path / "gifW" / "W_1"), W)
    assert np.array_equal(np.loadtxt(p, delimiter="\t"), W)
    v = rng.standard_normal(5)
    p2 = write_dlm(str(tmp_path / "v"), v)
    assert np.array_equal(np.loadtxt(p2, delimiter="\t"), v)
    assert open(p).readline().count("\t") == 3


def test_vtr_3d_round_trip(tmp_path):
    from titus_b200.output import write_dose_vtk_3d
    from titus_b200.settings import Settings3D

    s = Settings3D(Nx=6, Ny=5, Nz=4, nPN=1, L=1.0)
    n = s.NCellsX * s.NCellsY * s.NCellsZ
    rng = np.random.default_rng(3)
    dose = np.abs(rng.standard_normal(n))
    u = rng.standard_normal(n)
    p = write_dose_vtk_3d(s, dose, u, 2.0, outdir=str(tmp_path))
    assert p.endswith(f"dose_csd_nx{s.NCellsX}ny{s.NCellsY}nz{s.NCellsZ}.vtr")
    x, y, z, d = read_vtr(p, with_z=True)
    assert np.array_equal(x, s.xMid) and np.array_equal(y, s.yMid) and np.array_equal(z, s.zMid)
    assert f'WholeExtent="0 {s.NCellsX - 1} 0 {s.NCellsY - 1} 0 {s.NCellsZ - 1}"' in open(p).read(300)
    # VTK order: x fastest; the solver's row of cell (i, j, k) is (k nx + i) ny + j
    i, j, k = 3, 2, 1
    vtk = i + s.NCellsX * (j + s.NCellsY * k)
    row = (k * s.NCellsX + i) * s.NCellsY + j
    assert d["dose"][vtk] == dose[row]
    assert np.array_equal(np.sort(d["dose"]), np.sort(dose))
    assert d["u"][vtk] == u[row] / 0.5 / math.sqrt(2.0)


def test_vtr_2d_file_unchanged_by_3d_support(tmp_path):
    x = np.linspace(0.0, 1.0, 3)
    y = np.linspace(0.0, 2.0, 2)
    p = write_vtr(str(tmp_path / "p"), x, y, {"a": np.arange(6.0)})
    txt = open(p).read()
    assert '<DataArray type="Float64" Name="z" format="ascii">0.0</DataArray>' in txt
    assert 'WholeExtent="0 2 0 1 0 0"' in txt
