"""Result files in the reference's formats.

* VTK rectilinear grid (``code/main.jl:189-193``): ``vtk_grid(name, xMid, yMid)``
  with point arrays ``dose``, ``dose_normalized`` (= dose / max dose) and ``u``
  (= scalar flux / (1/2 sqrt(gamma_0))), written by WriteVTK.jl as a ``.vtr``
  XML file. The flat arrays go in the order the reference passes them (cell
  (i, j) at i*ny + j); WriteVTK reads a flat vector with its first grid index
  fastest, and so does any VTK reader of this file.
* Delimited text (``code/SolverCSD.jl:878``, ``writedlm(file, W*V)``): one matrix
  row per line, tab-separated.
* 3D problems (no counterpart in the reference): the same rectilinear grid with
  z coordinates, the point arrays in VTK's own order (x fastest, then y, then
  z), converted from the solver's row order (k nx + i) ny + j.

Data are written inline as ASCII with 17 significant digits, which every VTK
reader accepts and which round-trips FP64 exactly.
"""
from __future__ import annotations

import math
import os

import numpy as np


def _ascii(a) -> str:
    return " ".join(repr(float(v)) for v in np.asarray(a, dtype=np.float64).ravel())


def write_vtr(path: str, x, y, point_data: dict, z=None) -> str:
    """Rectilinear grid with coordinates x (nx), y (ny), z (nz; None = the
    plane z = [0]) and point arrays of nx*ny*nz values each, passed in the
    order the file stores them. Returns the file name (``.vtr`` appended)."""
    x = np.asarray(x, dtype=np.float64).ravel()
    y = np.asarray(y, dtype=np.float64).ravel()
    zc = None if z is None else np.asarray(z, dtype=np.float64).ravel()
    nz = 1 if zc is None else zc.size
    npts = x.size * y.size * nz
    if not path.endswith(".vtr"):
        path = path + ".vtr"
    ext = f"0 {x.size - 1} 0 {y.size - 1} 0 {nz - 1}"
    lines = ['<?xml version="1.0"?>',
             '<VTKFile type="RectilinearGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
             f'  <RectilinearGrid WholeExtent="{ext}">', f'    <Piece Extent="{ext}">', "      <PointData>"]
    for name, arr in point_data.items():
        a = np.asarray(arr, dtype=np.float64).ravel()
        if a.size != npts:
            raise ValueError(f"{name}: {a.size} values for {npts} grid points")
        lines.append(f'        <DataArray type="Float64" Name="{name}" format="ascii">{_ascii(a)}</DataArray>')
    lines += ["      </PointData>", "      <CellData>", "      </CellData>", "      <Coordinates>",
              f'        <DataArray type="Float64" Name="x" format="ascii">{_ascii(x)}</DataArray>',
              f'        <DataArray type="Float64" Name="y" format="ascii">{_ascii(y)}</DataArray>',
              ('        <DataArray type="Float64" Name="z" format="ascii">0.0</DataArray>' if zc is None else
               f'        <DataArray type="Float64" Name="z" format="ascii">{_ascii(zc)}</DataArray>'),
              "      </Coordinates>", "    </Piece>", "  </RectilinearGrid>", "</VTKFile>"]
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def write_dose_vtk(settings, dose, u, gamma0: float, name: str | None = None, outdir: str = "output") -> str:
    """``main.jl:189-193``: ``output/dose_csd_nx{NCellsX}ny{NCellsY}.vtr`` with
    dose, dose_normalized and u / 0.5 / sqrt(gamma[1])."""
    dose = np.asarray(dose, dtype=np.float64)
    if name is None:
        name = f"dose_csd_nx{settings.NCellsX}ny{settings.NCellsY}"
    return write_vtr(os.path.join(outdir, name), settings.xMid, settings.yMid, {
        "dose": dose,
        "dose_normalized": dose / dose.max(),
        "u": np.asarray(u, dtype=np.float64) / 0.5 / math.sqrt(gamma0),
    })


def write_dose_vtk_3d(settings, dose, u, gamma0: float, name: str | None = None, outdir: str = "output") -> str:
    """Dose of a 3D problem (``Settings3D``): ``output/dose_csd_nx{NX}ny{NY}nz{NZ}.vtr``
    with dose, dose_normalized and u / 0.5 / sqrt(gamma[1]) on the cell
    centres, in VTK's x-fastest order."""
    s = settings
    shape = (s.NCellsZ, s.NCellsX, s.NCellsY)

    def vtk_order(a):
        return np.asarray(a, dtype=np.float64).reshape(shape).transpose(0, 2, 1).ravel()

    dose = np.asarray(dose, dtype=np.float64)
    if name is None:
        name = f"dose_csd_nx{s.NCellsX}ny{s.NCellsY}nz{s.NCellsZ}"
    return write_vtr(os.path.join(outdir, name), s.xMid, s.yMid, {
        "dose": vtk_order(dose),
        "dose_normalized": vtk_order(dose / dose.max()),
        "u": vtk_order(np.asarray(u, dtype=np.float64) / 0.5 / math.sqrt(gamma0)),
    }, z=s.zMid)


def write_dlm(path: str, a) -> str:
    """``writedlm(path, a)``: rows of a 2-D array (a vector is one column),
    tab-separated, shortest round-trip float text."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        a = a[:, None]
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w") as f:
        for row in a:
            f.write("\t".join(repr(float(v)) for v in row) + "\n")
    return path


def read_vtr(path: str, with_z: bool = False):
    """(x, y, {name: array}) of a file written by ``write_vtr``; with
    ``with_z``, (x, y, z, {name: array})."""
    import xml.etree.ElementTree as ET

    root = ET.parse(path).getroot()
    piece = root.find("RectilinearGrid/Piece")
    coords = [np.array(e.text.split(), dtype=np.float64) for e in piece.find("Coordinates")]
    data = {e.get("Name"): np.array(e.text.split(), dtype=np.float64) for e in piece.find("PointData")}
    if with_z:
        return coords[0], coords[1], coords[2], data
    return coords[0], coords[1], data
