"""Density-weighted spatial stencils (oracle restatement of ``code/stencils.jl:7-130``).

Row/column index of cell (i, j) (1-based) is ``(i-1)*ny + j`` (``utils.jl:98-100``);
here 0-based ``i*ny + j``. Only interior cells (2..nx-1, 2..ny-1) get rows.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


class Stencils:
    def __init__(self, settings):
        rho = settings.density
        nx, ny = settings.NCellsX, settings.NCellsY
        dx, dy = settings.dx, settings.dy
        n = nx * ny
        ii, jj = np.meshgrid(np.arange(1, nx - 1), np.arange(1, ny - 1), indexing="ij")
        ii = ii.ravel()
        jj = jj.ravel()
        idx = ii * ny + jj
        ixp = (ii + 1) * ny + jj
        ixm = (ii - 1) * ny + jj
        iyp = ii * ny + jj + 1
        iym = ii * ny + jj - 1
        # L1x: stencils.jl:26-49; diagonal 2/2/dx/rho_ij, off-diagonal -1/2/dx/rho_nbr
        rows = np.concatenate([idx, idx, idx])
        cols = np.concatenate([ixm, idx, ixp])
        vals = np.concatenate([-1 / 2 / dx / rho[ii - 1, jj], 2.0 / 2 / dx / rho[ii, jj], -1 / 2 / dx / rho[ii + 1, jj]])
        self.L1x = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
        # L1y: stencils.jl:54-78
        cols = np.concatenate([iym, idx, iyp])
        vals = np.concatenate([-1 / 2 / dy / rho[ii, jj - 1], 2.0 / 2 / dy / rho[ii, jj], -1 / 2 / dy / rho[ii, jj + 1]])
        self.L1y = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
        # L2x: stencils.jl:83-103; central difference
        rows2 = np.concatenate([idx, idx])
        cols = np.concatenate([ixm, ixp])
        vals = np.concatenate([-1 / 2 / dx / rho[ii - 1, jj], 1 / 2 / dx / rho[ii + 1, jj]])
        self.L2x = sp.csr_matrix((vals, (rows2, cols)), shape=(n, n))
        # L2y: stencils.jl:108-128
        cols = np.concatenate([iym, iyp])
        vals = np.concatenate([-1 / 2 / dy / rho[ii, jj - 1], 1 / 2 / dy / rho[ii, jj + 1]])
        self.L2y = sp.csr_matrix((vals, (rows2, cols)), shape=(n, n))
