"""``solveFlux!(obj, phi, flux)`` (code/SolverCSD.jl:295-386) on the GPU.

The second-order limited upwind flux of the uncollided ordinates (limiter
``slopefit`` over ``minmod``, :288-293), computed by the CUDA operator
``titus_limited_flux`` of libtitus. Arrays are (nx, ny, q) float64 with the
ordinate fastest (cell (i, j) at row i*ny + j, as psi everywhere in this
package). Only interior cells 2 <= i < nx-2, 2 <= j < ny-2 are written, as in
the reference; the other entries of ``flux`` keep their values.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _check_tensor(t, name, shape=None):
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise TypeError(f"{name}: expected a contiguous float64 CUDA tensor")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name}: shape {tuple(t.shape)}, expected {tuple(shape)}")


def limited_flux_device(phi, flux, omega_x, omega_z, dx: float, dy: float, stream=None):
    """Device path: ``phi``, ``flux`` (nx, ny, q) and ``omega_x``, ``omega_z`` (q,)
    are float64 CUDA tensors; runs asynchronously on ``stream`` (a
    torch.cuda.Stream; default: the current stream) and updates ``flux``."""
    import torch

    _check_tensor(phi, "phi")
    if phi.dim() != 3:
        raise ValueError("phi: expected (nx, ny, q)")
    nx, ny, q = phi.shape
    _check_tensor(flux, "flux", phi.shape)
    _check_tensor(omega_x, "omega_x", (q,))
    _check_tensor(omega_z, "omega_z", (q,))
    s = (stream if stream is not None else torch.cuda.current_stream()).cuda_stream
    lib = _lib.load()
    _lib.check(lib.titus_limited_flux(nx, ny, q, float(dx), float(dy), omega_x.data_ptr(), omega_z.data_ptr(),
                                      phi.data_ptr(), flux.data_ptr(), s), "titus_limited_flux")
    return flux


def solveFlux(solver, phi, flux):
    """``solveFlux!(obj, phi, flux)``: ordinates ``solver.qReduced`` (x and z
    components), spacing ``solver.settings.dx``, ``.dy``. ``phi`` and ``flux``
    are numpy arrays (copied to the GPU and back; ``flux`` is updated in place)
    or CUDA tensors (updated in place on the current stream)."""
    import torch

    ox = np.ascontiguousarray(solver.qReduced[:, 0], dtype=np.float64)
    oz = np.ascontiguousarray(solver.qReduced[:, 2], dtype=np.float64)
    dx, dy = solver.settings.dx, solver.settings.dy
    if isinstance(phi, torch.Tensor):
        dev = phi.device
        limited_flux_device(phi, flux, torch.from_numpy(ox).to(dev), torch.from_numpy(oz).to(dev), dx, dy)
        return flux
    phi = np.asarray(phi)
    if phi.dtype != np.float64 or flux.dtype != np.float64 or flux.shape != phi.shape or phi.ndim != 3:
        raise ValueError("phi, flux: float64 arrays of one (nx, ny, q) shape")
    dev = torch.device("cuda", torch.cuda.current_device())
    d_phi = torch.from_numpy(np.ascontiguousarray(phi)).to(dev)
    d_flux = torch.from_numpy(np.ascontiguousarray(flux)).to(dev)
    limited_flux_device(d_phi, d_flux, torch.from_numpy(ox).to(dev), torch.from_numpy(oz).to(dev), dx, dy)
    flux[...] = d_flux.cpu().numpy()
    return flux
