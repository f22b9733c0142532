"""Second-order limited upwind flux (solveFlux!, SolverCSD.jl:295-386):
the FP64 restatement against a literal transcription of the reference loops and
known answers; the CUDA operator titus_limited_flux bit for bit against it."""
import ctypes as C

import numpy as np
import pytest

from oracle.flux import limited_flux, limited_flux_loops, slopefit
from titus_b200 import _lib


def _case(seed, shape, zeros=True):
    rng = np.random.default_rng(seed)
    phi = rng.standard_normal(shape)
    q = shape[2]
    ox = rng.uniform(-1, 1, q)
    oz = rng.uniform(-1, 1, q)
    if zeros and q >= 4:
        ox[0], oz[1], ox[2], oz[3] = 0.0, 0.0, -0.0, -0.0   # >= 0 takes the positive branch, -0.0 included
    return phi, ox, oz, rng.standard_normal(shape)


@pytest.mark.parametrize("shape", [(11, 9, 6), (5, 7, 4), (8, 5, 3), (4, 9, 2), (6, 6, 1)])
def test_oracle_matches_reference_loops(shape):
    phi, ox, oz, f0 = _case(1, shape)
    a = limited_flux(phi, ox, oz, 0.1, 0.07, f0)
    b = limited_flux_loops(phi, ox, oz, 0.1, 0.07, f0)
    assert np.array_equal(a, b)
    nx, ny, _ = shape
    inner = np.zeros(shape, bool)
    inner[2:nx - 2, 2:ny - 2] = True
    assert np.array_equal(a[~inner], f0[~inner])      # cells outside 3:N-2 untouched


def test_slopefit_known_values():
    # monotonised central limiter: linear data keeps its slope, extrema flatten
    assert slopefit(1.0, 2.0, 3.0) == 1.0
    assert slopefit(3.0, 2.0, 1.0) == -1.0
    assert slopefit(1.0, 3.0, 2.0) == 0.0                # local maximum
    assert slopefit(0.0, 0.1, 5.0) == pytest.approx(0.2, rel=1e-14)   # limited by 2 (c - l)
    assert slopefit(0.0, 4.9, 5.0) == pytest.approx(0.2, rel=1e-13)   # limited by 2 (r - c)


def test_linear_and_constant_fields():
    nx, ny, q = 12, 10, 5
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    rng = np.random.default_rng(2)
    ox, oz = rng.uniform(-1, 1, q), rng.uniform(-1, 1, q)
    b, c = 0.25, -0.5
    phi = np.repeat((3.0 + b * i + c * j)[:, :, None], q, axis=2)
    f = limited_flux(phi, ox, oz, 0.5, 0.25)
    np.testing.assert_allclose(f[2:-2, 2:-2], np.broadcast_to(ox / 0.5 * b + oz / 0.25 * c, (nx - 4, ny - 4, q)),
                               rtol=1e-13, atol=1e-13)
    assert np.array_equal(limited_flux(np.full((7, 7, 3), 2.5), ox[:3], oz[:3], 0.1, 0.1), np.zeros((7, 7, 3)))


def test_abi_argument_errors():
    """Checked on the host before any CUDA call (no device memory is touched)."""
    lib = _lib.load()
    fake = C.c_void_p(4096)
    other = C.c_void_p(1 << 40)
    assert lib.titus_limited_flux(-1, 8, 4, 0.1, 0.1, fake, fake, fake, other, None) == 1
    assert lib.titus_limited_flux(8, 8, 0, 0.1, 0.1, fake, fake, fake, other, None) == 1
    assert lib.titus_limited_flux(8, 8, 4, 0.0, 0.1, fake, fake, fake, other, None) == 1
    assert lib.titus_limited_flux(8, 8, 4, 0.1, 0.1, None, fake, fake, other, None) == 1
    assert lib.titus_limited_flux(8, 8, 4, 0.1, 0.1, fake, fake, fake, fake, None) == 1   # phi == flux
    assert "overlap" in _lib.last_error()
    assert lib.titus_limited_flux(4, 8, 4, 0.1, 0.1, fake, fake, fake, other, None) == 0  # no interior cell


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(37, 29, 16), (203, 198, 16), (5, 5, 3), (64, 70, 1), (9, 300, 24)])
def test_gpu_bit_exact(shape):
    import torch

    from titus_b200.flux import limited_flux_device

    phi, ox, oz, f0 = _case(3, shape)
    dev = torch.device("cuda", 0)
    d_phi = torch.from_numpy(phi).to(dev)
    d_flux = torch.from_numpy(f0).to(dev)
    limited_flux_device(d_phi, d_flux, torch.from_numpy(ox).to(dev), torch.from_numpy(oz).to(dev), 0.013, 0.021)
    torch.cuda.synchronize()
    assert np.array_equal(d_flux.cpu().numpy(), limited_flux(phi, ox, oz, 0.013, 0.021, f0))


@pytest.mark.gpu
def test_gpu_solveflux_host_arrays_with_solver_ordinates():
    from oracle.settings import Settings as OSettings
    from oracle.solver import SolverCSD as OSolver
    from titus_b200.flux import solveFlux

    sv = OSolver(OSettings(41, 41, 8, "csdPhantom", nPN=5))
    sv.setup_directions()
    nx, ny, q = sv.settings.NCellsX, sv.settings.NCellsY, sv.qReduced.shape[0]
    rng = np.random.default_rng(4)
    phi = np.abs(rng.standard_normal((nx, ny, q)))
    flux = np.zeros_like(phi)
    solveFlux(sv, phi, flux)
    assert np.array_equal(flux, sv.flux_limited(phi))


@pytest.mark.gpu
def test_gpu_rejects_bad_tensors():
    import torch

    from titus_b200.flux import limited_flux_device

    dev = torch.device("cuda", 0)
    phi = torch.zeros((8, 8, 4), dtype=torch.float64, device=dev)
    o = torch.zeros(4, dtype=torch.float64, device=dev)
    with pytest.raises(TypeError):
        limited_flux_device(phi.transpose(0, 1), torch.zeros_like(phi), o, o, 0.1, 0.1)
    with pytest.raises(ValueError):
        limited_flux_device(phi, torch.zeros((8, 8, 3), dtype=torch.float64, device=dev), o, o, 0.1, 0.1)
    with pytest.raises(_lib.TitusError, match="overlap"):
        limited_flux_device(phi, phi, o, o, 0.1, 0.1)
