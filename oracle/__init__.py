"""FP64 CPU oracle for the TITUS CSD energy step.

TEST INFRASTRUCTURE ONLY. This package is a plain numpy/scipy restatement of
the reference Julia solver (CSMMLab/TITUS, ``code/SolverCSD.jl`` and the files
it includes) evaluated at ``T = Float64``. It is the parity checker for the
CUDA path and the timed CPU baseline. Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it; the product package ``titus_b200`` never
does.

Every function cites the reference ``file:line`` it follows. Where the
reference is undefined (LAPACK's completion of numerically null singular
directions, the undefined name ``rmax`` in the rejection variants) the
restatement fixes one deterministic reading and says so in the docstring.

Third-party arithmetic that is not part of the reference tree and is restated
here from its published definition:

* FastGaussQuadrature.jl 0.5.0 ``gausslegendre`` -> ``numpy.polynomial.legendre.leggauss``.
* SphericalHarmonics.jl 0.1.19 ``computePlmx(x, lmax, norm=Unnormalized())`` ->
  associated Legendre functions without the Condon-Shortley phase
  (``oracle.quadrature.plm_unnormalized``), pinned by ``M diag(Omega_x) O = Ax``.
* Interpolations.jl 0.14.6 ``LinearInterpolation(...; extrapolation_bc=Throw())`` ->
  ``oracle.csd.linear_interp`` (piecewise linear, error outside the table).
* LAPACK ``gesdd`` / numpy ``qr`` -> ``numpy.linalg`` (same routines), plus the
  deterministic completion rule in ``oracle.linalg``.
"""

__all__ = ["pn", "quadrature", "csd", "settings", "stencils", "solver", "linalg", "flux"]
