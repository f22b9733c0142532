"""The C ABI library loads and exports every symbol that include/titus.h declares."""
import os
import re

import pytest

from titus_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "titus.h")).read()
    return sorted(set(re.findall(r"\b(titus_[a-z0-9_]+)\s*\(", txt)))


def test_header_matches_binding():
    names = {n for n, _, _ in _lib.SIGNATURES}
    assert set(declared_symbols()) == names


def test_library_exports():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libtitus.so not built (run titus_b200.build)")
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.titus_max_rank() >= 20
    assert lib.titus_version().startswith(b"titus-b200")


def test_invalid_problem_is_rejected_without_gpu():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libtitus.so not built")
    import ctypes as C
    lib = _lib.load()
    p = _lib.Problem()
    p.nx = 2  # too small: rejected by validation before any CUDA call
    h = C.c_void_p()
    rc = lib.titus_create(C.byref(p), C.byref(h))
    assert rc == 1
    assert "nx" in _lib.last_error()


def _problem_with(field, index, value):
    """A small valid problem (host arrays) with one entry set to `value`."""
    from titus_b200 import Settings, SolverCSD
    sv = SolverCSD(Settings(12, 12, 4, "csdWaterBeam", nPN=3))
    p, keep = sv.problem_struct()
    arr = getattr(p, field)
    arr[index] = value
    return p, keep


@pytest.mark.parametrize("field,index", [("density", 5), ("stopping", 3), ("sigma", 2), ("bc_space", 0),
                                         ("m_reduced", 7), ("omega", 4), ("e_trafo", 1)])
@pytest.mark.parametrize("value", [float("nan"), float("inf")])
def test_non_finite_inputs_are_rejected_without_gpu(field, index, value):
    """titus_create validates every float input before touching the device."""
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libtitus.so not built")
    import ctypes as C
    lib = _lib.load()
    p, keep = _problem_with(field, index, value)
    h = C.c_void_p()
    rc = lib.titus_create(C.byref(p), C.byref(h))
    assert rc == 1
    err = _lib.last_error()
    assert ("not finite" in err or "density must be > 0" in err) and field.split("_")[0] in err, err


def test_invalid_3d_extension_is_rejected_without_gpu():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libtitus.so not built")
    import ctypes as C
    lib = _lib.load()
    p = _lib.Problem()
    e = _lib.Problem3D()
    e.nz, e.dz = 2, 0.1   # too few z layers: rejected before any CUDA call
    h = C.c_void_p()
    assert lib.titus_create_3d(C.byref(p), C.byref(e), C.byref(h)) == _lib.TITUS_ERR_ARG
    assert "nz" in _lib.last_error()
    e.nz, e.dz = 5, float("nan")
    assert lib.titus_create_3d(C.byref(p), C.byref(e), C.byref(h)) == _lib.TITUS_ERR_ARG
    assert lib.titus_create_3d(C.byref(p), None, C.byref(h)) == _lib.TITUS_ERR_ARG
