"""The MIXED mode's tensor-core Gram run (tcgen05 kind::tf32, hi/lo split
operands, FP32 accumulation in TMEM) against an FP64 product, through the C
ABI test hook titus_debug_tc_gram.

The split keeps about 21 significant bits per product and the accumulation is
FP32, so the bound is relative to the sum of |products| of each entry:
|D - D64| <= 2e-6 * (|O_d A|^T |A|), elementwise.
"""
import numpy as np
import pytest

from titus_b200 import _lib

pytestmark = pytest.mark.gpu


def tc_gram(F, nw, nops):
    rows = F.shape[0]
    out = np.zeros((nops, nw, nw))
    F = np.ascontiguousarray(F, dtype=np.float64)
    _lib.check(_lib.load().titus_debug_tc_gram(_lib.as_dp(F), rows, nw, nops, _lib.as_dp(out)), "titus_debug_tc_gram")
    return out


@pytest.mark.parametrize("rows,nw,nops", [(16, 16, 4), (37, 20, 4), (1000, 32, 4), (513, 40, 4), (300, 80, 4),
                                          (64, 8, 1), (200, 48, 2)])
def test_tc_gram_matches_fp64(rows, nw, nops):
    rng = np.random.default_rng(rows + nw)
    F = rng.standard_normal((rows, (nops + 1) * nw)) * np.exp(rng.uniform(-3, 3, (nops + 1) * nw))
    got = tc_gram(F, nw, nops)
    A = F[:, :nw]
    for d in range(nops):
        O = F[:, (d + 1) * nw:(d + 2) * nw]
        want = O.T @ A
        scale = np.abs(O).T @ np.abs(A)
        err = np.abs(got[d] - want) / scale
        assert err.max() <= 2e-6, (d, err.max())


def test_tc_gram_rejects_bad_shapes():
    F = np.zeros((4, 5 * 81))
    with pytest.raises(_lib.TitusError):
        tc_gram(F, 81, 4)
    with pytest.raises(_lib.TitusError):
        tc_gram(np.zeros((4, 4 * 8)), 8, 3)
