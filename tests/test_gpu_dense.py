"""Gauss-Jordan inverses of the coarse operators (tf_invert_dense), against numpy's LU inverse.

Tolerance: ||A X - I||_max <= 1e-12 * cond_1(A) per matrix (the backward error of partial
pivoting on these well-scaled matrices), and the zero-pivot step reported as LAPACK's getrf
reports it (info = k + 1).
"""
import ctypes

import numpy as np
import pytest

from tissueorigami_b200 import capi

pytestmark = pytest.mark.gpu


def _invert(a, cooperative):
    L = capi.load()
    a = np.array(a, dtype=np.float64, copy=True)
    count, n = a.shape[0], a.shape[1]
    cm = np.ascontiguousarray(np.transpose(a, (0, 2, 1)))  # column-major per matrix
    info = np.zeros(count, dtype=np.int32)
    rc = L.tf_invert_dense(0, n, count, int(cooperative), cm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           info.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    assert rc == capi.TF_OK
    return np.transpose(cm, (0, 2, 1)), info


def _coarse_like(rng, count, n):
    """Symmetric positive definite, diagonally graded matrices like P^T J P, permuted so that
    pivoting has to swap rows."""
    out = []
    for _ in range(count):
        b = rng.normal(size=(n, n))
        m = b @ b.T / n + np.diag(rng.uniform(0.5, 2.0, n))
        s = np.exp(rng.uniform(-2, 2, n))
        m = s[:, None] * m * s[None, :]
        p = rng.permutation(n)
        out.append(m[p])
    return np.stack(out)


@pytest.mark.parametrize("cooperative,n,count", [(False, 48, 5), (False, 300, 3), (True, 48, 1), (True, 1500, 1)])
def test_inverse_matches_lu(cooperative, n, count):
    rng = np.random.default_rng(n + count)
    a = _coarse_like(rng, count, n)
    x, info = _invert(a, cooperative)
    assert (info == 0).all()
    for t in range(count):
        cond = np.linalg.cond(a[t], 1)
        res = np.abs(a[t] @ x[t] - np.eye(n)).max()
        assert res <= 1e-12 * cond, (t, res, cond)
        ref = np.linalg.inv(a[t])
        assert np.abs(x[t] - ref).max() <= 1e-10 * cond * np.abs(ref).max()


@pytest.mark.parametrize("cooperative", [False, True])
def test_zero_pivot_reports_step(cooperative):
    n = 40
    rng = np.random.default_rng(7)
    a = _coarse_like(rng, 1, n)[0]
    a[:, 5] = 0.0  # column 5 stays zero through the elimination: step 5 finds no pivot
    x, info = _invert(a[None], cooperative)
    assert info[0] == 6
