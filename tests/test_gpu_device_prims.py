"""Device<GPU> primitives through the C ABI (ves3d_dev_*) against numpy in FP64: axpy,
AlgebraicDot, Transpose, Reduce (the reference's smooth surface integral) and gemm in
column-major BLAS semantics, including transposed operands and padded leading dimensions."""
import ctypes

import numpy as np
import pytest

from ves3d_b200 import _lib

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def test_axpy_and_dot():
    L = _lib.lib()
    rng = np.random.default_rng(1)
    x, y = rng.standard_normal((2, 100003))
    dx, dy = dev(x), dev(y)
    out = dev(np.zeros_like(x))
    assert L.ves3d_dev_axpy(-0.75, dx.data_ptr(), dy.data_ptr(), x.size, out.data_ptr(), None) == 0
    assert np.abs(out.cpu().numpy() - (-0.75 * x + y)).max() < 1e-15
    assert L.ves3d_dev_axpy(2.0, dx.data_ptr(), dy.data_ptr(), x.size, dy.data_ptr(), None) == 0  # in place
    assert np.abs(dy.cpu().numpy() - (2.0 * x + y)).max() < 1e-14
    r = ctypes.c_double(0)
    assert L.ves3d_dev_algebraic_dot(dx.data_ptr(), dx.data_ptr(), x.size, ctypes.byref(r), None) == 0
    assert abs(r.value / (x @ x) - 1) < 1e-13


@pytest.mark.parametrize("h,w", [(1, 1), (7, 45), (64, 32), (300, 129)])
def test_transpose(h, w):
    a = np.random.default_rng(h * w).standard_normal((h, w))
    da = dev(a)
    out = dev(np.zeros(h * w))
    assert _lib.lib().ves3d_dev_transpose(da.data_ptr(), h, w, out.data_ptr(), None) == 0
    assert np.array_equal(out.cpu().numpy().reshape(w, h), a.T)


def test_reduce():
    rng = np.random.default_rng(2)
    ns, dim, stride = 5, 3, 544
    x = rng.standard_normal((ns, dim, stride))
    w = rng.random((ns, stride))
    qw = rng.random(stride)
    out = dev(np.zeros(ns * dim))
    L = _lib.lib()
    assert L.ves3d_dev_reduce(dev(x).data_ptr(), dim, dev(w).data_ptr(), dev(qw).data_ptr(), stride, ns,
                              out.data_ptr(), None) == 0
    ref = np.einsum("sdi,si,i->sd", x, w, qw).reshape(-1)
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-12 * np.abs(ref).max()
    area = dev(np.zeros(ns))
    assert L.ves3d_dev_reduce(None, 0, dev(w).data_ptr(), dev(qw).data_ptr(), stride, ns, area.data_ptr(), None) == 0
    assert np.abs(area.cpu().numpy() - (w * qw).sum(1)).max() < 1e-12 * (w * qw).sum(1).max()


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_gemm_column_major(ta, tb):
    rng = np.random.default_rng(3)
    m, n, k = 37, 29, 41
    lda, ldb, ldc = (m if ta == "N" else k) + 3, (k if tb == "N" else n) + 2, m + 5
    A = rng.standard_normal((k if ta == "N" else m, lda)).T  # column-major [lda][cols] storage
    B = rng.standard_normal((n if tb == "N" else k, ldb)).T
    C = rng.standard_normal((n, ldc)).T
    opA = (A[:m, :k] if ta == "N" else A[:k, :m].T)
    opB = (B[:k, :n] if tb == "N" else B[:n, :k].T)
    ref = 1.5 * opA @ opB - 0.5 * C[:m, :n]
    dA, dB, dC = dev(A.T.reshape(-1)), dev(B.T.reshape(-1)), dev(C.T.reshape(-1))
    assert _lib.lib().ves3d_dev_gemm(ta.encode(), tb.encode(), m, n, k, 1.5, dA.data_ptr(), lda, dB.data_ptr(), ldb,
                                     -0.5, dC.data_ptr(), ldc, None) == 0
    got = dC.cpu().numpy().reshape(n, ldc).T
    assert np.abs(got[:m, :n] - ref).max() < 1e-12 * np.abs(ref).max()
    assert np.array_equal(got[m:, :], C[m:, :])  # rows beyond m untouched
