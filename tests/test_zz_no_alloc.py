"""The all-to-all entry point that allocates nothing, checked against the one that does
and against the oracle's restatement of StokesAlltoAll. Its users are programs whose
device memory belongs to another allocator, which cannot let the library call
cudaMalloc; it stages data through one fixed device array instead. This file is
collected last on purpose."""
import ctypes

import numpy as np
import pytest

from tests.helpers import rel_err
from ves3d_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-12
MAX_POINTS = 524288  # VES3D_NOALLOC_MAX_POINTS in include/ves3d_b200.h


def _existing(src, den):
    pot = np.empty_like(src)
    ctx = ctypes.c_void_p()
    _lib.lib().ves3d_stokes_alltoall_f64(src.ctypes.data, den.ctypes.data, src.size // 3, pot.ctypes.data,
                                         ctypes.byref(ctx))
    _lib.lib().ves3d_interaction_free(ctypes.byref(ctx))
    assert np.isfinite(pot).all(), _lib.lib().ves3d_last_error()
    return pot


def _noalloc(src, den, stream=None):
    pot = np.full_like(src, np.nan)
    st = _lib.lib().ves3d_stokes_alltoall_noalloc_f64(src.ctypes.data, den.ctypes.data, src.size // 3,
                                                      pot.ctypes.data, stream)
    _lib.check(st, "ves3d_stokes_alltoall_noalloc_f64")
    return pot


def _case(rng, np_):
    src = rng.standard_normal(3 * np_) * 3.0
    den = rng.standard_normal(3 * np_)
    src[3:6] = src[0:3]  # one coincident pair
    return src, den


def test_noalloc_matches_allocating_entry_point_twice():
    rng = np.random.default_rng(2024)
    # two calls in a row; the second is smaller, so stale contents of the shared array
    # from the first call would show up if the entry point read past np
    for np_ in (3001, 1234):
        src, den = _case(rng, np_)
        got = _noalloc(src, den)
        ref = _existing(src, den)
        assert np.isfinite(got).all()
        assert rel_err(got, ref) < TOL


def test_noalloc_matches_oracle_on_a_created_stream():
    from oracle import stokes as ostokes
    import torch
    rng = np.random.default_rng(77)
    src, den = _case(rng, 2500)
    s = torch.cuda.Stream()
    got = _noalloc(src, den, ctypes.c_void_p(s.cuda_stream))
    ref = ostokes.alltoall(src, den)
    assert rel_err(got, ref) < TOL


def test_noalloc_empty_call_leaves_result_untouched():
    pot = np.full(6, 7.0)
    one = np.zeros(6)
    st = _lib.lib().ves3d_stokes_alltoall_noalloc_f64(one.ctypes.data, one.ctypes.data, 0, pot.ctypes.data, None)
    assert st == 0
    assert (pot == 7.0).all()


def test_noalloc_rejects_oversize_request():
    n = MAX_POINTS + 1
    buf = np.zeros(3 * n)
    pot = np.zeros(3 * n)
    st = _lib.lib().ves3d_stokes_alltoall_noalloc_f64(buf.ctypes.data, buf.ctypes.data, n, pot.ctypes.data, None)
    assert st == 1  # VES3D_ERR_ARG
    assert b"VES3D_NOALLOC_MAX_POINTS" in _lib.lib().ves3d_last_error()
    assert np.isnan(pot).all()  # errors fill the result with NaN, as the allocating call does
