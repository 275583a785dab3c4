"""Test infrastructure only: ctypes loader for oracle/_ref/libves3d_ref.so, the
reference's own CPU code built by oracle/ref/Makefile. Only tests/, bench.py's
reference / cpu_baseline arm and __graft_entry__.smoke() may use it, and only as
the checker or the timed CPU baseline, never as the product path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libves3d_ref.so")
NAIVE_LIB_PATH = os.path.join(HERE, "_ref", "libves3d_ref_naive.so")

_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_L = ctypes.c_long


def available():
    return os.path.exists(LIB_PATH)


def _load(path):
    # include/ves3d_common.h:79 reads VES3D_DIR at static-initialisation time;
    # nothing on this path opens files relative to it.
    os.environ.setdefault("VES3D_DIR", HERE)
    L = ctypes.CDLL(path)
    for name in ("ref_grid2shc", "ref_shc2grid", "ref_shc2pole", "ref_rotate_all",
                 "ref_legendre_nodes", "ref_legendre_weights", "ref_singular_weights",
                 "ref_singular_matrices", "ref_alltoall", "ref_direct_stokes", "ref_direct_stokes_dl",
                 "ref_area_weights", "ref_self_apply", "ref_far_sl",
                 "ref_stokes_velocity_sl", "ref_set_threads"):
        getattr(L, name).restype = ctypes.c_int
    return L


def naive_singular_matrices(X, p0, p1):
    """SL self matrices from the reference built with plain-loop GEMMs."""
    L = _load(NAIVE_LIB_PATH)
    ngrid = 2 * p0 * (p0 + 1)
    nves = X.size // (3 * ngrid)
    n = 3 * p0 * (p0 + 2)
    SL = np.empty(nves * n * n)
    L.ref_singular_matrices(_p(np.ascontiguousarray(X, np.float64)), _L(nves), _L(p0), _L(p1), _p(SL), None)
    return SL


def lib():
    global _lib
    if _lib is None:
        _lib = _load(LIB_PATH)
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def set_threads(n):
    return lib().ref_set_threads(ctypes.c_int(n))


def grid2shc(X, p0, p1):
    nfun = X.size // (2 * p0 * (p0 + 1))
    S = np.empty(nfun * p1 * (p1 + 2))
    lib().ref_grid2shc(_p(np.ascontiguousarray(X, np.float64)), _L(nfun), _L(p0), _L(p1), _p(S))
    return S


def shc2grid(S, p0, p1, grads=False):
    nfun = S.size // (p0 * (p0 + 2))
    n = nfun * 2 * p1 * (p1 + 1)
    X = np.empty(n)
    Xt = np.empty(n) if grads else None
    Xp = np.empty(n) if grads else None
    lib().ref_shc2grid(_p(np.ascontiguousarray(S, np.float64)), _L(nfun), _L(p0), _L(p1), _p(X), _p(Xt), _p(Xp))
    return (X, Xt, Xp) if grads else X


def shc2pole(S, p0):
    nfun = S.size // (p0 * (p0 + 2))
    P = np.empty(2 * nfun)
    lib().ref_shc2pole(_p(np.ascontiguousarray(S, np.float64)), _L(nfun), _L(p0), _p(P))
    return P


def rotate_all(S, p0, dof):
    nves = S.size // (dof * p0 * (p0 + 2))
    out = np.empty(S.size * p0 * (p0 + 1))
    lib().ref_rotate_all(_p(np.ascontiguousarray(S, np.float64)), _L(nves), _L(p0), _L(dof), _p(out))
    return out


def legendre_nodes(p):
    o = np.empty(p + 1); lib().ref_legendre_nodes(_L(p), _p(o)); return o


def legendre_weights(p):
    o = np.empty(p + 1); lib().ref_legendre_weights(_L(p), _p(o)); return o


def singular_weights(p):
    o = np.empty(p + 1); lib().ref_singular_weights(_L(p), _p(o)); return o


def singular_matrices(X, p0, p1, sl=True, dl=False):
    ngrid = 2 * p0 * (p0 + 1)
    nves = X.size // (3 * ngrid)
    n = 3 * p0 * (p0 + 2)
    SL = np.empty(nves * n * n) if sl else None
    DL = np.empty(nves * n * n) if dl else None
    lib().ref_singular_matrices(_p(np.ascontiguousarray(X, np.float64)), _L(nves), _L(p0), _L(p1), _p(SL), _p(DL))
    return SL, DL


def alltoall(src, den):
    np_ = src.size // 3
    pot = np.empty(3 * np_)
    lib().ref_alltoall(_p(np.ascontiguousarray(src, np.float64)), _p(np.ascontiguousarray(den, np.float64)), _L(np_), _p(pot))
    return pot


def direct_stokes(src_stride, trg_stride, n_surfs, head, tail, qw, trg, src, den):
    pot = np.zeros(3 * n_surfs * trg_stride)
    c = ctypes.c_int
    lib().ref_direct_stokes(c(src_stride), c(trg_stride), c(n_surfs), c(head), c(tail), _p(qw), _p(trg), _p(src), _p(den), _p(pot))
    return pot


def direct_stokes_dl(src_stride, trg_stride, n_surfs, head, tail, qw, trg, src, norm, den):
    """DirectStokesDoubleLayerKernel (double); qw None for the unweighted form."""
    pot = np.zeros(3 * n_surfs * trg_stride)
    c = ctypes.c_int
    lib().ref_direct_stokes_dl(c(src_stride), c(trg_stride), c(n_surfs), c(head), c(tail), _p(qw), _p(trg), _p(src),
                               _p(norm), _p(den), _p(pot))
    return pot


def area_weights(X, p):
    ngrid = 2 * p * (p + 1)
    nves = X.size // (3 * ngrid)
    area = np.empty(nves * ngrid)
    qw = np.empty(ngrid)
    lib().ref_area_weights(_p(np.ascontiguousarray(X, np.float64)), _L(nves), _L(p), _p(area), _p(qw))
    return area, qw


def self_apply(SL, f, p):
    ngrid = 2 * p * (p + 1)
    nves = f.size // (3 * ngrid)
    vel = np.empty(f.size)
    lib().ref_self_apply(_p(SL), _p(np.ascontiguousarray(f, np.float64)), _L(nves), _L(p), _p(vel))
    return vel


def far_sl(X, f, p):
    ngrid = 2 * p * (p + 1)
    nves = X.size // (3 * ngrid)
    vel = np.empty(X.size)
    t = ctypes.c_double(0)
    lib().ref_far_sl(_p(np.ascontiguousarray(X, np.float64)), _p(np.ascontiguousarray(f, np.float64)), _L(nves), _L(p), _p(vel), ctypes.byref(t))
    return vel, t.value


def stokes_velocity_sl(X, f, p, p_up):
    ngrid = 2 * p * (p + 1)
    nves = X.size // (3 * ngrid)
    vel = np.empty(X.size)
    t = np.zeros(3)
    lib().ref_stokes_velocity_sl(_p(np.ascontiguousarray(X, np.float64)), _p(np.ascontiguousarray(f, np.float64)), _L(nves), _L(p), _L(p_up), _p(vel), _p(t))
    return vel, t
