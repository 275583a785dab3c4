"""CPU oracle (test infrastructure only): the FP64 StokesVelocity composition used as
the parity reference. Only tests/, bench.py's cpu_baseline leg and
__graft_entry__.smoke() may import it, and only as the checker.

Composition (the non-FMM form of the reference's operator):
    u = SHC2Grid(Grid2SHC(f) . SLMatrix)                 self, p_up = 2p by default
                                                         (src/StokesVelocity.cc:164-473)
      + sum over points of OTHER vesicles of the Stokeslet with density f * area * qw
                                                         (StokesAlltoAll - DirectStokesKernel,
                                                          src/InterfacialVelocity.cc:1261-1291)
with area = |X_theta x X_phi| at order p (src/StokesVelocity.cc:252-273) and
qw = LegendreWeights(p) (src/SphericalHarmonics.cc:558-570).

The direct sums run in oracle/direct.c (compiled to oracle/_build/liboracle_direct.so by
oracle/build.py); the SH algebra is oracle/sh.py.
"""
import ctypes
import os

import numpy as np

from . import sh

HERE = os.path.dirname(os.path.abspath(__file__))
DIRECT_SO = os.path.join(HERE, "_build", "liboracle_direct.so")

_direct = None
_dp = ctypes.POINTER(ctypes.c_double)
_lp = ctypes.POINTER(ctypes.c_long)


def build_direct(force=False):
    """Compile oracle/direct.c with gcc -O3 -fopenmp (no CUDA)."""
    import subprocess
    if os.path.exists(DIRECT_SO) and not force and os.path.getmtime(DIRECT_SO) >= os.path.getmtime(os.path.join(HERE, "direct.c")):
        return DIRECT_SO
    os.makedirs(os.path.dirname(DIRECT_SO), exist_ok=True)
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.check_call([cc, "-O3", "-fopenmp", "-fPIC", "-shared", "-o", DIRECT_SO,
                           os.path.join(HERE, "direct.c"), "-lm"])
    return DIRECT_SO


def direct_lib():
    global _direct
    if _direct is None:
        build_direct()
        _direct = ctypes.CDLL(DIRECT_SO)
        for n in ("oracle_alltoall", "oracle_direct_stokes", "oracle_far", "oracle_direct_stokes_dl",
                  "oracle_far_dl"):
            getattr(_direct, n).restype = None
    return _direct


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def alltoall(src_pm, den_pm):
    src_pm = np.ascontiguousarray(src_pm, np.float64)
    den_pm = np.ascontiguousarray(den_pm, np.float64)
    pot = np.empty_like(src_pm)
    direct_lib().oracle_alltoall(_p(src_pm), _p(den_pm), ctypes.c_long(src_pm.size // 3), _p(pot))
    return pot


def direct_stokes(src_stride, trg_stride, n_surfs, head, tail, qw, trg, src, den):
    pot = np.zeros(3 * n_surfs * trg_stride)
    c = ctypes.c_int
    direct_lib().oracle_direct_stokes(c(src_stride), c(trg_stride), c(n_surfs), c(head), c(tail),
                                      _p(np.ascontiguousarray(qw, np.float64)), _p(np.ascontiguousarray(trg, np.float64)),
                                      _p(np.ascontiguousarray(src, np.float64)), _p(np.ascontiguousarray(den, np.float64)), _p(pot))
    return pot


def far(X, D, pt_off, trg_idx=None):
    """Far field at targets (all points, or the global point indices trg_idx).
    Returns [n_trg][3] point-major."""
    X = np.ascontiguousarray(X, np.float64)
    D = np.ascontiguousarray(D, np.float64)
    pt_off = np.ascontiguousarray(pt_off, np.int64)
    nves = pt_off.size - 1
    if trg_idx is None:
        n_trg = int(pt_off[-1])
        tp = None
    else:
        trg_idx = np.ascontiguousarray(trg_idx, np.int64)
        n_trg = trg_idx.size
        tp = trg_idx.ctypes.data_as(_lp)
    out = np.empty(3 * n_trg)
    direct_lib().oracle_far(_p(X), _p(D), ctypes.c_long(nves), pt_off.ctypes.data_as(_lp), tp,
                            ctypes.c_long(n_trg), _p(out))
    return out.reshape(n_trg, 3)


def uniform_offsets(nves, p):
    return np.arange(nves + 1, dtype=np.int64) * sh.ngrid(p)


def far_density(X, f, p):
    """den = f * area * qw on the order-p grid, AxisMajor like f."""
    ng = sh.ngrid(p)
    area = sh.area_element(X, p).reshape(-1, 1, ng)
    qw = sh.smooth_weights_grid(p).reshape(1, 1, ng)
    return (np.asarray(f, np.float64).reshape(-1, 3, ng) * area * qw).reshape(-1)


def far_velocity(X, f, p, trg_idx=None):
    """Far part in the AxisMajor layout of X (all targets), or [n][3] at trg_idx."""
    ng = sh.ngrid(p)
    nves = np.asarray(X).size // (3 * ng)
    D = far_density(X, f, p)
    out = far(X, D, uniform_offsets(nves, p), trg_idx)
    if trg_idx is not None:
        return out
    return out.reshape(nves, ng, 3).transpose(0, 2, 1).reshape(-1)


def stokes_velocity_sl(X, f, p, p_up=None, SL=None):
    """Full FP64 single-layer velocity at the surface grid points, AxisMajor."""
    if p_up is None:
        p_up = 2 * p
    if SL is None:
        SL = sh.stokes_singular_matrix(X, p, p_up)
    return sh.self_apply(SL, f, p) + far_velocity(X, f, p)


def direct_stokes_dl(src_stride, trg_stride, n_surfs, head, tail, qw, trg, src, norm, den):
    """DirectStokesDoubleLayerKernel: per-surface double layer, qw None for no weights."""
    pot = np.zeros(3 * n_surfs * trg_stride)
    c = ctypes.c_int
    direct_lib().oracle_direct_stokes_dl(c(src_stride), c(trg_stride), c(n_surfs), c(head), c(tail),
                                         None if qw is None else _p(np.ascontiguousarray(qw, np.float64)),
                                         _p(np.ascontiguousarray(trg, np.float64)),
                                         _p(np.ascontiguousarray(src, np.float64)),
                                         _p(np.ascontiguousarray(norm, np.float64)),
                                         _p(np.ascontiguousarray(den, np.float64)), _p(pot))
    return pot


def unit_normal(X, p):
    """(X_theta x X_phi) / |X_theta x X_phi| on the order-p grid, AxisMajor like X: the
    outward normal (src/StokesVelocity.cc:245-275)."""
    ng = sh.ngrid(p)
    S = sh.grid2shc(X, p, p)
    _, Xt, Xp = sh.shc2grid(S, p, p, grads=True)
    n = np.cross(Xt.reshape(-1, 3, ng), Xp.reshape(-1, 3, ng), axis=1)
    return (n / np.sqrt((n * n).sum(axis=1))[:, None, :]).reshape(-1)


def far_dl(X, nrm, D, pt_off):
    """Far double layer at every point over the points of the other vesicles: positions,
    unit normals and weighted densities as per-vesicle AxisMajor blocks at offsets pt_off.
    Returns [N][3] point-major."""
    pt_off = np.ascontiguousarray(pt_off, np.int64)
    out = np.empty(3 * int(pt_off[-1]))
    direct_lib().oracle_far_dl(_p(np.ascontiguousarray(X, np.float64)), _p(np.ascontiguousarray(nrm, np.float64)),
                               _p(np.ascontiguousarray(D, np.float64)), ctypes.c_long(pt_off.size - 1),
                               pt_off.ctypes.data_as(_lp), _p(out))
    return out.reshape(-1, 3)


def far_dl_velocity(X, g, p):
    """Far double layer at every point, AxisMajor: the points of the other vesicles with unit
    normals and densities g * area * qw (the single layer's composition)."""
    ng = sh.ngrid(p)
    nves = np.asarray(X).size // (3 * ng)
    out = far_dl(X, unit_normal(X, p), far_density(X, g, p), uniform_offsets(nves, p))
    return out.reshape(nves, ng, 3).transpose(0, 2, 1).reshape(-1)


def stokes_velocity_dl(X, g, p, p_up=None, DL=None):
    """Full FP64 double-layer velocity at the surface grid points, AxisMajor: the self part
    by the DL matrix (src/StokesVelocity.cc:418-436) plus the far double layer."""
    if p_up is None:
        p_up = 2 * p
    if DL is None:
        DL = sh.stokes_singular_matrix(X, p, p_up, single=False)
    return sh.self_apply(DL, g, p) + far_dl_velocity(X, g, p)


def target_velocity(X, f, p, T, g=None):
    """Velocity at off-surface targets T ([M][3], point-major, as SetTrgCoord,
    src/StokesVelocity.cc:146-161) by the smooth quadrature over every surface point: the
    single layer of f * area * qw (DirectStokesKernel over all points as one surface) plus,
    with g, the double layer of g * area * qw (DirectStokesDoubleLayerKernel). No
    near-singular correction: accurate away from the surfaces. Returns [M][3]."""
    ng = sh.ngrid(p)
    nv = np.asarray(X).size // (3 * ng)
    N = nv * ng
    T = np.asarray(T, np.float64).reshape(-1, 3)
    M = T.shape[0]

    def whole(A):
        return np.ascontiguousarray(np.asarray(A).reshape(nv, 3, ng).transpose(1, 0, 2).reshape(-1))

    Tw = np.ascontiguousarray(T.T.reshape(-1))
    u = direct_stokes(N, M, 1, 0, M, np.ones(N), Tw, whole(X), whole(far_density(X, f, p)))
    if g is not None:
        u = u + direct_stokes_dl(N, M, 1, 0, M, None, Tw, whole(X), whole(unit_normal(X, p)),
                                 whole(far_density(X, g, p)))
    return u.reshape(3, M).T.reshape(-1)


def stokes_velocity_poly(X, f, orders, g=None):
    """FP64 velocity of a polydisperse suspension (per-vesicle AxisMajor blocks concatenated;
    each vesicle's self part at its own order, p_up = 2p). With g, the double layer of g as
    well: each vesicle's DL matrix at its own order and the far double layer over the points
    of the other vesicles (SetDensityDL, src/StokesVelocity.cc:107-142, 418-436)."""
    X = np.asarray(X, np.float64)
    f = np.asarray(f, np.float64)
    orders = np.asarray(orders)
    ng = np.array([sh.ngrid(int(p)) for p in orders])
    off = np.concatenate([[0], np.cumsum(ng)]).astype(np.int64)
    D = np.empty_like(f)
    vel = np.empty_like(f)
    if g is not None:
        g = np.asarray(g, np.float64)
        Dg = np.empty_like(g)
        nrm = np.empty_like(g)
    for v, p in enumerate(orders):
        p = int(p)
        a, b = 3 * off[v], 3 * off[v + 1]
        D[a:b] = far_density(X[a:b], f[a:b], p)
        SL = sh.stokes_singular_matrix(X[a:b], p, 2 * p)
        vel[a:b] = sh.self_apply(SL, f[a:b], p)
        if g is not None:
            DL = sh.stokes_singular_matrix(X[a:b], p, 2 * p, single=False)
            vel[a:b] += sh.self_apply(DL, g[a:b], p)
            Dg[a:b] = far_density(X[a:b], g[a:b], p)
            nrm[a:b] = unit_normal(X[a:b], p)
    farv = far(X, D, off)
    if g is not None:
        farv = farv + far_dl(X, nrm, Dg, off)
    for v in range(orders.size):
        a = off[v]
        n = ng[v]
        vel[3 * a:3 * (a + n)] += farv[a:a + n].T.reshape(-1)
    return vel
