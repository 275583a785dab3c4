"""Edge cases of the GPU path: empty and ragged inputs, non-finite inputs injected on the
host (the context must stay usable and report, never crash), degenerate all-to-all
calls. Reference behaviour: BiCGStab reports RelresIsNan (src/BiCGStab.cc:74-75,
include/BiCGStab.h:19-23); StokesAlltoAll skips coincident pairs."""
import ctypes

import numpy as np
import pytest

from oracle import sh, stokes
from tests.helpers import rel_err, small_suspension
from ves3d_b200 import _lib
from ves3d_b200.stokes_velocity import PolydisperseStokesVelocity, StokesVelocity

pytestmark = pytest.mark.gpu


def test_empty_suspension_is_rejected_and_context_survives():
    L = _lib.lib()
    with StokesVelocity(6) as sv:
        x = np.zeros(3)
        assert L.ves3d_sv_set_src_coord(sv._h, x.ctypes.data, 0, 0) == 1  # ERR_ARG
        X, f = small_suspension(1, 6, 5)
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        v = sv()
    SL = sh.stokes_singular_matrix(X, 6, 12)
    assert rel_err(v, sh.self_apply(SL, f, 6)) < 1e-12
    with PolydisperseStokesVelocity() as g:
        with pytest.raises(_lib.Ves3dError):
            g.SetSrcCoord(np.zeros(0), np.zeros(0, dtype=np.int32))


@pytest.mark.parametrize("nv,p,prec,tol", [(3, 6, "fp64", 1e-12), (5, 8, "fp64", 1e-12), (3, 6, "mixed", 1e-6),
                                           (7, 12, "mixed", 1e-6)])
def test_ragged_vesicle_counts(nv, p, prec, tol):
    """Vesicle and point counts that are not multiples of any tile, chunk or CTA size."""
    X, f = small_suspension(2, p, 90 + nv, spacing=2.6)
    ng = 2 * p * (p + 1)
    X, f = X[: nv * 3 * ng].copy(), f[: nv * 3 * ng].copy()
    with StokesVelocity(p, precision=prec) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        v = sv()
    ref = stokes.stokes_velocity_sl(X, f, p, 2 * p)
    assert rel_err(v, ref) < tol


def test_nan_density_propagates_and_context_recovers():
    X, f = small_suspension(2, 6, 31, spacing=2.8)
    bad = f.copy()
    bad[5] = np.nan
    with StokesVelocity(6) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(bad)
        v = sv()
        assert np.isnan(v).any()
        sv.SetDensitySL(f)
        v = sv()
    assert rel_err(v, stokes.stokes_velocity_sl(X, f, 6, 12)) < 1e-12


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_implicit_solve_reports_nan(prec):
    """Non-finite surfaces: the solve returns BiCGSReturn RelresIsNan (104) instead of
    iterating or faulting; good surfaces afterwards solve normally."""
    X, _ = small_suspension(2, 6, 32, spacing=2.8)
    bad = X.copy()
    bad[17] = np.nan
    with StokesVelocity(6, precision=prec) as sv:
        sv.set_implicit_params(0.01, 0.05, 1.0)
        sv.SetSrcCoord(bad)
        x, it, relres, code = sv.implicit_solve(tol=1e-8, max_iter=50)
        assert code == 104 and not np.isfinite(relres)
        sv.SetSrcCoord(X)
        x, it, relres, code = sv.implicit_solve(tol=1e-8, max_iter=600)
        assert code == 100 and relres < 1e-8


def test_alltoall_degenerate_sizes():
    L = _lib.lib()
    ctx = ctypes.c_void_p()
    src = np.array([0.3, -0.2, 1.0])
    den = np.array([1.0, 2.0, 3.0])
    pot = np.full(3, 7.0)
    L.ves3d_stokes_alltoall_f64(src.ctypes.data, den.ctypes.data, 1, pot.ctypes.data, ctypes.byref(ctx))
    assert np.all(pot == 0.0)  # a single point has no partner (its own pair is skipped)
    L.ves3d_stokes_alltoall_f64(src.ctypes.data, den.ctypes.data, 0, pot.ctypes.data, ctypes.byref(ctx))
    L.ves3d_interaction_free(ctypes.byref(ctx))
    # all points coincident: every pair is skipped
    src4 = np.tile(src, 4)
    den4 = np.random.default_rng(0).standard_normal(12)
    pot4 = np.empty(12)
    L.ves3d_stokes_alltoall_f64(src4.ctypes.data, den4.ctypes.data, 4, pot4.ctypes.data, ctypes.byref(ctx))
    L.ves3d_interaction_free(ctypes.byref(ctx))
    assert np.all(pot4 == 0.0)
