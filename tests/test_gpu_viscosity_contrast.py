"""GPU implicit step with a viscosity contrast (ves3d_sv_set_viscosity_contrast) against the
CPU oracle's contrast operator (oracle/surface.py ImplicitStep(viscosity_contrast=...)):
the operator at 1e-12 (FP64), the rigid-translation property, and solves whose true
residual through the oracle operator meets the tolerance."""
import numpy as np
import pytest

from oracle import surface as su
from tests.helpers import rel_err, small_suspension
from ves3d_b200.stokes_velocity import StokesVelocity

pytestmark = pytest.mark.gpu
TOL = 1e-12
DT, KAPPA, RATE = 0.01, 0.05, 1.0
LAM8 = np.array([3.0, 0.2, 1.0, 5.0, 0.5, 2.0, 1.0, 0.1])


def test_contrast_operator_matches_oracle():
    p = 8
    X, _ = small_suspension(2, p, 41, spacing=2.8)
    step = su.ImplicitStep(X, p, KAPPA, DT, RATE, viscosity_contrast=LAM8)
    z = np.random.default_rng(7).standard_normal(4 * step.nv * step.ng)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.set_implicit_params(DT, KAPPA, RATE)
        sv.set_viscosity_contrast(LAM8)
        y = sv.surface_op("implicit_matvec", z)
        rhs = sv.surface_op("implicit_rhs")
        sv.set_viscosity_contrast(1.0)  # a contrast of one is the plain operator
        y1 = sv.surface_op("implicit_matvec", z)
    assert rel_err(y, step.matvec(z)) < TOL
    assert rel_err(rhs, step.rhs()) < TOL  # the right-hand side does not see the contrast
    assert rel_err(y1, su.ImplicitStep(X, p, KAPPA, DT, RATE, SL=step.SL).matvec(z)) < TOL


def test_contrast_keeps_rigid_translations():
    """A constant velocity per vesicle with zero tension is a fixed point of the operator
    for any contrast (the oracle measures 3.5e-5 here, the double layer's quadrature error)."""
    p = 12
    X, _ = small_suspension(2, p, 3)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.set_implicit_params(DT, KAPPA, RATE)
        sv.set_viscosity_contrast(LAM8)
        ng = 2 * p * (p + 1)
        nv = X.size // (3 * ng)
        C = np.random.default_rng(1).standard_normal((nv, 3))
        z = np.concatenate([np.repeat(C[:, :, None], ng, axis=2).reshape(-1), np.zeros(nv * ng)])
        y = sv.surface_op("implicit_matvec", z)
    assert np.abs(y - z).max() < 1e-4 * np.abs(C).max()


@pytest.mark.parametrize("prec,scheme", [("fp64", "none"), ("fp64", "self_block"), ("mixed", "self_block"),
                                         ("mixed", "diag_spectral")])
def test_contrast_solves_reach_the_true_residual(prec, scheme):
    p = 8
    X, _ = small_suspension(2, p, 47, spacing=2.6)
    step = su.ImplicitStep(X, p, KAPPA, DT, RATE, viscosity_contrast=LAM8)
    b = step.to_coef(step.rhs())
    with StokesVelocity(p, precision=prec) as sv:
        sv.SetSrcCoord(X)
        sv.set_implicit_params(DT, KAPPA, RATE)
        sv.set_viscosity_contrast(LAM8)
        sv.set_precond(scheme)
        x, it, relres, code = sv.implicit_solve(tol=1e-9, max_iter=3000)
    assert code == 100, (it, relres)
    r = b - step.matvec_sh(step.to_coef(x))
    assert np.linalg.norm(r) / np.linalg.norm(b) < 3e-9
