"""Double layer and viscosity contrast of a polydisperse suspension on the GPU
(ves3d_svp_set_density_dl, ves3d_svp_set_viscosity_contrast) against the oracle: the
evaluation at 1e-12 (FP64) and 1e-6 (mixed; the far double layer stays FP64), the captured
evaluation bitwise equal to the eager one, and implicit solves under a per-vesicle contrast
whose true residual through the oracle's polydisperse operator meets the tolerance."""
import numpy as np
import pytest

from oracle import stokes
from oracle import surface as su
from tests.helpers import rel_err, small_suspension
from ves3d_b200 import workloads
from ves3d_b200.stokes_velocity import PolydisperseStokesVelocity, StokesVelocity

pytestmark = pytest.mark.gpu
DT, KAPPA = 0.01, 0.05


@pytest.fixture(scope="module")
def poly_case():
    X, f, orders = workloads.polydisperse(10, orders=(4, 6, 8, 12), radius=(0.7, 1.3), volume_fraction=0.05,
                                          seed=77)
    g = np.random.default_rng(78).standard_normal(X.size)
    return X, f, g, orders


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_poly_double_layer_vs_oracle(poly_case, prec, tol):
    X, f, g, orders = poly_case
    ref = stokes.stokes_velocity_poly(X, f, orders, g=g)
    ref_sl = stokes.stokes_velocity_poly(X, f, orders)
    with PolydisperseStokesVelocity(prec) as sv:
        sv.SetSrcCoord(X, orders)
        sv.SetDensitySL(f)
        sv.SetDensityDL(g)
        vel = sv()
        sv.SetDensityDL(None)
        vel_sl = sv()
    assert rel_err(vel, ref) < tol
    assert rel_err(vel_sl, ref_sl) < tol


def test_poly_double_layer_graph_matches_eager(poly_case):
    X, f, g, orders = poly_case
    rng = np.random.default_rng(79)
    with PolydisperseStokesVelocity("fp64") as sv:
        sv.SetSrcCoord(X, orders)
        sv.SetDensitySL(f)
        sv.SetDensityDL(g)
        sv.capture_eval()
        f2 = rng.standard_normal(X.size)
        g2 = rng.standard_normal(X.size)
        sv.SetDensitySL(f2)
        sv.SetDensityDL(g2)
        vg = sv.launch_eval_graph()
        ve = sv()
    assert np.array_equal(vg, ve)
    assert rel_err(ve, stokes.stokes_velocity_poly(X, f2, orders, g=g2)) < 1e-12


def test_poly_double_layer_single_order_is_uniform():
    p = 8
    X, f = small_suspension(2, p, 81)
    g = np.random.default_rng(82).standard_normal(X.size)
    with StokesVelocity(p) as a:
        a.SetSrcCoord(X)
        a.SetDensitySL(f)
        a.SetDensityDL(g)
        u = a()
    with PolydisperseStokesVelocity() as b:
        b.SetSrcCoord(X, np.full(X.size // (3 * 2 * p * (p + 1)), p))
        b.SetDensitySL(f)
        b.SetDensityDL(g)
        w = b()
    assert rel_err(w, u) < 1e-14


@pytest.fixture(scope="module")
def contrast_case():
    X, _, orders = workloads.polydisperse(6, orders=(6, 8), radius=(0.8, 1.2), volume_fraction=0.08, seed=91)
    assert len(set(orders.tolist())) == 2
    lam = np.array([3.0, 0.2, 1.0, 5.0, 0.5, 2.0])[:orders.size]
    step = su.PolyImplicitStep(X, orders, KAPPA, DT, 1.0, viscosity_contrast=lam)
    b = step.to_coef(step.rhs())
    return X, orders, lam, step, b


@pytest.mark.parametrize("prec,scheme", [("fp64", "none"), ("fp64", "self_block"), ("mixed", "self_block")])
def test_poly_contrast_solve_true_residual(contrast_case, prec, scheme):
    X, orders, lam, step, b = contrast_case
    with PolydisperseStokesVelocity(prec) as sv:
        sv.SetSrcCoord(X, orders)
        sv.set_implicit_params(DT, KAPPA, 1.0)
        sv.set_viscosity_contrast(lam)
        sv.set_precond(scheme)
        x, it, relres, code = sv.implicit_solve(tol=1e-9, max_iter=3000)
    assert code == 100, (prec, scheme, it, relres)
    r = b - step.matvec_sh(step.to_coef(x))
    assert np.linalg.norm(r) / np.linalg.norm(b) < 3e-9, (prec, scheme)


def test_poly_contrast_single_order_is_the_uniform_step():
    P = 8
    X, _ = small_suspension(2, P, 53, spacing=2.7)
    nv = X.size // (3 * 2 * P * (P + 1))
    lam = np.linspace(0.3, 3.0, nv)
    with StokesVelocity(P) as a:
        a.SetSrcCoord(X)
        a.set_implicit_params(DT, KAPPA, 1.0)
        a.set_viscosity_contrast(lam)
        xa, ia, ra, ca = a.implicit_solve(tol=1e-10, max_iter=600)
    with PolydisperseStokesVelocity("fp64") as b:
        b.SetSrcCoord(X, np.full(nv, P))
        b.set_implicit_params(DT, KAPPA, 1.0)
        b.set_viscosity_contrast(lam)
        xb, ib, rb, cb = b.implicit_solve(tol=1e-10, max_iter=600)
    assert ca == cb == 100
    assert rel_err(xb[:X.size], xa[:X.size]) < 1e-8
