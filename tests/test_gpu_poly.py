"""Polydisperse suspensions (vesicles of different SH orders in one evaluation) against
the FP64 oracle."""
import numpy as np
import pytest

from oracle import stokes
from tests.helpers import rel_err
from ves3d_b200 import workloads
from ves3d_b200.stokes_velocity import PolydisperseStokesVelocity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def poly_case():
    return workloads.polydisperse(10, orders=(4, 6, 8, 12), radius=(0.7, 1.3), volume_fraction=0.05, seed=77)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_polydisperse_vs_oracle(poly_case, prec, tol):
    X, f, orders = poly_case
    assert len(set(orders.tolist())) > 1
    ref = stokes.stokes_velocity_poly(X, f, orders)
    with PolydisperseStokesVelocity(prec) as sv:
        sv.SetSrcCoord(X, orders)
        sv.SetDensitySL(f)
        vel = sv()
    assert rel_err(vel, ref) < tol


def test_polydisperse_matches_uniform_operator():
    """With a single order the polydisperse driver is the uniform operator."""
    from tests.helpers import small_suspension
    from ves3d_b200.stokes_velocity import StokesVelocity
    X, f = small_suspension(2, 8, 51)
    with StokesVelocity(8) as a:
        a.SetSrcCoord(X)
        a.SetDensitySL(f)
        u = a()
    with PolydisperseStokesVelocity() as b:
        b.SetSrcCoord(X, np.full(8, 8))
        b.SetDensitySL(f)
        w = b()
    assert rel_err(w, u) < 1e-14


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_polydisperse_graph_matches_eager(poly_case, prec):
    """The captured polydisperse evaluation, relaunched on new densities, equals the eager
    evaluation bitwise (fixed-order reductions) and stays on the oracle."""
    X, f, orders = poly_case
    rng = np.random.default_rng(9)
    with PolydisperseStokesVelocity(prec) as sv:
        sv.SetSrcCoord(X, orders)
        sv.SetDensitySL(f)
        sv.capture_eval()
        for _ in range(2):
            g = rng.standard_normal(X.size)
            sv.SetDensitySL(g)
            vg = sv.launch_eval_graph()
            ve = sv()
            assert np.array_equal(vg, ve)
    assert rel_err(ve, stokes.stokes_velocity_poly(X, g, orders)) < (1e-12 if prec == "fp64" else 1e-6)
