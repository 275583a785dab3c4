"""The implicit step of a polydisperse suspension (vesicles of different SH orders, forces
at each vesicle's own order, one single layer over all points) against the CPU oracle's
PolyImplicitStep: every solve is checked by its true residual through the oracle's Galerkin
operator, FP64 throughout."""
import numpy as np
import pytest

from oracle import surface as su
from tests.helpers import rel_err, small_suspension
from ves3d_b200 import workloads
from ves3d_b200.stokes_velocity import PolydisperseStokesVelocity, StokesVelocity

pytestmark = pytest.mark.gpu
DT, KAPPA = 0.01, 0.05


@pytest.fixture(scope="module")
def case():
    X, _, orders = workloads.polydisperse(6, orders=(6, 8), radius=(0.8, 1.2), volume_fraction=0.08, seed=91)
    assert len(set(orders.tolist())) == 2
    step = su.PolyImplicitStep(X, orders, KAPPA, DT, 0.0, excess_density=1.0, gravity=(0.0, 0.0, -1.0))
    b = step.to_coef(step.rhs())
    return X, orders, step, b


def true_relres(step, b, x):
    r = b - step.matvec_sh(step.to_coef(x))
    return np.linalg.norm(r) / np.linalg.norm(b)


def mean_vertical_velocity(x, orders):
    k, acc, n = 0, 0.0, 0
    for p in orders:
        ng = 2 * int(p) * (int(p) + 1)
        acc += x[k + 2 * ng:k + 3 * ng].sum()
        n += ng
        k += 3 * ng
    return acc / n


@pytest.mark.parametrize("prec,scheme", [("fp64", "none"), ("fp64", "self_block"), ("mixed", "self_block"),
                                         ("mixed", "diag_spectral")])
def test_poly_implicit_solve_true_residual(case, prec, scheme):
    X, orders, step, b = case
    with PolydisperseStokesVelocity(prec) as sv:
        sv.SetSrcCoord(X, orders)
        sv.set_implicit_params(DT, KAPPA, 0.0)
        sv.set_gravity(1.0, (0.0, 0.0, -1.0))
        sv.set_precond(scheme)
        x, it, relres, code = sv.implicit_solve(tol=1e-9, max_iter=3000)
        stats = sv.solver_stats()
    assert code == 100, (prec, scheme, it, relres)
    assert relres < 1e-9
    assert true_relres(step, b, x) < 3e-9, (prec, scheme)
    assert mean_vertical_velocity(x, orders) < 0  # the suspension sinks
    if prec == "mixed":
        assert stats["outer"] >= 2


def test_poly_solution_matches_oracle_solve(case):
    X, orders, step, b = case
    xo, co, io, ro = step.solve(tol=1e-10, max_iter=600)
    assert co == 100
    with PolydisperseStokesVelocity("fp64") as sv:
        sv.SetSrcCoord(X, orders)
        sv.set_implicit_params(DT, KAPPA, 0.0)
        sv.set_gravity(1.0, (0.0, 0.0, -1.0))
        sv.set_precond("self_block")
        x, it, relres, code = sv.implicit_solve(tol=1e-10, max_iter=600)
        # a converged solution as the guess: nothing left to do
        x2, it2, relres2, code2 = sv.implicit_solve(x0=x, tol=1e-9, max_iter=600)
    assert code == 100 and code2 == 100 and it2 <= 1
    nu = X.size
    assert rel_err(x[:nu], xo[:nu]) < 1e-7


def test_poly_single_order_is_the_uniform_step():
    """With one order, the polydisperse implicit step is the uniform one."""
    P = 8
    X, _ = small_suspension(2, P, 53, spacing=2.7)
    with StokesVelocity(P) as a:
        a.SetSrcCoord(X)
        a.set_implicit_params(DT, KAPPA, 1.0)
        a.set_gravity(0.5, (0.0, 0.0, -1.0))
        xa, ia, ra, ca = a.implicit_solve(tol=1e-10, max_iter=600)
    with PolydisperseStokesVelocity("fp64") as b:
        b.SetSrcCoord(X, np.full(X.size // (3 * 2 * P * (P + 1)), P))
        b.set_implicit_params(DT, KAPPA, 1.0)
        b.set_gravity(0.5, (0.0, 0.0, -1.0))
        xb, ib, rb, cb = b.implicit_solve(tol=1e-10, max_iter=600)
    assert ca == cb == 100
    assert rel_err(xb[:X.size], xa[:X.size]) < 1e-8


def test_poly_combination_of_guesses(case):
    """The residual-minimising combination over the polydisperse operator: a converged
    solution among the candidates gets weight ~1 and the combination keeps its residual;
    a non-finite candidate gets weight 0; two earlier solutions of a moving suspension
    (whose span holds the linear extrapolation in time) start the next solve closer than
    the last one alone."""
    X, orders, step, b = case
    with PolydisperseStokesVelocity("fp64") as sv:
        sv.SetSrcCoord(X, orders)
        sv.set_implicit_params(DT, KAPPA, 0.0)
        sv.set_gravity(1.0, (0.0, 0.0, -1.0))
        sv.set_precond("self_block")
        x, it, relres, code = sv.implicit_solve(tol=1e-10, max_iter=600)
        junk = np.random.default_rng(3).standard_normal(x.size)
        bad = np.full(x.size, np.nan)
        x0, w, rr = sv.implicit_combine([junk, x, bad])
        assert abs(w[1] - 1.0) < 1e-6 and w[2] == 0.0 and abs(w[0]) < 1e-6
        assert rr[-1] < 1e-9 and not np.isfinite(rr[2])
        assert true_relres(step, b, x0) < 3e-9
        # three steps: the combination of the two previous solutions against the last one
        Xk, sols = X.copy(), []
        for k in range(3):
            sv.SetSrcCoord(Xk, orders)
            if k < 2:
                xk, _, _, ck = sv.implicit_solve(x0=sols[-1] if sols else None, tol=1e-10, max_iter=600)
                assert ck == 100
                sols.append(xk)
                Xk = Xk + DT * xk[:X.size]
        x0, w, rr = sv.implicit_combine([sols[-1], sols[-2]])
        assert rr[-1] < 0.5 * rr[0], (w, rr)
        xn, itn, rn, cn = sv.implicit_solve(x0=x0, tol=1e-10, max_iter=600)
        assert cn == 100
        stepn = su.PolyImplicitStep(Xk, orders, KAPPA, DT, 0.0, excess_density=1.0, gravity=(0.0, 0.0, -1.0))
        bn = stepn.to_coef(stepn.rhs())
        assert true_relres(stepn, bn, xn) < 3e-10
