"""GPU tests of the learned initial guess: the BF16 MLP kernels against the CPU oracle
(oracle/mlp.py, which rounds the same operands to BF16), the feature/target maps, the
residual-minimising choice among candidate guesses, and the gain of a network trained on
solves of the method itself over the solve without it."""
import numpy as np
import pytest

from oracle import mlp as om
from tests.helpers import small_suspension
from ves3d_b200.learned_guess import MLP, LearnedGuess, generate_dataset, initial_guess
from ves3d_b200.stokes_velocity import StokesVelocity, ncoef, ngrid

pytestmark = pytest.mark.gpu


def _scaling(rng, n_in, n_out):
    return (rng.standard_normal(n_in).astype(np.float32), rng.uniform(0.5, 2, n_in).astype(np.float32),
            rng.standard_normal(n_out).astype(np.float32), rng.uniform(0.5, 2, n_out).astype(np.float32))


@pytest.mark.parametrize("shape", [(40, 72, 3, 24, 100), (130, 64, 2, 70, 67), (864, 256, 4, 1152, 256)])
def test_mlp_gradients_match_oracle(shape):
    n_in, n_hid, n_layers, n_out, B = shape
    rng = np.random.default_rng(sum(shape))
    net = MLP(n_in, n_hid, n_layers, n_out, seed=3)
    sc = _scaling(rng, n_in, n_out)
    net.set_scaling(*sc)
    X = rng.standard_normal((B, n_in)).astype(np.float32)
    T = rng.standard_normal((B, n_out)).astype(np.float32)
    w = net.get_params().astype(np.float64)
    loss, g = net.gradients(X, T)
    loss_o, g_o = om.loss_and_grad(w, net.dims, X, T, sc, bf16_round=True)
    assert abs(loss - loss_o) <= 1e-5 * loss_o
    off = 0
    for di, do in net.dims:
        for n in (di * do, do):
            a, b = g[off:off + n], g_o[off:off + n]
            assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b), (di, do, n)
            off += n
    # the prediction (denormalised); an activation whose FP32 sum lands on the other side
    # of a BF16 rounding boundary moves by one BF16 step (2^-8 relative), so deep networks
    # differ from the oracle by a few 1e-4
    Y = net.forward(X)
    Yo = om.predict(w, net.dims, X, sc, bf16_round=True)
    assert np.linalg.norm(Y - Yo) <= 1e-3 * np.linalg.norm(Yo)
    net.close()


def test_mlp_adam_step_matches_oracle():
    rng = np.random.default_rng(5)
    net = MLP(50, 64, 3, 30, seed=1)
    X = rng.standard_normal((64, 50)).astype(np.float32)
    T = rng.standard_normal((64, 30)).astype(np.float32)
    w0 = net.get_params().astype(np.float64)
    _, g = net.gradients(X, T)
    lr = 1e-3
    net.train_step(X, T, lr)
    w1 = net.get_params().astype(np.float64)
    w1o, _, _ = om.adam_step(w0, g.astype(np.float64), np.zeros_like(w0), np.zeros_like(w0), 1, lr)
    # Adam's first step is lr * sign(g) wherever |g| >> eps: compare in units of lr
    assert np.mean(np.abs(w1 - w1o)) < 1e-3 * lr
    assert np.max(np.abs(w1 - w1o)) < 0.05 * lr


def test_mlp_training_reduces_loss():
    rng = np.random.default_rng(7)
    A = rng.standard_normal((32, 16)) / np.sqrt(32)
    X = rng.standard_normal((2048, 32)).astype(np.float32)
    T = np.tanh(X @ A).astype(np.float32)
    net = MLP(32, 128, 3, 16, seed=2)
    l0 = net.gradients(X, T)[0]
    for k in range(600):
        idx = rng.integers(0, 2048, 256)
        net.train_step(X[idx], T[idx], 2e-3)
    l1 = net.gradients(X, T)[0]
    assert l1 < 0.05 * l0
    net.close()


def test_mlp_rejects_bad_arguments():
    from ves3d_b200._lib import Ves3dError
    with pytest.raises(Ves3dError):
        MLP(0, 8, 2, 4)
    net = MLP(4, 8, 2, 3)
    with pytest.raises(ValueError):
        net.set_params(np.zeros(3, np.float32))
    net.close()


P = 8
DT, KAPPA, RATE = 0.01, 0.05, 1.0


@pytest.fixture(scope="module")
def solved():
    X, _ = small_suspension(2, P, 61, spacing=2.6)
    sv = StokesVelocity(P)
    sv.SetSrcCoord(X)
    sv.set_implicit_params(DT, KAPPA, RATE)
    x, it, rr, code = sv.implicit_solve(tol=1e-10, max_iter=1000)
    assert code == 100
    yield X, sv, x, it
    sv.close()


def test_guess_targets_round_trip(solved):
    X, sv, x, _ = solved
    t = sv.guess_targets(x)
    assert t.shape == (sv.n_ves, 4 * ncoef(P))
    back = sv.guess_from_targets(t)
    # the solution lies in the band-limited space; only FP32 storage of the coefficients is lost
    assert np.linalg.norm(back - x) <= 1e-6 * np.linalg.norm(x)
    f = sv.guess_features()
    assert f.shape == (sv.n_ves, 3 * ncoef(P))
    assert np.all(f[:, ::ncoef(P)] == 0)  # degree 0 removed: translation invariant
    sv2 = StokesVelocity(P)
    sv2.SetSrcCoord(X + np.repeat(np.array([0.3, -1.0, 2.0]), 2 * P * (P + 1))[None].repeat(sv.n_ves, 0).reshape(-1))
    assert np.max(np.abs(sv2.guess_features() - f)) <= 1e-6 * np.max(np.abs(f))
    sv2.close()


def test_combine_picks_by_true_residual(solved):
    X, sv, x, _ = solved
    rng = np.random.default_rng(0)
    garbage = rng.standard_normal(x.size) * np.abs(x).max()
    near = x + 1e-3 * np.abs(x).max() * rng.standard_normal(x.size)
    x0, w, r = sv.implicit_combine([garbage, near])
    assert r[-1] <= min(r[:-1]) * (1 + 1e-9)
    assert abs(w[0]) < 1e-2 and abs(w[1] - 1) < 1e-2
    # the exact solution alone: weight 1 and the solve's own residual
    x0, w, r = sv.implicit_combine([x])
    assert abs(w[0] - 1) < 1e-6 and r[-1] < 1e-8
    # a non-finite candidate is dropped
    bad = np.full_like(x, np.nan)
    x0, w, r = sv.implicit_combine([bad, near])
    assert w[0] == 0 and np.all(np.isfinite(x0)) and r[-1] <= r[1] * (1 + 1e-9)


def test_learned_guess_saves_iterations(tmp_path):
    """Train on implicit solves of 12 seeded 8-vesicle suspensions (the method's own
    output), then solve a held-out suspension from zero and from the learned guess."""
    cfgs = [dict(nves_side=2, spacing=2.6, semi_axes=(1.0, 1.0, 0.6), deg=4, amp=0.05, seed=300 + s) for s in range(12)]
    F, T, _ = generate_dataset(cfgs, steps=2, p=P, dt=DT, kappa=KAPPA, shear_rate=RATE, tol=1e-8)
    g = LearnedGuess(P, DT, KAPPA, RATE, n_hidden=128, n_layers=3, seed=0)
    g.fit(F, T, epochs=300, batch=64, lr=2e-3)
    path = tmp_path / "guess.bin"
    g.save(path)
    g2 = LearnedGuess.load(path)
    np.testing.assert_array_equal(g2.predict(F[:5]), g.predict(F[:5]))
    X, _ = small_suspension(2, P, 999, spacing=2.6)
    sv = StokesVelocity(P)
    sv.SetSrcCoord(X)
    sv.set_implicit_params(DT, KAPPA, RATE)
    # with the self-block preconditioner convergence is smooth enough that a closer start
    # shows up as fewer iterations (unpreconditioned counts vary by +-15% with the start)
    sv.set_precond("self_block")
    _, it0, _, c0 = sv.implicit_solve(tol=1e-10, max_iter=2000)
    x0, info = initial_guess(sv, learned=g2)
    _, it1, _, c1 = sv.implicit_solve(x0=x0, tol=1e-10, max_iter=2000)
    assert c0 == 100 and c1 == 100
    # measured by the true residual: the learned start is far closer than the zero start
    # (relative residual 1), and the solve from it is shorter
    assert info["relres_combined"] < 0.1, info
    assert it1 < it0, (it0, it1, info)
    # a broken network: the fallback (previous solution) keeps the solve where it was
    g2.net.set_params(np.random.default_rng(1).standard_normal(g2.net.num_params()).astype(np.float32) * 10)
    xs, _, _, _ = sv.implicit_solve(tol=1e-10, max_iter=2000)
    x0b, infob = initial_guess(sv, learned=g2, previous=xs)
    assert abs(infob["weights"][0]) < 1e-3 and infob["relres_combined"] <= 1e-9
    sv.close()
    g.close()
    g2.close()
