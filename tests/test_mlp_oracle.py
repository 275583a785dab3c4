"""CPU checks of the MLP oracle (oracle/mlp.py) that the GPU training kernels are tested
against: FP64 backpropagation against central finite differences, BF16 rounding against
hand-computed cases, and the Adam step against its closed form on the first step."""
import numpy as np

from oracle import mlp as om


def _net(rng, dims):
    return np.concatenate([np.concatenate([rng.standard_normal(di * do) / np.sqrt(di), 0.1 * rng.standard_normal(do)])
                           for di, do in dims])


def test_bf16_rounding():
    one = 1.0
    ulp = 2.0 ** -7  # BF16 spacing at 1
    assert om.bf16(one) == one
    assert om.bf16(one + 0.25 * ulp) == one                    # below half: down
    assert om.bf16(one + 0.75 * ulp) == one + ulp               # above half: up
    assert om.bf16(one + 0.5 * ulp) == one                      # tie to even (mantissa 0)
    assert om.bf16(one + 1.5 * ulp) == one + 2 * ulp            # tie to even (mantissa 1 -> 2)
    assert om.bf16(-3.0) == -3.0
    x = np.random.default_rng(0).standard_normal(1000)
    r = om.bf16(x)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8 * (1 + 1e-12))


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    dims = om.layer_dims(7, 9, 3, 5)
    w = _net(rng, dims)
    X = rng.standard_normal((11, 7))
    T = rng.standard_normal((11, 5))
    scaling = (rng.standard_normal(7), rng.uniform(0.5, 2, 7), rng.standard_normal(5), rng.uniform(0.5, 2, 5))
    loss, g = om.loss_and_grad(w, dims, X, T, scaling, bf16_round=False)
    h = 1e-6
    fd = np.empty_like(w)
    for i in range(w.size):
        e = np.zeros_like(w)
        e[i] = h
        fd[i] = (om.loss_and_grad(w + e, dims, X, T, scaling, False)[0] -
                 om.loss_and_grad(w - e, dims, X, T, scaling, False)[0]) / (2 * h)
    assert np.max(np.abs(fd - g)) < 1e-7 * max(1.0, np.max(np.abs(g)))
    # the loss is the MSE of the normalised prediction
    pred = om.predict(w, dims, X, scaling, False)
    tn = (T - scaling[2]) / scaling[3]
    assert abs(loss - np.mean(((pred - scaling[2]) / scaling[3] - tn) ** 2)) < 1e-12


def test_adam_first_step():
    rng = np.random.default_rng(2)
    w = rng.standard_normal(50)
    g = rng.standard_normal(50)
    w1, m, v = om.adam_step(w, g, np.zeros(50), np.zeros(50), 1, 1e-3)
    # after one step m_hat = g, v_hat = g^2
    assert np.allclose(w1, w - 1e-3 * g / (np.abs(g) + 1e-8), rtol=0, atol=1e-15)
