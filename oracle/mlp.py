"""CPU oracle (test infrastructure only): the multilayer perceptron of the learned initial
guess, its loss gradient and one Adam step, in numpy FP64. Only tests/ may use it, as the
checker of the library's BF16 training and inference kernels.

The learned guess has no counterpart in the reference (which starts each implicit solve
from the previous step, InterfacialVelocity::AssembleInitial,
src/InterfacialVelocity.cc:874-919), so this oracle restates published algorithms only:
  forward / backward      reverse-mode differentiation of x -> [Linear -> ReLU]* -> Linear
                          under the mean squared error (Rumelhart, Hinton & Williams 1986)
  optimiser               Adam (Kingma & Ba 2015, Algorithm 1; beta1 0.9, beta2 0.999,
                          eps 1e-8 added to sqrt(v_hat))
With bf16=True the oracle rounds exactly the operands the GPU kernels round to BF16
(round to nearest even): the normalised input, the weights, the hidden activations and
the back-propagated error signals that enter the tensor-core products; everything else
(biases, pre-activations, bias gradients) stays unrounded. The remaining GPU/oracle
difference is then FP32 accumulation order only. With bf16=False it is plain FP64
backpropagation, checked against finite differences in the tests.

Parameter layout (flat): per layer W [in][out] (row-major) then b [out].
Normalisation: network input (x - in_shift) * in_scale; loss on the normalised target
(t - out_shift) * out_inv with out_inv = 1 / out_scale (0 where out_scale is 0); the
prediction is z * out_scale + out_shift.
"""
import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layer_dims(n_in, n_hidden, n_layers, n_out):
    return [(n_in if l == 0 else n_hidden, n_out if l == n_layers - 1 else n_hidden) for l in range(n_layers)]


def unpack(params, dims):
    out, off = [], 0
    for di, do in dims:
        W = params[off:off + di * do].reshape(di, do)
        off += di * do
        b = params[off:off + do]
        off += do
        out.append((W, b))
    assert off == params.size
    return out


def _scaling(n_in, n_out, scaling):
    in_shift, in_scale, out_shift, out_scale = scaling if scaling is not None else (None,) * 4
    in_shift = np.zeros(n_in) if in_shift is None else np.asarray(in_shift, np.float64)
    in_scale = np.ones(n_in) if in_scale is None else np.asarray(in_scale, np.float64)
    out_shift = np.zeros(n_out) if out_shift is None else np.asarray(out_shift, np.float64)
    out_scale = np.ones(n_out) if out_scale is None else np.asarray(out_scale, np.float64)
    out_inv = np.where(out_scale != 0, 1.0 / np.where(out_scale != 0, out_scale, 1.0), 0.0)
    return in_shift, in_scale, out_shift, out_scale, out_inv


def _forward(params, dims, X, scaling, rnd):
    n_in, n_out = dims[0][0], dims[-1][1]
    in_shift, in_scale, _, _, _ = _scaling(n_in, n_out, scaling)
    layers = unpack(np.asarray(params, np.float64), dims)
    a = rnd((np.asarray(X, np.float64) - in_shift) * in_scale)
    acts, zs = [a], []
    for l, (W, b) in enumerate(layers):
        z = acts[-1] @ rnd(W) + b
        zs.append(z)
        if l < len(layers) - 1:
            acts.append(rnd(np.maximum(z, 0.0)))
    return layers, acts, zs


def predict(params, dims, X, scaling=None, bf16_round=True):
    rnd = bf16 if bf16_round else (lambda v: v)
    n_in, n_out = dims[0][0], dims[-1][1]
    _, _, out_shift, out_scale, _ = _scaling(n_in, n_out, scaling)
    _, _, zs = _forward(params, dims, X, scaling, rnd)
    return zs[-1] * out_scale + out_shift


def loss_and_grad(params, dims, X, T, scaling=None, bf16_round=True):
    """Mean squared error over all batch x output entries (normalised space) and its
    gradient in the flat parameter layout."""
    rnd = bf16 if bf16_round else (lambda v: v)
    n_in, n_out = dims[0][0], dims[-1][1]
    _, _, out_shift, _, out_inv = _scaling(n_in, n_out, scaling)
    layers, acts, zs = _forward(params, dims, X, scaling, rnd)
    tn = (np.asarray(T, np.float64) - out_shift) * out_inv
    e = zs[-1] - tn
    loss = float(np.mean(e * e))
    d = 2.0 * e / e.size
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        d16 = rnd(d)
        gW = acts[l].T @ d16
        gb = d.sum(axis=0)
        grads[l] = (gW, gb)
        if l == 0:
            break
        dh = d16 @ rnd(W).T
        d = np.where(zs[l - 1] > 0, dh, 0.0)
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat


def adam_step(params, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (step counts from 1); returns (params, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
