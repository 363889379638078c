"""CPU oracle of the learned CG warm start's network (test infrastructure only).

A float64 numpy restatement of the network in csrc/warmstart.cu, used by the
tests to check the CUDA forward pass and gradients.  The network has no
counterpart in the reference: ImmersedBodies.jl starts cg! from the previous
F~b (src/coupling.jl:194-202); the warm start only changes that initial guess.

Layer l: out[b, co, n] = bias[co] + sum_{ci, k} W[co, ci, k] x[b, ci, n + k - K//2]
(zero padding), tanh after every layer but the last.  Inputs are normalised
per channel, (x - in_mean) / in_std.  With e the last layer's output minus the
normalised target (t - out_mean) / out_std, the loss over the S sequences of n
points is (sum e^2 + sum E^2) / (S n), E the running sum of e along the points
divided by sqrt(n).
Parameters: one flat vector, per layer W [Co][Ci][K] then b [Co].
"""
from __future__ import annotations

import numpy as np


def layer_shapes(cin: int, width: int, kernel: int, layers: int, cout: int):
    return [((cout if l + 1 == layers else width), (cin if l == 0 else width), kernel) for l in range(layers)]


def num_params(cin, width, kernel, layers, cout) -> int:
    return sum(co * ci * k + co for co, ci, k in layer_shapes(cin, width, kernel, layers, cout))


def unpack(params: np.ndarray, shapes):
    out, o = [], 0
    for co, ci, k in shapes:
        W = params[o:o + co * ci * k].reshape(co, ci, k)
        o += co * ci * k
        b = params[o:o + co]
        o += co
        out.append((W, b))
    return out


def _pad(x, h):
    return np.pad(x, ((0, 0), (0, 0), (h, h)))


def forward(params, shapes, norm, x):
    """Normalised outputs and every layer's activation (a[0] the normalised input)."""
    in_mean, in_std = norm[0], norm[1]
    a = [(np.asarray(x, np.float64) - in_mean[None, :, None]) / in_std[None, :, None]]
    layers = unpack(np.asarray(params, np.float64), shapes)
    for l, (W, b) in enumerate(layers):
        K = W.shape[2]
        h = K // 2
        xp = _pad(a[-1], h)
        N = a[-1].shape[2]
        out = np.broadcast_to(b[None, :, None], (a[-1].shape[0], W.shape[0], N)).copy()
        for k in range(K):
            out += np.einsum("oc,bcn->bon", W[:, :, k], xp[:, :, k:k + N])
        a.append(np.tanh(out) if l + 1 < len(layers) else out)
    return a[-1], a


def predict(params, shapes, norm, x):
    """Prediction in solver units: out_mean + out_std * y."""
    y, _ = forward(params, shapes, norm, x)
    return norm[2][None, :, None] + norm[3][None, :, None] * y


def loss_grad(params, shapes, norm, x, t):
    """The loss on normalised targets and its gradient (flat vector)."""
    y, a = forward(params, shapes, norm, x)
    tn = (np.asarray(t, np.float64) - norm[2][None, :, None]) / norm[3][None, :, None]
    e = y - tn
    N = e.shape[2]
    E = np.cumsum(e, axis=2) / np.sqrt(N)
    loss = float((np.sum(e ** 2) + np.sum(E ** 2)) / e.size)
    gE = 2.0 * E / e.size / np.sqrt(N)
    d = 2.0 * e / e.size + np.cumsum(gE[:, :, ::-1], axis=2)[:, :, ::-1]
    layers = unpack(np.asarray(params, np.float64), shapes)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, b = layers[l]
        K = W.shape[2]
        h = K // 2
        N = d.shape[2]
        if l + 1 < len(layers):
            d = d * (1.0 - a[l + 1] ** 2)
        xp = _pad(a[l], h)
        dW = np.stack([np.einsum("bon,bcn->oc", d, xp[:, :, k:k + N]) for k in range(K)], axis=2)
        db = d.sum(axis=(0, 2))
        grads[l] = (dW, db)
        if l > 0:
            dxp = np.zeros_like(xp)
            for k in range(K):
                dxp[:, :, k:k + N] += np.einsum("oc,bon->bcn", W[:, :, k], d)
            d = dxp[:, :, h:h + N]
    return loss, np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
