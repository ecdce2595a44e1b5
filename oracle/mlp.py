"""numpy restatement of the warm-start network (TEST INFRASTRUCTURE ONLY).

The checker for the device kernels in magritte_b200/csrc/learned.cu: same
parameter layout, standardisation, tanh hidden layers, log-softmax loss with
per-level weights, and its gradient by backpropagation in float64.  The
network has no counterpart in the reference.
"""
import numpy as np

HIDDEN = 128


def layer_shapes(nin, nout):
    return [(HIDDEN, nin), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (nout, HIDDEN)]


def unpack(params, nin, nout):
    out, p = [], 0
    for (o, i) in layer_shapes(nin, nout):
        W = params[p:p + o * i].reshape(o, i)
        p += o * i
        b = params[p:p + o]
        p += o
        out.append((W, b))
    return out


def forward(params, mean, istd, X, nout):
    nin = X.shape[1]
    layers = unpack(params.astype(np.float64), nin, nout)
    a = (X.astype(np.float64) - mean) * istd
    acts = [a]
    for l, (W, b) in enumerate(layers):
        z = a @ W.T + b
        a = np.tanh(z) if l < len(layers) - 1 else z
        acts.append(a)
    return a, acts


def loss_and_grad(params, mean, istd, X, lte, tgt):
    """Summed loss over samples and d(loss)/d(params), float64."""
    nout = lte.shape[1]
    nin = X.shape[1]
    delta, acts = forward(params, mean, istd, X, nout)
    z = lte.astype(np.float64) + delta
    c = np.log(np.exp(z - z.max(1, keepdims=True)).sum(1, keepdims=True)) + z.max(1, keepdims=True)
    r = z - c - tgt
    w = np.where(tgt > np.log(1e-8), 1.0, np.where(tgt > np.log(1e-12), 0.1, 0.0))
    loss = float((w * r * r).sum())
    sm = np.exp(z - c)
    g = 2.0 * (w * r - sm * (w * r).sum(1, keepdims=True))
    layers = unpack(params.astype(np.float64), nin, nout)
    grads = []
    dA = g
    for l in range(len(layers) - 1, -1, -1):
        W, b = layers[l]
        if l < len(layers) - 1:
            dA = dA * (1.0 - acts[l + 1] ** 2)
        grads.append((dA.T @ acts[l], dA.sum(0)))
        dA = dA @ W
    grads = grads[::-1]
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
