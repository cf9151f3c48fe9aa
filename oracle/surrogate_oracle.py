"""Test infrastructure: an FP32 CPU restatement of the surrogate network (numpy), the checker of
libsurrogate.so's forward, gradient and training kernels. It rounds to BF16 exactly where the
device does (the products' operands and the stored activations) and accumulates the products in
float64 before rounding them to FP32 (the device accumulates in FP32 in its own order, so the two
agree to FP32 rounding of the sums, not bit for bit). tanh is exact here and an approximation on
the device (tanh.approx.f32, relative error below 2^-10.9); tests compare with tolerances.

The network (include/pacuda_surrogate.h): four hidden layers of 256 with
silu(z) = z (1 + tanh(z / 2)) / 2, one output, loss mean((out - y)^2) -- the sum over the batch
of (out - y)^2 is what `gradients` returns as the loss.
"""
from __future__ import annotations

import numpy as np

WIDTH, IN = 256, 64


def bf16(x):
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


class _Arith:
    """The device's arithmetic (FP32 values, BF16 rounding points) or, with exact=True, the same
    formulas in float64 without rounding (to check the gradients by finite differences)."""

    def __init__(self, exact=False):
        self.exact = exact
        self.t = np.float64 if exact else np.float32

    def r(self, x):  # a BF16 rounding point
        return np.asarray(x, dtype=np.float64) if self.exact else bf16(x)

    def c(self, x):  # a value kept in the working precision
        return np.asarray(x, dtype=self.t)

    def mm(self, a, b):
        return self.c(np.asarray(a, np.float64) @ np.asarray(b, np.float64))

    def silu(self, z):
        z = self.c(z)
        h = self.t(0.5)
        return self.c(h * z * (self.t(1) + np.tanh(h * z)))

    def silu_grad(self, z):
        z = self.c(z)
        s = self.t(0.5) + self.t(0.5) * np.tanh(self.t(0.5) * z)
        return self.c(s * (self.t(1) + z * (self.t(1) - s)))


def silu(z):
    return _Arith().silu(z)


def silu_grad(z):
    return _Arith().silu_grad(z)


def unpack(p):
    """The parameter vector as (W1 [256][64], b1, W2, b2, W3, b3, W4, b4, w5 [256], b5 [1])."""
    p = np.asarray(p)
    out, at = [], 0
    for shape in [(WIDTH, IN), (WIDTH,), (WIDTH, WIDTH), (WIDTH,), (WIDTH, WIDTH), (WIDTH,), (WIDTH, WIDTH), (WIDTH,),
                  (WIDTH,), (1,)]:
        n = int(np.prod(shape))
        out.append(p[at:at + n].reshape(shape))
        at += n
    assert at == p.size
    return out


def param_count():
    return WIDTH * IN + 3 * WIDTH * WIDTH + 5 * WIDTH + 1


def forward(params, x, keep=False, exact=False):
    A = _Arith(exact)
    W1, b1, W2, b2, W3, b3, W4, b4, w5, b5 = [A.c(q) for q in unpack(params)]
    n, inputs = x.shape
    X = np.zeros((n, IN), dtype=A.t)
    X[:, :inputs] = x
    X = A.r(X)
    h, zs, hs = X, [], [X]
    for W, b in ((W1, b1), (W2, b2), (W3, b3), (W4, b4)):
        z = A.c(A.mm(h, A.r(W).T) + b)
        zs.append(z)
        h = A.r(A.silu(z))
        hs.append(h)
    out = A.c(A.mm(hs[-1], w5) + b5[0])
    return (out, zs, hs) if keep else out


def gradients(params, x, y, exact=False):
    """(gradient vector in param order, loss = sum over the batch of (out - y)^2)."""
    A = _Arith(exact)
    W1, b1, W2, b2, W3, b3, W4, b4, w5, b5 = [A.c(q) for q in unpack(params)]
    out, zs, hs = forward(params, x, keep=True, exact=exact)
    n = x.shape[0]
    e = A.c(out - A.c(y))
    dout = A.c(A.t(2) * e / A.t(n))
    g_w5 = A.mm(hs[4].T, dout)
    g_b5 = A.c([np.asarray(dout, np.float64).sum()])
    dz = A.c(dout[:, None] * w5[None, :] * A.silu_grad(zs[3]))
    grads = {}
    Ws = [W1, W2, W3, W4]
    for l in range(3, -1, -1):
        grads[f"b{l}"] = A.c(np.asarray(dz, np.float64).sum(axis=0))
        dzb = A.r(dz)
        grads[f"W{l}"] = A.mm(dzb.T, hs[l])
        if l > 0:
            dh = A.mm(dzb, A.r(Ws[l]))
            dz = A.c(dh * A.silu_grad(A.r(zs[l - 1])))
    parts = [grads["W0"], grads["b0"], grads["W1"], grads["b1"], grads["W2"], grads["b2"], grads["W3"], grads["b3"],
             g_w5, g_b5]
    return A.c(np.concatenate([q.reshape(-1) for q in parts])), float((np.asarray(e, np.float64) ** 2).sum())


def adam(params, m1, m2, grad, lr, step, inputs):
    """One Adam step as the device takes it (beta1 0.9, beta2 0.999, eps 1e-8); the padding
    columns of W1 (features at or beyond `inputs`) are left alone."""
    a = np.float32(0.9) * m1 + np.float32(0.1) * grad
    b = np.float32(0.999) * m2 + np.float32(0.001) * grad * grad
    c1, c2 = np.float32(1.0 / (1.0 - 0.9 ** step)), np.float32(1.0 / (1.0 - 0.999 ** step))
    upd = lr * (a * c1) / (np.sqrt(b * c2) + np.float32(1e-8))
    mask = np.ones_like(params, dtype=bool)
    mask[:WIDTH * IN] = (np.arange(WIDTH * IN) % IN) < inputs
    p = np.where(mask, params - upd, params).astype(np.float32)
    return p, np.where(mask, a, m1).astype(np.float32), np.where(mask, b, m2).astype(np.float32)
