"""The surrogate network's tensor-core kernels against the CPU oracle (oracle/surrogate_oracle.py):
the fused inference kernel's outputs, the gradient of every parameter (forward, backward and
weight-gradient products, the column sums of the epilogues), one Adam step, and a short training
run that fits a smooth function. Tolerances: the device rounds to BF16 at the same points as the
oracle but sums in its own order and uses tanh.approx, so values agree to a few BF16 ulps."""
import numpy as np
import pytest

from oracle import surrogate_oracle as O

pytestmark = pytest.mark.gpu

INPUTS = 12


def _params(seed, scale=1.0):
    """Weights of a trained-looking scale: uniform in +-scale * sqrt(6 / fan_in), small biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(O.param_count(), dtype=np.float32)
    parts = O.unpack(p)
    for k, q in enumerate(parts):
        fan = INPUTS if k == 0 else O.WIDTH
        if q.ndim == 2 or k == 8:
            q[...] = rng.uniform(-1, 1, q.shape) * scale * np.sqrt(6.0 / fan)
        else:
            q[...] = rng.uniform(-0.1, 0.1, q.shape)
    parts[0][:, INPUTS:] = 0.0
    return p


def _net(seed, batch=1024):
    from pacuda_b200 import surrogate as S

    n = S.Network(INPUTS, max_batch=batch, seed=seed)
    p = _params(seed)
    n.set_params(p)
    return n, p


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (n, INPUTS)).astype(np.float32)
    x[:, 5:] = 0.0
    x[np.arange(n), 5 + rng.integers(0, 7, n)] = 1.0  # a subprocess one-hot
    return x


def _close(got, want, rel):
    scale = np.sqrt(np.mean(want.astype(np.float64) ** 2)) + 1e-30
    return np.max(np.abs(got - want)) / scale, rel


@pytest.mark.parametrize("count", [128, 1000, 40000])
def test_forward_matches_oracle(count):
    import torch

    net, p = _net(1)
    x = _inputs(count, 2)
    out = net.forward(torch.tensor(x, device="cuda")).cpu().numpy()
    want = O.forward(p, x)
    err = np.abs(out - want) / (np.abs(want) + np.sqrt(np.mean(want ** 2)))
    assert net.error() == 0
    assert np.all(np.isfinite(out))
    assert np.max(err) < 2e-2, np.max(err)
    assert np.mean(err) < 2e-3, np.mean(err)


@pytest.mark.parametrize("batch", [256, 384, 1024])
def test_gradients_match_oracle(batch):
    import torch

    net, p = _net(3, batch=1024)
    x = _inputs(batch, 4)
    y = np.random.default_rng(5).normal(size=batch).astype(np.float32)
    g, loss = net.gradients(torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda"))
    g = g.cpu().numpy()
    want, want_loss = O.gradients(p, x, y)
    assert net.error() == 0
    assert float(loss.cpu()[0]) == pytest.approx(want_loss, rel=1e-2)
    parts_g, parts_w = O.unpack(g), O.unpack(want)
    names = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4", "w5", "b5"]
    for name, a, b in zip(names, parts_g, parts_w):
        a, b = a.astype(np.float64).ravel(), b.astype(np.float64).ravel()
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
        assert rel < 3e-2 and cos > 0.999, (name, rel, cos)
    # the padding columns of W1 get no gradient
    assert np.all(parts_g[0][:, 32:] == 0.0)


def test_adam_step_matches_oracle():
    import torch

    net, p = _net(6, batch=512)
    x = _inputs(512, 7)
    y = np.random.default_rng(8).normal(size=512).astype(np.float32)
    xt, yt = torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda")
    g, _ = net.gradients(xt, yt)
    net.train_step(xt, yt, 1e-3)
    got = net.params()
    want, _, _ = O.adam(p, np.zeros_like(p), np.zeros_like(p), g.cpu().numpy(), np.float32(1e-3), 1, INPUTS)
    assert net.error() == 0
    assert np.allclose(got, want, rtol=0, atol=2e-6)


def test_training_fits_a_smooth_function():
    """200 Adam steps on batches of 1024 points of a smooth function of five inputs plus a
    one-hot offset bring the loss down by more than 20x (a CPU-free check that the forward,
    backward and update kernels work together)."""
    import torch

    from pacuda_b200 import surrogate as S

    net = S.Network(INPUTS, max_batch=1024, seed=11)
    rng = np.random.default_rng(12)

    def target(x):
        return (np.sin(3 * x[:, 0]) + x[:, 1] * x[:, 2] - np.cos(2 * x[:, 3] + x[:, 4]) + 0.5 * np.argmax(x[:, 5:], axis=1)
                ).astype(np.float32)

    xs = _inputs(1024 * 8, 13)
    ys = target(xs)
    ys = (ys - ys.mean()) / ys.std()
    xt, yt = torch.tensor(xs, device="cuda"), torch.tensor(ys, device="cuda")
    loss = torch.zeros(1, device="cuda")
    losses = []
    for step in range(200):
        k = step % 8
        if step % 8 == 0:
            loss.zero_()
        net.train_step(xt[1024 * k:1024 * (k + 1)], yt[1024 * k:1024 * (k + 1)], 2e-3, loss)
        if step % 8 == 7:
            losses.append(float(loss.cpu()[0]) / (8 * 1024))
    assert net.error() == 0
    assert losses[-1] < losses[0] / 20, losses
    pred = net.forward(xt).cpu().numpy()
    assert np.mean((pred - ys) ** 2) < losses[0] / 20


def test_kernels_are_deterministic():
    """The same inputs give the same bits: the inference kernel's outputs, the gradient and loss
    of one batch computed twice, and two networks of one seed after the same 40 Adam steps (the
    kernels' sums run in fixed orders; no atomics in any value)."""
    import torch

    from pacuda_b200 import surrogate as S

    net, _ = _net(3, batch=4096)
    x = torch.tensor(_inputs(4096, 4), device="cuda")
    y = torch.tensor(np.random.default_rng(5).normal(size=4096).astype(np.float32), device="cuda")
    g1, l1 = net.gradients(x, y)
    g2, l2 = net.gradients(x, y)
    assert torch.equal(g1, g2) and torch.equal(l1, l2)
    xs = torch.tensor(_inputs(40000, 9), device="cuda")
    assert torch.equal(net.forward(xs), net.forward(xs))
    a, b = S.Network(INPUTS, max_batch=4096, seed=21), S.Network(INPUTS, max_batch=4096, seed=21)
    for step in range(40):
        for n in (a, b):
            n.train_step(x, y, 1e-3 * (1 + step % 3))
    assert a.error() == 0 and b.error() == 0
    assert np.array_equal(a.params().view(np.uint32), b.params().view(np.uint32))
