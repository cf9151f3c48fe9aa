"""The surrogate's CPU oracle pinned on its own: its analytic gradients equal central finite
differences of its loss (float64, no BF16 rounding), its BF16 rounding is ties-to-even, and its
Adam step is the published update (Kingma & Ba 2015, Algorithm 1)."""
import numpy as np
import pytest

from oracle import surrogate_oracle as S


def _params(seed, scale=0.2, inputs=7):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-scale, scale, S.param_count())
    W1 = p[: S.WIDTH * S.IN].reshape(S.WIDTH, S.IN)
    W1[:, inputs:] = 0.0
    return p


@pytest.mark.parametrize("seed", [0, 1])
def test_gradients_equal_finite_differences(seed):
    rng = np.random.default_rng(10 + seed)
    x = rng.uniform(0, 1, (16, 7))
    y = rng.normal(size=16)
    p = _params(seed)
    g, loss = S.gradients(p, x, y, exact=True)
    idx = np.concatenate([rng.choice(S.WIDTH * 7, 6, replace=False)] +  # W1 (inside the used columns)
                         [np.arange(S.param_count())[-1:]] +            # b5
                         [rng.choice(S.param_count() - S.WIDTH * S.IN, 24, replace=False) + S.WIDTH * S.IN])
    idx = [int(i) if i >= S.WIDTH * S.IN or (i % S.IN) < 7 else int(i) for i in idx]

    def loss_at(q):
        out = S.forward(q, x, exact=True)
        return float(((out - y) ** 2).mean())

    h = 1e-6
    for i in idx:
        if i < S.WIDTH * S.IN and i % S.IN >= 7:
            continue
        q1, q2 = p.copy(), p.copy()
        q1[i] += h
        q2[i] -= h
        fd = (loss_at(q1) - loss_at(q2)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
    assert loss == pytest.approx(float(((S.forward(p, x, exact=True) - y) ** 2).sum()))


def test_bf16_rounding_is_ties_to_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e38, 1e-40], dtype=np.float32)
    got = S.bf16(vals)
    # 1 + 2^-8 is half way between 1 and 1 + 2^-7: to the even 1; 1 + 3 * 2^-8 to the even 1 + 2^-6
    want = np.array([1.0, 1.0, 1.0 + 4 * 2 ** -8, 1.0, -2.5], dtype=np.float32)
    assert np.array_equal(got[:5], want)
    assert np.all(got.view(np.uint32) & 0xFFFF == 0)


def test_device_rounding_gradients_stay_close_to_exact():
    """The BF16 rounding points move the gradient by a few per mille of its norm, not more."""
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, (256, 7)).astype(np.float32)
    y = rng.normal(size=256).astype(np.float32)
    p = _params(3).astype(np.float32)
    g32, _ = S.gradients(p, x, y)
    g64, _ = S.gradients(p, x, y, exact=True)
    assert np.linalg.norm(g32 - g64) <= 0.02 * np.linalg.norm(g64)


def test_adam_step():
    rng = np.random.default_rng(4)
    p = _params(4).astype(np.float32)
    g = rng.normal(size=p.size).astype(np.float32)
    m1, m2 = np.zeros_like(p), np.zeros_like(p)
    q, a, b = S.adam(p, m1, m2, g, np.float32(1e-3), 1, 7)
    used = np.ones(p.size, dtype=bool)
    used[: S.WIDTH * S.IN] = (np.arange(S.WIDTH * S.IN) % S.IN) < 7
    # the first step moves every used parameter by lr * sign(g) (where |g| is well above eps)
    big = used & (np.abs(g) > 1e-4)
    assert np.allclose(q[big], p[big] - 1e-3 * np.sign(g[big]), rtol=0, atol=2e-7)
    assert np.array_equal(q[~used], p[~used])
