"""CPU checks of the unweighting's restatement (oracle/unweight_oracle.py), which the GPU tests
use as the checker of the device kernels: the five-number phase-space map against RAMBO, the
jet cuts against the benchmark's, and two-stage unweighting on a toy with a known density."""
import math

import numpy as np
import pytest

from oracle import unweight_oracle as U
from pacuda_b200 import phase_space, unweight


def test_map_is_massless_and_conserves_momentum():
    u = U.uniforms(5, np.arange(4096, dtype=np.uint64))
    p, jac = U.phase_space(u, 13000.0)
    assert np.allclose(p[:, :, 0] ** 2 - (p[:, :, 1:] ** 2).sum(axis=2), 0.0, atol=1e-6 * 13000.0 ** 2 * 1e-6)
    assert np.allclose(p[:, :2].sum(axis=1), p[:, 2:].sum(axis=1), atol=1e-8 * 13000.0)
    assert np.all(p[:, 2:, 0] >= 0) and np.all(jac >= 0)


def test_map_volume_and_distributions_match_rambo():
    """The map's weight integrates to the massless three-body volume s / (256 pi^3), RAMBO's
    constant weight, and the weighted distributions of symmetric observables (every final
    parton's energy, every pair's invariant mass) equal RAMBO's flat ones."""
    sqrt_s, n = 1000.0, 1 << 18
    s = sqrt_s * sqrt_s
    vol = s / (256.0 * math.pi ** 3)
    u = U.uniforms(11, np.arange(n, dtype=np.uint64))
    p, jac = U.phase_space(u, sqrt_s)
    # the mean of J estimates the volume: within four standard errors (the map leaves out a
    # q-frame solid angle of 1.7e-6 and |eta1| > 5.5, far below that)
    assert abs(jac.mean() - vol) < 4 * jac.std() / math.sqrt(n) + 1e-4 * vol
    r = phase_space.rambo(5, n, 12, ecm=sqrt_s)

    def obs(q):  # point-major: [point][3] flattened
        e = q[:, 2:, 0].reshape(-1)
        m = []
        for i, j in ((2, 3), (2, 4), (3, 4)):
            k = q[:, i] + q[:, j]
            m.append(np.sqrt(np.maximum(0.0, k[:, 0] ** 2 - (k[:, 1:] ** 2).sum(axis=1))))
        return e, np.stack(m, axis=1).reshape(-1)

    for a, b in zip(obs(p), obs(r)):
        edges = np.linspace(0, max(a.max(), b.max()), 21)
        wa = np.repeat(jac, 3)
        ha, _ = np.histogram(a, edges, weights=wa)
        va, _ = np.histogram(a, edges, weights=wa ** 2)
        hb, _ = np.histogram(b, edges)
        hb = hb * vol
        vb = hb * vol
        chi2 = ((ha - hb) ** 2 / (va + vb + 1e-300))[hb > 0].sum()
        assert chi2 / 20 < 3.0, chi2


def test_four_parton_map_is_massless_and_conserves_momentum():
    u = U.uniforms(5, np.arange(4096, dtype=np.uint64), final_state=4)
    assert u.shape == (4096, 10)
    p, jac = U.momenta(u, 13000.0, final_state=4)
    assert p.shape == (4096, 6, 4)
    assert np.allclose(p[:, :, 0] ** 2 - (p[:, :, 1:] ** 2).sum(axis=2), 0.0, atol=1e-6 * 13000.0 ** 2 * 1e-6)
    assert np.allclose(p[:, :2].sum(axis=1), p[:, 2:].sum(axis=1), atol=1e-8 * 13000.0)
    assert np.all(p[:, 2:, 0] >= 0) and np.all(jac >= 0)


def test_four_parton_map_volume_and_distributions_match_rambo():
    """The 2 -> 4 map's weight, taken at flat invariants and angles (s_Q / s, s_R / s_Q,
    (1 + cos theta) / 2 uniform: the uniforms that give them, times the inverse transforms'
    derivatives), is the flat sequential-decay density s s_Q (1 - s_Q / s)(1 - s_R / s_Q) / (2048 pi^5)
    at every point, which integrates to the massless four-body volume s^2 / (24576 pi^5); and the
    map's momenta weighted by it follow RAMBO's flat distributions (every parton's energy, every
    pair's invariant mass)."""
    sqrt_s, n = 1000.0, 1 << 18
    s = sqrt_s * sqrt_s
    vol = s * s / (24576.0 * math.pi ** 5)
    v = np.random.default_rng(13).uniform(size=(n, 8))
    u = np.zeros((n, 10))
    dxdv = np.ones(n)
    for k in (0, 3):  # logistic invariants
        u[:, k] = (np.log(v[:, k] / (1.0 - v[:, k])) / U.MAP_L + 1.0) / 2.0
        dxdv /= 2.0 * U.MAP_L * v[:, k] * (1.0 - v[:, k])
    for k, e in ((1, U.MAP_E1), (4, U.MAP_E2), (6, U.MAP_E2)):  # tanh angles
        c = 2.0 * v[:, k] - 1.0
        u[:, k] = (np.arctanh(c) / e + 1.0) / 2.0
        dxdv /= e * (1.0 - c * c)
    for k in (2, 5, 7):
        u[:, k] = v[:, k]
    inside = ((u[:, :8] > 0) & (u[:, :8] < 1)).all(axis=1)  # all but the map's uncovered edges
    assert inside.mean() > 0.9999
    u, v, dxdv = u[inside], v[inside], dxdv[inside]
    p, jac = U.momenta(u, sqrt_s, final_state=4)
    flat = jac * dxdv
    sq = s * v[:, 0]
    want = s * sq * (1.0 - v[:, 0]) * (1.0 - v[:, 3]) / (2048.0 * math.pi ** 5)
    assert np.allclose(flat, want, rtol=1e-9, atol=0)
    assert abs(flat.mean() - vol) < 4 * flat.std() / math.sqrt(flat.size)
    r = phase_space.rambo(6, n, 14, ecm=sqrt_s)
    pairs = [(i, j) for i in range(2, 6) for j in range(i + 1, 6)]

    def obs(q):
        e = q[:, 2:, 0].reshape(-1)
        m = []
        for i, j in pairs:
            k = q[:, i] + q[:, j]
            m.append(np.sqrt(np.maximum(0.0, k[:, 0] ** 2 - (k[:, 1:] ** 2).sum(axis=1))))
        return (e, 4), (np.stack(m, axis=1).reshape(-1), len(pairs))

    for (a, na), (b, _) in zip(obs(p), obs(r)):
        edges = np.linspace(0, max(a.max(), b.max()), 21)
        wa = np.repeat(flat, na) * n / flat.size
        ha, _ = np.histogram(a, edges, weights=wa)
        va, _ = np.histogram(a, edges, weights=wa ** 2)
        hb, _ = np.histogram(b, edges)
        hb = hb * vol
        vb = hb * vol
        chi2 = ((ha - hb) ** 2 / (va + vb + 1e-300))[hb > 0].sum()
        assert chi2 / 20 < 3.0, chi2


def test_four_parton_features_and_cuts():
    u = U.uniforms(21, np.arange(5000, dtype=np.uint64), final_state=4)
    f = U.features(u, 2, 4, final_state=4)
    assert f.shape == (5000, 12) and np.array_equal(f[:, :8], u[:, :8].astype(np.float32))
    assert np.all(f[:, 8 + 2] == 1.0) and np.all(f[:, [8, 9, 11]] == 0.0)
    p, _ = U.momenta(u, 13000.0, final_state=4)
    ok = U.passes(p, 20.0, 5.0, 0.4)
    assert 0.05 < ok.mean() < 1.0
    assert np.array_equal(ok, phase_space.passes_cuts(p))


def test_cuts_agree_with_the_benchmark_cuts():
    u = U.uniforms(3, np.arange(20000, dtype=np.uint64))
    p, _ = U.phase_space(u, 13000.0)
    ok = U.passes(p)
    assert 0.2 < ok.mean() < 1.0
    assert np.array_equal(ok, phase_space.passes_cuts(p))


def test_uniform_stream_matches_the_generator_construction():
    """Uniform k of candidate i is draw k of the per-point stream pacuda_b200.phase_space.rambo
    uses (the same seeding and xorshift), so the two generators share one construction."""
    u = U.uniforms(99, np.arange(8, dtype=np.uint64))
    assert u.shape == (8, 7) and np.all((u > 0) & (u < 1))
    assert len(np.unique(u)) == u.size


def test_two_stage_toy_is_unbiased():
    """With a surrogate off by up to 20 % the two-stage events, with their weights, follow the
    exact density as the plain events do (chi^2 per bin near 1), and each exact evaluation
    gives several times more events."""
    x, f, (xp, wp), (x2, w2) = U.toy_two_stage(1 << 21, 7)
    edges = np.linspace(0, 1, 21)
    for axis in (0, 1):
        for xs, ws in ((xp, wp), (x2, w2)):
            chi2, bins = unweight.chi2_against(x[:, axis], f, xs[:, axis], ws, edges)
            assert chi2 / bins < 2.0, (axis, chi2, bins)
    # events per exact evaluation: plain = kept / all, two-stage = kept / first-stage survivors
    eff_plain = len(xp) / len(x)
    s = f * (1.0 + 0.2 * np.sin(7.0 * x[:, 0]) * np.cos(5.0 * x[:, 1]))
    first = (np.random.default_rng(7).uniform(size=(4, len(x)))[2] * s.max() * 0.9 < s).sum()
    assert len(x2) / max(1, first) > 2 * eff_plain


def test_two_stage_toy_detects_a_biased_rule():
    """The chi^2 check has power: events of the first stage alone (the surrogate's distribution,
    no exact second stage) differ visibly from the density when the surrogate is 30 % off."""
    rng = np.random.default_rng(8)
    n = 1 << 21
    x = rng.uniform(size=(n, 2))
    f = np.exp(-((x[:, 0] - 0.3) ** 2 + (x[:, 1] - 0.6) ** 2) / 0.02) + 0.2
    s = f * (1.0 + 0.3 * np.sin(7.0 * x[:, 0]) * np.cos(5.0 * x[:, 1]))
    keep = U.stage1_decide(s, rng.uniform(size=n), s.max())
    edges = np.linspace(0, 1, 21)
    chi2_bad, bins = unweight.chi2_against(x[:, 0], f, x[keep, 0], np.ones(keep.sum()), edges)
    assert chi2_bad > 10 * bins


def test_reduced_maximum():
    """The reduced maximum leaves at most the asked share of the total above it, and is the
    largest value for a share of 0."""
    rng = np.random.default_rng(9)
    v = rng.pareto(3.0, 100000) + 1e-3
    for eps in (0.0, 1e-4, 1e-3, 1e-2):
        t = unweight.maxima(v, overweight=eps)
        assert np.maximum(0, v - t).sum() <= eps * v.sum() * (1 + 1e-9)
        if eps == 0.0:
            assert t == v.max()
    assert unweight.maxima(v, overweight=1e-2) < unweight.maxima(v, overweight=1e-4)
    w = rng.uniform(0, 2, v.size)
    t = unweight.maxima(v, w, 1e-3)
    assert (w * np.maximum(0, v - t)).sum() <= 1e-3 * (w * v).sum() * (1 + 1e-9)


def test_map_weight_integrates_to_the_three_body_volume():
    """J factorises into one function of x1, x2 and x4 each: their integrals by quadrature give
    the massless three-body volume s / (256 pi^3) up to the two truncated rapidity ranges."""
    from scipy.integrate import quad

    sqrt_s = 13000.0
    s = sqrt_s * sqrt_s

    def j(x1, x2, x4):
        u = np.zeros((1, 7))
        u[0, 0], u[0, 1], u[0, 3] = x1, x2, x4
        return U.weight(u, sqrt_s)[0]

    g1 = quad(lambda x: j(x, 0.5, 0.5), 0, 1, points=[0.5], limit=200)[0]
    g2 = quad(lambda x: j(0.5, x, 0.5), 0, 1, limit=200)[0] / j(0.5, 0.5, 0.5)
    g4 = quad(lambda x: j(0.5, 0.5, x), 0, 1, limit=200)[0] / j(0.5, 0.5, 0.5)
    vol = g1 * g2 * g4
    assert vol == pytest.approx(s / (256.0 * math.pi ** 3), rel=5e-5)
    assert vol < s / (256.0 * math.pi ** 3)
