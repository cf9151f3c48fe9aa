"""Test infrastructure: numpy restatement of the unweighting kernels (libsurrogate.so), the checker
of their phase-space points, cuts and accept/reject decisions, and a CPU toy of two-stage
unweighting with a known density.

Candidate i of a stream with seed S draws its uniforms from a xorshift64 stream (shifts 13, 7,
17; uniform = ((state >> 11) + 0.5) / 2^53) started at splitmix64(S ^ (i * 0xD1B54A32D192ED03)) | 1
-- the construction pacuda_b200/phase_space.rambo uses. With N final-state partons, uniforms
0 .. 3N - 5 are the phase-space numbers, 3N - 4 the first accept/reject number, 3N - 3 the second
(N = 3: 0-4, 5, 6; N = 4: 0-7, 8, 9).

The phase-space map (massless 2 -> 3 at fixed sqrt(s), sequential two-body decays, each
variable importance-sampled where |M|^2 peaks):
  s23 = s sigma(y), y = L (2 x1 - 1), sigma the logistic function; p1 in the centre-of-mass frame
  with |p1| = (s - s23) / (2 sqrt(s)), cos(theta) = tanh(E1 (2 x2 - 1)), phi = 2 pi x3; p2, p3
  back to back in the rest frame of q = P - p1 with |p| = sqrt(s23) / 2, cos(theta) =
  tanh(E2 (2 x4 - 1)), phi = 2 pi x5, boosted along q; L = 16, E1 = 5.5, E2 = 7.
  Its weight (the phase-space density of the unit cube):
  J = s (1 - sigma) / (128 pi^3) 2 L sigma (1 - sigma) E1 (1 - cos^2 theta1) E2 (1 - cos^2 theta2);
  with L, E1, E2 unbounded its integral is s / (256 pi^3), the massless three-body volume
  (RAMBO's); at these values it misses m23 below 4.4 GeV at 13 TeV (the cuts need 8 GeV) and a
  q-frame solid angle of 1.7e-6.

The 2 -> 4 map adds one decay (P -> p1 + Q, Q -> p2 + R, R -> p3 + p4):
  s_Q = s sigma(L (2 x1 - 1)), s_R = s_Q sigma(L (2 x4 - 1)); p1 as above from x2, x3 with
  |p1| = (s - s_Q) / (2 sqrt(s)); p2 in the rest frame of Q with |p2| = (s_Q - s_R) / (2 sqrt(s_Q)),
  cos(theta) = tanh(E2 (2 x5 - 1)), phi = 2 pi x6, R opposite with energy (s_Q + s_R) / (2 sqrt(s_Q));
  p3, p4 back to back in the rest frame of R with |p| = sqrt(s_R) / 2, cos(theta) = tanh(E2 (2 x7 - 1)),
  phi = 2 pi x8, boosted to Q's frame along R, then with p2 to the lab along Q. From
  dPhi_4 = dPhi_2(P; p1, Q) ds_Q / 2 pi dPhi_2(Q; p2, R) ds_R / 2 pi dPhi_2(R; p3, p4) with
  dPhi_2(K; massless, mass^2 m) = (K^2 - m) / (32 pi^2 K^2) dOmega, its weight is
  J = s s_Q (1 - sigma1) (1 - sigma2) / (2048 pi^5) 2 L sigma1 (1 - sigma1) 2 L sigma2 (1 - sigma2)
      E1 (1 - c1^2) E2 (1 - c2^2) E2 (1 - c3^2),
  whose flat form integrates to the massless four-body volume s^2 / (24576 pi^5).
"""
from __future__ import annotations

import math

import numpy as np

_M64 = (1 << 64) - 1
UNIFORMS = 7
MAP_L, MAP_E1, MAP_E2 = 16.0, 5.5, 7.0


def _splitmix(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_M64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_M64)
    return z ^ (z >> np.uint64(31))


def numbers(final_state):
    """The phase-space numbers of N final-state partons: 3N - 4."""
    return 3 * final_state - 4


def uniforms(seed, index, final_state=3):
    """[len(index)][3N - 2] uniforms of the candidates `index` (uint64 array) of stream `seed`."""
    count = numbers(final_state) + 2
    with np.errstate(over="ignore"):
        idx = np.asarray(index, dtype=np.uint64)
        state = _splitmix(np.uint64(seed) ^ (idx * np.uint64(0xD1B54A32D192ED03))) | np.uint64(1)
        u = np.empty((idx.size, count))
        for k in range(count):
            state ^= state << np.uint64(13)
            state ^= state >> np.uint64(7)
            state ^= state << np.uint64(17)
            u[:, k] = ((state >> np.uint64(11)).astype(np.float64) + 0.5) / float(1 << 53)
    return u


def _boost(p, b):
    """p [n][4] boosted by velocity b [n][3] (the frame moving with -b sees p at rest if b = v)."""
    b2 = (b * b).sum(axis=1)
    g = 1.0 / np.sqrt(1.0 - b2)
    bp = (b * p[:, 1:]).sum(axis=1)
    gg = np.where(b2 > 0, (g - 1.0) / np.where(b2 > 0, b2, 1.0), 0.0)
    out = np.empty_like(p)
    out[:, 0] = g * (p[:, 0] + bp)
    out[:, 1:] = p[:, 1:] + (gg * bp + g * p[:, 0])[:, None] * b
    return out


def weight(u, sqrt_s):
    """The map's weight J from the uniforms alone."""
    s = sqrt_s * sqrt_s
    sg = 1.0 / (1.0 + np.exp(-MAP_L * (2.0 * u[:, 0] - 1.0)))
    c1 = np.tanh(MAP_E1 * (2.0 * u[:, 1] - 1.0))
    c2 = np.tanh(MAP_E2 * (2.0 * u[:, 3] - 1.0))
    return (s * (1.0 - sg) / (128.0 * math.pi ** 3) * (2.0 * MAP_L * sg * (1.0 - sg)) * (MAP_E1 * (1.0 - c1 * c1)) *
            (MAP_E2 * (1.0 - c2 * c2)))


def phase_space(u, sqrt_s):
    """Point-major momenta [n][5][4] (beams first) and the weight J of the uniforms u[:, :5]."""
    s = sqrt_s * sqrt_s
    n = u.shape[0]
    sg = 1.0 / (1.0 + np.exp(-MAP_L * (2.0 * u[:, 0] - 1.0)))
    s23 = s * sg
    e1 = (s - s23) / (2.0 * sqrt_s)
    c1 = np.tanh(MAP_E1 * (2.0 * u[:, 1] - 1.0))
    st1 = np.sqrt(np.maximum(0.0, 1.0 - c1 * c1))
    f1 = 2.0 * math.pi * u[:, 2]
    p1 = np.stack([e1, e1 * st1 * np.cos(f1), e1 * st1 * np.sin(f1), e1 * c1], axis=1)
    k = 0.5 * np.sqrt(s23)
    c2 = np.tanh(MAP_E2 * (2.0 * u[:, 3] - 1.0))
    st2 = np.sqrt(np.maximum(0.0, 1.0 - c2 * c2))
    f2 = 2.0 * math.pi * u[:, 4]
    p2r = np.stack([k, k * st2 * np.cos(f2), k * st2 * np.sin(f2), k * c2], axis=1)
    p3r = np.stack([k, -p2r[:, 1], -p2r[:, 2], -p2r[:, 3]], axis=1)
    eq = sqrt_s - e1
    b = -p1[:, 1:] / eq[:, None]
    p = np.empty((n, 5, 4))
    p[:, 0] = (0.5 * sqrt_s, 0.0, 0.0, 0.5 * sqrt_s)
    p[:, 1] = (0.5 * sqrt_s, 0.0, 0.0, -0.5 * sqrt_s)
    p[:, 2] = p1
    p[:, 3] = _boost(p2r, b)
    p[:, 4] = _boost(p3r, b)
    return p, weight(u, sqrt_s)


def weight4(u, sqrt_s):
    """The 2 -> 4 map's weight J from the uniforms alone."""
    s = sqrt_s * sqrt_s
    sg1 = 1.0 / (1.0 + np.exp(-MAP_L * (2.0 * u[:, 0] - 1.0)))
    sg2 = 1.0 / (1.0 + np.exp(-MAP_L * (2.0 * u[:, 3] - 1.0)))
    sq = s * sg1
    c1 = np.tanh(MAP_E1 * (2.0 * u[:, 1] - 1.0))
    c2 = np.tanh(MAP_E2 * (2.0 * u[:, 4] - 1.0))
    c3 = np.tanh(MAP_E2 * (2.0 * u[:, 6] - 1.0))
    return (s * sq * (1.0 - sg1) * (1.0 - sg2) / (2048.0 * math.pi ** 5) * (2.0 * MAP_L * sg1 * (1.0 - sg1)) *
            (2.0 * MAP_L * sg2 * (1.0 - sg2)) * (MAP_E1 * (1.0 - c1 * c1)) * (MAP_E2 * (1.0 - c2 * c2)) *
            (MAP_E2 * (1.0 - c3 * c3)))


def _direction(k, c, f):
    st = np.sqrt(np.maximum(0.0, 1.0 - c * c))
    return np.stack([k, k * st * np.cos(f), k * st * np.sin(f), k * c], axis=1)


def phase_space4(u, sqrt_s):
    """Point-major momenta [n][6][4] (beams first) and the weight J of the uniforms u[:, :8]."""
    s = sqrt_s * sqrt_s
    n = u.shape[0]
    sg1 = 1.0 / (1.0 + np.exp(-MAP_L * (2.0 * u[:, 0] - 1.0)))
    sq = s * sg1
    sg2 = 1.0 / (1.0 + np.exp(-MAP_L * (2.0 * u[:, 3] - 1.0)))
    sr = sq * sg2
    e1 = (s - sq) / (2.0 * sqrt_s)
    p1 = _direction(e1, np.tanh(MAP_E1 * (2.0 * u[:, 1] - 1.0)), 2.0 * math.pi * u[:, 2])
    mq = np.sqrt(sq)
    q2 = _direction((sq - sr) / (2.0 * mq), np.tanh(MAP_E2 * (2.0 * u[:, 4] - 1.0)), 2.0 * math.pi * u[:, 5])
    er = (sq + sr) / (2.0 * mq)
    r3 = _direction(0.5 * np.sqrt(sr), np.tanh(MAP_E2 * (2.0 * u[:, 6] - 1.0)), 2.0 * math.pi * u[:, 7])
    r4 = np.stack([r3[:, 0], -r3[:, 1], -r3[:, 2], -r3[:, 3]], axis=1)
    br = -q2[:, 1:] / er[:, None]
    q3, q4 = _boost(r3, br), _boost(r4, br)
    bq = -p1[:, 1:] / (sqrt_s - e1)[:, None]
    p = np.empty((n, 6, 4))
    p[:, 0] = (0.5 * sqrt_s, 0.0, 0.0, 0.5 * sqrt_s)
    p[:, 1] = (0.5 * sqrt_s, 0.0, 0.0, -0.5 * sqrt_s)
    p[:, 2] = p1
    p[:, 3] = _boost(q2, bq)
    p[:, 4] = _boost(q3, bq)
    p[:, 5] = _boost(q4, bq)
    return p, weight4(u, sqrt_s)


def momenta(u, sqrt_s, final_state=3):
    """The map of N final-state partons: momenta [n][N + 2][4] and J."""
    return phase_space4(u, sqrt_s) if final_state == 4 else phase_space(u, sqrt_s)


def passes(p, pt_min=20.0, eta_max=5.0, dr_min=0.4):
    """The cuts on the final-state legs 2 ..: pT^2 > pt_min^2, |pz| < pT sinh(eta_max)
    (|eta| < eta_max), pairwise Delta R > dr_min with eta = asinh(pz / pT), phi = atan2(py, px)."""
    fin = p[:, 2:]
    pt2 = fin[..., 1] ** 2 + fin[..., 2] ** 2
    pt = np.sqrt(pt2)
    ok = (pt2 > pt_min * pt_min).all(axis=1) & (np.abs(fin[..., 3]) < pt * math.sinh(eta_max)).all(axis=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        eta = np.arcsinh(fin[..., 3] / pt)
    phi = np.arctan2(fin[..., 2], fin[..., 1])
    nf = fin.shape[1]
    for i in range(nf):
        for j in range(i + 1, nf):
            d = np.abs(phi[:, i] - phi[:, j])
            d = np.where(d > math.pi, 2.0 * math.pi - d, d)
            de = eta[:, i] - eta[:, j]
            ok &= de * de + d * d > dr_min * dr_min
    return ok


def features(u, family, families, final_state=3):
    """The network's inputs: the 3N - 4 phase-space numbers, then the subprocess one-hot."""
    x = numbers(final_state)
    f = np.zeros((u.shape[0], x + families), dtype=np.float32)
    f[:, :x] = u[:, :x]
    f[:, x + family] = 1.0
    return f


def plain_decide(w, u, w_max):
    """Plain unweighting: keep a point when u w_max < w; its weight max(1, w / w_max)."""
    keep = u * w_max < w
    return keep, np.where(keep, np.maximum(1.0, w / w_max), 0.0)


def stage1_decide(s, u, s_max):
    return u * s_max < s


def stage2_decide(w, s, s_over, u, r_max):
    """Second stage: r = w / s; keep when u r_max < r; weight max(1, s / s_max) max(1, r / r_max)
    (`s_over` = max(1, s / s_max) of the first stage)."""
    r = w / s
    keep = u * r_max < r
    return keep, np.where(keep, s_over * np.maximum(1.0, r / r_max), 0.0), r


def toy_two_stage(n, seed, bias=0.2):
    """A CPU toy of two-stage unweighting on [0,1]^2 with the density f(x, y) = exp(-((x - 0.3)^2 +
    (y - 0.6)^2) / 0.02) + 0.2 and a surrogate off by a smooth factor up to 1 +- bias: the accepted
    events with their weights, and the plain unweighting's, for unbiasedness tests."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(size=(n, 2))
    f = np.exp(-((x[:, 0] - 0.3) ** 2 + (x[:, 1] - 0.6) ** 2) / 0.02) + 0.2
    s = f * (1.0 + bias * np.sin(7.0 * x[:, 0]) * np.cos(5.0 * x[:, 1]))
    u1, u2, u3 = rng.uniform(size=(3, n))
    f_max, s_max = f.max() * 0.9, s.max() * 0.9  # reduced maxima: some weights above 1
    keep_p, w_p = plain_decide(f, u1, f_max)
    k1 = stage1_decide(s, u2, s_max)
    keep2, w2, _ = stage2_decide(f[k1], s[k1], np.maximum(1.0, s[k1] / s_max), u3[k1], np.quantile(f[k1] / s[k1], 0.99))
    return x, f, (x[keep_p], w_p[keep_p]), (x[k1][keep2], w2[keep2])
