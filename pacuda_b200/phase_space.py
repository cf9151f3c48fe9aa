"""Seeded massless phase space (RAMBO) and jet cuts, for synthetic benchmark and test points.

RAMBO (Kleiss, Stirling, Ellis, Comput. Phys. Commun. 40 (1986) 359), massless, with the
uniforms drawn as the reference's recorder draws them (convert/src/record.rs:17-52): a
xorshift64 stream (shifts 13, 7, 17), uniform = ((state >> 11) + 0.5) / 2^53, four per
final-state particle in the order cos(theta), phi, and the two factors of the energy
-ln(u1 u2). Beams are (sqrt(s)/2)(1, 0, 0, +-1).

`rambo_reference` reproduces the recorder's single stream point by point; `rambo` is the
vectorised form used for large samples, one stream per point (seeded by splitmix64 of the
sample seed and the point index), so that any point can be regenerated alone.
"""
from __future__ import annotations

import math

import numpy as np

_M64 = (1 << 64) - 1


def _xorshift(state):
    state ^= (state << 13) & _M64
    state ^= state >> 7
    state ^= (state << 17) & _M64
    return state


def rambo_reference(n, points, seed, ecm=1000.0):
    """Point-major momenta [point][leg][E, px, py, pz] of `n` legs, one xorshift stream."""
    state = (seed | 1) & _M64
    out = np.empty((points, n, 4))

    def uniform():
        nonlocal state
        state = _xorshift(state)
        return ((state >> 11) + 0.5) / float(1 << 53)

    m = n - 2
    for i in range(points):
        q = np.empty((m, 4))
        for j in range(m):
            c = 2.0 * uniform() - 1.0
            s = math.sqrt(1.0 - c * c)
            f = 2.0 * math.pi * uniform()
            e = -math.log(uniform() * uniform())
            q[j] = (e, e * s * math.cos(f), e * s * math.sin(f), e * c)
        out[i, :2] = _boost(q[None], ecm)[1][0, :2]
        out[i, 2:] = _boost(q[None], ecm)[1][0, 2:]
    return out


def _boost(q, ecm):
    """RAMBO's conformal transformation of the massless vectors q[point][j] to the centre-of-mass
    frame of energy ecm; returns (weights unused, momenta [point][leg] with the two beams first)."""
    total = q.sum(axis=1)
    mass = np.sqrt(total[:, 0] ** 2 - total[:, 1] ** 2 - total[:, 2] ** 2 - total[:, 3] ** 2)
    b = -total[:, 1:] / mass[:, None]
    x = ecm / mass
    g = total[:, 0] / mass
    a = 1.0 / (1.0 + g)
    bq = (b[:, None, :] * q[:, :, 1:]).sum(axis=2)
    p = np.empty_like(q)
    p[:, :, 0] = x[:, None] * (g[:, None] * q[:, :, 0] + bq)
    p[:, :, 1:] = x[:, None, None] * (q[:, :, 1:] + b[:, None, :] * (q[:, :, :1] + a[:, None, None] * bq[:, :, None]))
    points = q.shape[0]
    out = np.empty((points, q.shape[1] + 2, 4))
    out[:, 0] = (ecm / 2, 0.0, 0.0, ecm / 2)
    out[:, 1] = (ecm / 2, 0.0, 0.0, -ecm / 2)
    out[:, 2:] = p
    return None, out


def _splitmix(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_M64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_M64)
    return z ^ (z >> np.uint64(31))


def rambo(n, points, seed, ecm=1000.0, first=0):
    """Point-major momenta [point][leg][4] of `n` legs for points first .. first+points-1."""
    with np.errstate(over="ignore"):
        idx = np.arange(first, first + points, dtype=np.uint64)
        state = _splitmix(np.uint64(seed) ^ (idx * np.uint64(0xD1B54A32D192ED03))) | np.uint64(1)
        m = n - 2
        u = np.empty((points, m, 4))
        for j in range(m):
            for k in range(4):
                state ^= state << np.uint64(13)
                state ^= state >> np.uint64(7)
                state ^= state << np.uint64(17)
                u[:, j, k] = ((state >> np.uint64(11)).astype(np.float64) + 0.5) / float(1 << 53)
    c = 2.0 * u[:, :, 0] - 1.0
    s = np.sqrt(1.0 - c * c)
    f = 2.0 * np.pi * u[:, :, 1]
    e = -np.log(u[:, :, 2] * u[:, :, 3])
    q = np.stack([e, e * s * np.cos(f), e * s * np.sin(f), e * c], axis=2)
    return _boost(q, ecm)[1]


def passes_cuts(p, pt_min=20.0, eta_max=5.0, dr_min=0.4):
    """Boolean mask of points whose final-state partons (legs 2..) all pass pT > pt_min,
    |eta| < eta_max and pairwise Delta R > dr_min."""
    fin = p[:, 2:]
    pt = np.hypot(fin[..., 1], fin[..., 2])
    pabs = np.sqrt(pt * pt + fin[..., 3] ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        eta = 0.5 * np.log((pabs + fin[..., 3]) / (pabs - fin[..., 3]))
    phi = np.arctan2(fin[..., 2], fin[..., 1])
    ok = (pt > pt_min).all(axis=1) & (np.abs(eta) < eta_max).all(axis=1)
    m = fin.shape[1]
    for i in range(m):
        for j in range(i + 1, m):
            dphi = np.abs(phi[:, i] - phi[:, j])
            dphi = np.where(dphi > np.pi, 2 * np.pi - dphi, dphi)
            ok &= np.hypot(eta[:, i] - eta[:, j], dphi) > dr_min
    return ok & np.isfinite(eta).all(axis=1)


def sample(n, points, seed, ecm=1000.0, pt_min=20.0, eta_max=5.0, dr_min=0.4):
    """`points` RAMBO points of `n` legs that pass the cuts (rejection), point-major."""
    out, have, first = [], 0, 0
    while have < points:
        batch = max(1024, 2 * (points - have))
        p = rambo(n, batch, seed, ecm, first)
        first += batch
        p = p[passes_cuts(p, pt_min, eta_max, dr_min)]
        out.append(p[: points - have])
        have += len(out[-1])
    return np.concatenate(out)


def source_major(p, crossing=None):
    """The external momenta of point-major momenta p[point][leg][4] as the runner reads them:
    planes [(leg * 4 + k) * points + i] (umami/umami_pacuda.c:628-643)."""
    points, n, _ = p.shape
    return np.ascontiguousarray(p.transpose(1, 2, 0).reshape(n * 4 * points))
