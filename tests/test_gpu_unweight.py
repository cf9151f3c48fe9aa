"""The unweighting kernels (libsurrogate.so) against their restatement (oracle/unweight_oracle.py):
candidates inside the cuts, their points and weights, the accept/reject decisions; then the whole
two-stage pipeline on g g -> g g g with a briefly trained surrogate: its events follow the exact
weighted distribution (chi^2 per bin) and each exact evaluation yields more events than plain
unweighting's."""
import ctypes as C

import numpy as np
import pytest

from oracle import unweight_oracle as U

pytestmark = pytest.mark.gpu
SQRT_S = 13000.0


def _pipeline(families=("gg>ggg",), capacity=1 << 18):
    from pacuda_b200 import unweight

    return unweight.Pipeline(families=list(families), capacity=capacity)


@pytest.mark.parametrize("family,final_state", [("gg>ggg", 3), ("gg>gggg", 4)])
def test_candidates_and_points_match_oracle(family, final_state):
    import torch

    from pacuda_b200 import unweight

    pl = _pipeline((family,))
    assert pl.final_state == final_state
    seed = pl.family_seed(0)
    n = 50000
    idx = pl.passing(0, 1000, n).cpu().numpy().astype(np.uint64)
    u = U.uniforms(seed, np.arange(1000, 1000 + n, dtype=np.uint64), final_state)
    p, jac = U.momenta(u, SQRT_S, final_state)
    want = np.arange(1000, 1000 + n, dtype=np.uint64)[U.passes(p)]
    assert np.array_equal(idx, want)
    # points of the passing candidates
    m, legs, nx = len(idx), final_state + 2, 3 * final_state - 4
    ti = torch.tensor(idx.astype(np.int64), device="cuda")
    mom = torch.empty(4 * legs * m, dtype=torch.float64, device="cuda")
    x = torch.empty(m, nx + 1, dtype=torch.float32, device="cuda")
    j = torch.empty(m, dtype=torch.float64, device="cuda")
    L = unweight._lib()
    assert L.pacuda_uw_points(seed, C.c_void_p(ti.data_ptr()), m, final_state, SQRT_S, C.c_void_p(mom.data_ptr()),
                              C.c_void_p(x.data_ptr()), nx + 1, 0, C.c_void_p(j.data_ptr()), None) == 0
    torch.cuda.synchronize()
    keep = U.passes(p)
    got = mom.cpu().numpy().reshape(legs, 4, m).transpose(2, 0, 1)
    # exp, tanh and the boosts' cancellations round differently on the device: 1e-9 relative
    assert np.allclose(got, p[keep], rtol=1e-9, atol=1e-7)
    assert np.allclose(j.cpu().numpy(), jac[keep], rtol=1e-10, atol=0)
    assert np.array_equal(x.cpu().numpy(), U.features(u[keep], 0, 1, final_state))


@pytest.mark.parametrize("family,final_state", [("qg>qgg", 3), ("qg>qggg", 4)])
def test_listing_of_many_candidates_matches_oracle(family, final_state):
    """2^22 candidates: the device's list (an f32 first look that drops only certain failures,
    then the f64 map and cuts for the rest) holds exactly the candidates the f64 restatement
    passes."""
    pl = _pipeline((family,), capacity=1 << 21)
    seed = pl.family_seed(0)
    n, first = 1 << 22, 12345
    got = pl.passing(0, first, n).cpu().numpy().astype(np.uint64)
    want = []
    for a in range(first, first + n, 1 << 20):
        idx = np.arange(a, min(first + n, a + (1 << 20)), dtype=np.uint64)
        p, _ = U.momenta(U.uniforms(seed, idx, final_state), SQRT_S, final_state)
        want.append(idx[U.passes(p)])
    want = np.concatenate(want)
    assert 0.01 < len(want) / n < 0.5
    assert np.array_equal(got, want), (len(got), len(want), np.setdiff1d(want, got)[:5], np.setdiff1d(got, want)[:5])


@pytest.mark.parametrize("count", [1, 255, 4095, 4097, 12289])
def test_listing_of_ragged_counts_matches_oracle(count):
    """Counts that leave a listing block partly filled (a block takes 16 rounds of 256 candidates),
    two families of different counts in one launch: each family's list is the f64 restatement's."""
    pl = _pipeline(("gg>ggg", "qg>qgg"))
    firsts = 777
    counts = [count, count + 3]
    n = pl.candidates(firsts, counts)
    for k in range(2):
        got = np.sort(pl.fams[k].cand[:n[k]].cpu().numpy().astype(np.uint64))
        idx = np.arange(firsts, firsts + counts[k], dtype=np.uint64)
        p, _ = U.momenta(U.uniforms(pl.family_seed(k), idx, 3), SQRT_S, 3)
        assert np.array_equal(got, idx[U.passes(p)])


def test_parts_of_a_family_add_up_to_the_oracle():
    """A subprocess of several plans (g g -> 4 g: three parts of its colour orderings): the
    pipeline's exact evaluation is the parts' outputs added in part order, bit for bit the
    oracle's parts added the same way."""
    import torch

    from oracle import oracle as O
    from pacuda_b200 import phase_space, processes

    pl = _pipeline(("gg>gggg",), capacity=1 << 12)
    fam = pl.fams[0]
    assert len(fam.plans) > 1
    idx = pl.passing(0, 0, 4000)[:300]
    m = idx.numel()
    out = pl.exact([idx], [m])[0].cpu().numpy()
    p = fam.momenta[: 24 * m].cpu().numpy().reshape(6, 4, m).transpose(2, 0, 1).copy()
    want = None
    for t in processes.parts("gg>gggg"):
        _, w = O.evaluate(t, p, kernel=1)
        want = w if want is None else want + w
    assert np.array_equal(out.view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("final_state", [3, 4])
def test_decisions_match_oracle(final_state):
    import torch

    from pacuda_b200 import unweight

    rng = np.random.default_rng(3)
    n, hel = 5000, 32
    idx = np.arange(77, 77 + n, dtype=np.uint64)
    seed = 1234
    out = rng.exponential(size=(n, hel))
    jac = rng.uniform(0.1, 1.0, n)
    s = rng.uniform(0.5, 2.0, n) * out.sum(axis=1) * jac
    dev = lambda a, t=torch.float64: torch.tensor(a, dtype=t, device="cuda")  # noqa: E731
    ti, to, tj, ts = dev(idx.astype(np.int64), torch.int64), dev(out.reshape(-1)), dev(jac), dev(s)
    keep = torch.empty(n, dtype=torch.uint8, device="cuda")
    wt = torch.empty(n, dtype=torch.float64, device="cuda")
    me = torch.empty(n, dtype=torch.float64, device="cuda")
    L = unweight._lib()
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    m2 = np.zeros(n)
    for h in range(hel):
        m2 = m2 + out[:, h]
    w = m2 * jac
    u = U.uniforms(seed, idx, final_state)
    nx = U.numbers(final_state)
    # plain
    w_max = float(np.quantile(w, 0.9))
    assert L.pacuda_uw_decide(seed, P(ti), n, final_state, P(to), hel, P(tj), None, w_max, 0.0, 0.0, P(keep), P(wt),
                              P(me), None) == 0
    k, weights = U.plain_decide(w, u[:, nx], w_max)
    assert np.array_equal(keep.cpu().numpy().astype(bool), k)
    assert np.array_equal(wt.cpu().numpy(), weights)
    assert np.array_equal(me.cpu().numpy(), m2)
    # second stage
    s_max, r_max = float(np.quantile(s, 0.95)), 1.2
    assert L.pacuda_uw_decide(seed, P(ti), n, final_state, P(to), hel, P(tj), P(ts), 0.0, s_max, r_max, P(keep),
                              P(wt), None, None) == 0
    k2, w2, _ = U.stage2_decide(w, s, np.maximum(1.0, s / s_max), u[:, nx + 1], r_max)
    assert np.array_equal(keep.cpu().numpy().astype(bool), k2)
    assert np.allclose(wt.cpu().numpy(), w2, rtol=1e-15, atol=0)


@pytest.mark.parametrize("family,final_state", [("gg>ggg", 3), ("gg>gggg", 4)])
def test_stage1_matches_oracle(family, final_state):
    """The fused first stage (inputs, network, decision in one launch) over a list of
    candidates keeps those the restatement keeps with the CPU network's values, except where
    u s_max lies within 2 % of s (the device network rounds differently)."""
    import torch

    from oracle import surrogate_oracle as SO
    from pacuda_b200 import surrogate as S
    from pacuda_b200 import unweight

    pl = _pipeline((family,))
    nx = U.numbers(final_state)
    net = S.Network(nx + 1, max_batch=1024, seed=5)
    p = net.params()
    mu, sigma = -2.0, 1.5
    n, first = 40000, 123
    seed = pl.family_seed(0)
    cand = pl.passing(0, first, n)  # sorted indices inside the cuts
    idx = cand.cpu().numpy().astype(np.uint64)
    u = U.uniforms(seed, idx, final_state)
    out = SO.forward(p, U.features(u, 0, 1, final_state)).astype(np.float64)
    sv = np.exp(mu + sigma * out)
    s_max = float(np.quantile(sv, 0.99))
    pl.counters.zero_()
    L = unweight._lib()
    f0 = pl.fams[0]
    assert L.pacuda_uw_stage1(net.handle, seed, C.c_void_p(cand.data_ptr()), cand.numel(), final_state, 0, mu, sigma,
                              s_max, C.c_void_p(f0.kept.data_ptr()), C.c_void_p(f0.kept_s.data_ptr()), pl.capacity,
                              C.c_void_p(pl.counters.data_ptr()), None) == 0
    torch.cuda.synchronize()
    assert net.error() == 0
    kept = int(pl.counters[0])
    got = f0.kept[:kept].cpu().numpy().astype(np.uint64)
    pos = {int(c): i for i, c in enumerate(idx)}
    want_keep = u[:, nx] * s_max < sv
    borderline = np.abs(u[:, nx] * s_max - sv) <= 0.02 * np.maximum(sv, 1e-300)
    got_mask = np.zeros(len(idx), dtype=bool)
    got_mask[[pos[int(c)] for c in got]] = True
    assert np.array_equal(got_mask[~borderline], want_keep[~borderline])
    ks = f0.kept_s[:kept].cpu().numpy()
    assert np.allclose(ks, sv[[pos[int(c)] for c in got]], rtol=0.05)


def test_two_stage_is_unbiased_and_gains_on_ggggg():
    """g g -> g g g at 13 TeV: a surrogate of log w trained for a few seconds on the labelled points
    of 2^20 candidates;
    two-stage and plain unweighting of the same 2^20 candidates, both with reduced maxima (1 % of
    the total above them). Both samples' histograms of the
    leading parton's pT, its pseudorapidity and m23 agree with the exact weighted histogram
    (chi^2 per bin below 2.5), and the two-stage events per exact evaluation exceed plain's."""
    import torch

    from pacuda_b200 import surrogate as S
    from pacuda_b200 import unweight

    pl = _pipeline(capacity=1 << 20)
    x, me, jac, _ = pl.labelled(0, 1 << 30, 1 << 20)
    w = me * jac
    logw = w.log()
    mu, sigma = float(logw.mean()), float(logw.std())
    y = ((logw - mu) / sigma).float()
    net = S.Network(6, max_batch=4096, seed=3)
    imp = (0.5 * (logw - logw.max())).exp().float()  # training points drawn in proportion to w^0.5
    unweight.train(net, x, y, epochs=80, batch=4096, lr=2e-3, lr_end=1e-5, importance=imp)
    assert net.error() == 0
    s = pl.surrogate_values(net, x, mu, sigma)
    # reduced maxima: at most 1 % of the total above each (those events keep weights above 1)
    w_max = unweight.maxima(w, overweight=1e-2)
    s_max = unweight.maxima(s, overweight=1e-2)
    r_max = unweight.maxima(w / s, s, overweight=1e-2)
    n_cand = 1 << 20
    xa, ma, ja, idx_all = pl.labelled(0, 0, n_cand)
    wa = (ma * ja).cpu().numpy()
    ev, exact_p = pl.plain(0, [n_cand], [w_max])
    ip, wp = ev[0].compact()
    assert int(ev[0].count()) == len(ip)
    ev, exact_2 = pl.two_stage(net, 0, [n_cand], mu, sigma, [s_max], [r_max])
    i2, w2 = ev[0].compact()
    assert exact_p == idx_all.numel()
    print(f"plain: {len(ip)} events from {exact_p} exact evaluations; two-stage: {len(i2)} from {exact_2}")
    assert len(ip) > 50 and len(i2) > 50, (len(ip), len(i2), exact_p, exact_2)
    seed = pl.family_seed(0)

    def moms(index):
        u = U.uniforms(seed, index.cpu().numpy().astype(np.uint64))
        return U.phase_space(u, SQRT_S)[0]

    ref = unweight.observables(moms(idx_all))
    ev_p, ev_2 = unweight.observables(moms(ip)), unweight.observables(moms(i2))
    for name in ref:
        edges = unweight.log_edges(ref[name], 12)
        for ev, ww in ((ev_p, wp), (ev_2, w2)):
            chi2, bins = unweight.chi2_against(ref[name], wa, ev[name], ww.cpu().numpy(), edges)
            assert chi2 / max(1, bins) < 2.5, (name, chi2, bins)
    eff_plain = len(ip) / exact_p
    eff_two = len(i2) / max(1, exact_2)
    assert eff_two > 3 * eff_plain, (eff_two, eff_plain)


def test_training_with_importance_is_reproducible():
    """Two trainings on the same points with the same importance and seed end in the same bits
    (the draws come from a seeded generator by inverse CDF)."""
    import torch

    from pacuda_b200 import surrogate as S
    from pacuda_b200 import unweight

    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    x = torch.rand(1 << 15, 9, device="cuda", generator=g)
    y = torch.randn(1 << 15, device="cuda", generator=g)
    imp = torch.rand(1 << 15, device="cuda", generator=g) ** 4
    runs = []
    for _ in range(2):
        net = S.Network(9, max_batch=4096, seed=2)
        hist = unweight.train(net, x, y, epochs=2, batch=4096, importance=imp, seed=3)
        runs.append((hist, net.params()))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1].view(np.uint32), runs[1][1].view(np.uint32))
