"""Two-stage unweighting of massless 2 -> 3 and 2 -> 4 subprocesses with the surrogate as its first stage
(include/pacuda_surrogate.h) and the f64 recurrence runner (include/pacuda_b200.h) as the exact
second stage; plain unweighting with the runner alone beside it.

Per subprocess ("family"), candidates are seeded points of the unit cube mapped to phase space
(`oracle/unweight_oracle.py` restates the map, the cuts and the decisions):

* plain: every candidate inside the cuts is evaluated exactly, w = |M|^2 J, and kept when
  u_a w_max < w, with weight max(1, w / w_max);
* two-stage: the surrogate s = exp(mu + sigma net(x)), trained on the standardized log of the
  weight w = |M|^2 J, is evaluated on every candidate inside the cuts (one fused launch: inputs,
  network, decision); the kept ones (u_a s_max < s) are evaluated exactly and kept when
  u_b r_max < r, r = w / s, with weight max(1, s / s_max) max(1, r / r_max)
(u_a, u_b: the candidate's two decision uniforms after its phase-space numbers).

With those weights both samples are unbiased estimates of the distribution of w: a kept event's
expected weight is w / (w_max) (plain) or w / (s_max r_max) (two-stage) for every candidate,
whatever the surrogate's error; the surrogate only changes how many exact evaluations an event
costs. The maxima are taken from a pilot sample; a larger weight than the maximum is kept as
weight above 1 rather than clipped.

The host side here sequences device work: launches of the two libraries, counters read back
once per step (the number of kept candidates sizes the exact evaluation).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import batch as B
from . import processes
from . import surrogate as S

FAMILIES = list(processes.PP3J)
ECM = 13000.0


def final_state_of(name):
    """The final-state partons of a subprocess (3 or 4)."""
    return len(processes.PROCESSES[name]) - 2


class Cuts(C.Structure):
    _fields_ = [("pt_min", C.c_double), ("eta_max", C.c_double), ("dr_min", C.c_double)]


class CandidateSegment(C.Structure):  # pacuda_uw_candidate_segment
    _fields_ = [("seed", C.c_uint64), ("first", C.c_uint64), ("count", C.c_uint32), ("index", C.c_void_p),
                ("counter", C.c_void_p)]


class Segment(C.Structure):  # pacuda_uw_segment
    _fields_ = [("seed", C.c_uint64), ("index", C.c_void_p), ("count", C.c_uint32), ("family", C.c_uint32),
                ("s_max", C.c_double), ("kept_index", C.c_void_p), ("kept_s", C.c_void_p), ("kept_count", C.c_void_p)]


def _lib():
    L = S.lib()
    if not getattr(L, "_uw_bound", False):
        L.pacuda_uw_candidates.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_double, C.c_void_p,
                                           C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        L.pacuda_uw_points.argtypes = [C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32, C.c_double, C.c_void_p,
                                       C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
        L.pacuda_uw_decide.argtypes = [C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
                                       C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]
        L.pacuda_uw_stage1.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_uint32,
                                       C.c_void_p, C.c_void_p]
        L.pacuda_uw_candidates_segments.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_double, C.c_void_p,
                                                    C.c_uint32, C.c_void_p]
        L.pacuda_uw_stage1_segments.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_double,
                                                C.c_double, C.c_uint32, C.c_void_p]
        L._uw_bound = True
    return L


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _check(status, what):
    if status != 0:
        raise S.SurrogateError(f"{what} returned {status}")


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Family:
    """One subprocess: its plans for the runner (f64; a subprocess too large for one plan's words
    has several, each over a part of its colour orderings, whose outputs add up) and its buffers
    (candidates inside the cuts, first-stage survivors, momenta and outputs of the exact
    evaluations, decisions)."""

    def __init__(self, name, index, capacity):
        import torch

        self.name, self.index = name, index
        self.templates = processes.parts(name)
        self.template = self.templates[0]
        self.helicities = self.template.outputs
        self.legs = len(processes.PROCESSES[name])
        self.plans = [B.Plan(t, "f64") for t in self.templates]
        self.capacity = capacity
        dev = "cuda"
        self.cand = torch.empty(capacity, dtype=torch.int64, device=dev)
        self.kept = torch.empty(capacity, dtype=torch.int64, device=dev)
        self.kept_s = torch.empty(capacity, dtype=torch.float64, device=dev)
        self.jac = torch.empty(capacity, dtype=torch.float64, device=dev)
        self.keep = torch.empty(capacity, dtype=torch.uint8, device=dev)
        self.weight = torch.empty(capacity, dtype=torch.float64, device=dev)
        self.momenta = torch.zeros(self.legs * 4 * capacity, dtype=torch.float64, device=dev)
        self.outputs = torch.empty(capacity * self.helicities, dtype=torch.float64, device=dev)
        # the other parts' outputs, added to the first part's after each evaluation
        self.part_outputs = [torch.empty(capacity * self.helicities, dtype=torch.float64, device=dev)
                             for _ in self.templates[1:]]


class Events:
    """One family's decided points of a run: candidate indices, keep flags and weights (views of the
    family's device buffers, valid until its next run); `compact()` gives the kept events alone."""

    def __init__(self, index, keep, weight):
        self.points, self.keep_flags, self.all_weights = index, keep, weight

    def count(self):
        """The number of kept events, as a device tensor (no host synchronisation)."""
        return self.keep_flags.sum(dtype=self.points.dtype) if self.points.numel() else self.points.new_zeros(())

    def compact(self):
        """(indices, weights) of the kept events (new tensors)."""
        keep = self.keep_flags.bool()
        return self.points[keep].clone(), self.all_weights[keep].clone()


class Pipeline:
    """Plain and two-stage unweighting over `families` at sqrt(s) with jet cuts. Every step works
    on all families at once: the candidates of every family listed (one read of the counts), the
    exact evaluations of every family in one batched launch of the runner."""

    def __init__(self, families=None, sqrt_s=ECM, cuts=(20.0, 5.0, 0.4), seed=20261204, capacity=1 << 20):
        import torch

        self.names = list(families or FAMILIES)
        states = {final_state_of(n) for n in self.names}
        if len(states) != 1:
            raise ValueError("the families of one pipeline have one final-state count")
        self.final_state = states.pop()
        self.numbers = 3 * self.final_state - 4
        self.sqrt_s = float(sqrt_s)
        self.cuts = Cuts(*cuts)
        self.seed = int(seed)
        self.inputs = self.numbers + len(self.names)
        self.capacity = capacity
        self.fams = [Family(n, k, capacity) for k, n in enumerate(self.names)]
        nf = len(self.fams)
        self.counters = torch.zeros(2 * nf, dtype=torch.int64, device="cuda")
        plans, moms, outs = self._parts([f.momenta[: 4 * f.legs * 1024] for f in self.fams], [1024] * nf)
        self.batch = B.Batch(plans, moms, outs)

    def _parts(self, moms, counts):
        """Every family's plans with their momenta and output buffers (the batch's order)."""
        plans, pm, po = [], [], []
        for f, m, c in zip(self.fams, moms, counts):
            for pl, o in zip(f.plans, [f.outputs] + f.part_outputs):
                plans.append(pl)
                pm.append(m)
                po.append(o[: c * f.helicities])
        return plans, pm, po

    def family_seed(self, k):
        return (self.seed * 1000003 + 7919 * (k + 1)) & ((1 << 64) - 1)

    # ---- steps on every family ----------------------------------------------------------------

    def candidates(self, first, counts):
        """Lists the candidates first .. first + counts[k] - 1 of every family k inside the cuts
        into the families' `cand` buffers (in no particular order); their numbers."""
        nf = len(self.fams)
        self.counters[:nf].zero_()
        segs = (CandidateSegment * nf)()
        for k, (fam, c) in enumerate(zip(self.fams, counts)):
            segs[k] = CandidateSegment(self.family_seed(k), first, int(c), fam.cand.data_ptr(),
                                       self.counters[k:k + 1].data_ptr())
        _check(_lib().pacuda_uw_candidates_segments(segs, nf, self.final_state, self.sqrt_s, C.byref(self.cuts),
                                                    self.capacity, _stream()), "candidates")
        n = [int(v) for v in self.counters[:nf].tolist()]
        if max(n) > self.capacity:
            raise S.SurrogateError(f"{max(n)} passing candidates exceed the capacity {self.capacity}")
        return n

    def exact(self, index, n, jac=True, inputs=None):
        """The f64 runner's outputs for candidates index[k][:n[k]] of every family (one batched
        launch; a family without points runs one stale point whose output is not used), with J into
        the families' `jac` buffers and, optionally, the network's inputs into inputs[k]."""
        import torch

        moms, counts = [], []
        if not any(n):
            return [f.outputs.view(-1, f.helicities)[:0] for f in self.fams]
        for k, (fam, idx, m) in enumerate(zip(self.fams, index, n)):
            if m:
                x = inputs[k] if inputs else None
                _check(_lib().pacuda_uw_points(self.family_seed(k), _ptr(idx), m, self.final_state, self.sqrt_s,
                                               _ptr(fam.momenta), _ptr(x) if x is not None else None,
                                               self.inputs if x is not None else 0, k,
                                               _ptr(fam.jac) if jac else None, _stream()), "points")
            mm = max(1, m)
            moms.append(fam.momenta[: 4 * fam.legs * mm])
            counts.append(mm)
        _, pm, po = self._parts(moms, counts)
        self.batch.update(pm, [c for f, c in zip(self.fams, counts) for _ in f.plans], po)
        self.batch.run(torch.cuda.current_stream())
        out = []
        for f, mm, m in zip(self.fams, counts, n):
            o = f.outputs[: mm * f.helicities]
            for extra in f.part_outputs:
                o += extra[: mm * f.helicities]
            out.append(o.view(-1, f.helicities)[:m])
        return out

    def tune(self):
        """Times the runner's launch choices on the points of the last exact evaluation (batch_tune)."""
        self.batch.tune()

    # ---- labelled points ------------------------------------------------------------------------

    def passing(self, k, first, count, sort=True):
        """Indices of the candidates first .. first + count - 1 of family k inside the cuts (sorted,
        a new tensor; or in no particular order, a view of the family's buffer)."""
        import torch

        counts = [0] * len(self.fams)
        counts[k] = count
        n = self.candidates(first, counts)[k]
        idx = self.fams[k].cand[:n]
        return torch.sort(idx)[0] if sort else idx

    def labelled(self, k, first, count):
        """(inputs [n][inputs] fp32, |M|^2 [n] f64, J [n] f64, index [n]) of the candidates of
        family k inside the cuts, in index order."""
        import torch

        idx = self.passing(k, first, count)
        n = idx.numel()
        x = torch.empty(n, self.inputs, dtype=torch.float32, device="cuda")
        index = [self.fams[j].cand[:0] for j in range(len(self.fams))]
        index[k] = idx
        counts = [0] * len(self.fams)
        counts[k] = n
        inputs = [None] * len(self.fams)
        inputs[k] = x
        out = self.exact(index, counts, jac=True, inputs=inputs)[k]
        return x, out.sum(dim=1), self.fams[k].jac[:n].clone(), idx

    # ---- the two pipelines -------------------------------------------------------------------

    def plain(self, first, counts, w_max):
        """Plain unweighting of candidates first .. first + counts[k] - 1 of every family k: the
        kept events per family and the number of exact evaluations."""
        n = self.candidates(first, counts)
        cand = [f.cand for f in self.fams]
        out = self.exact(cand, n)
        events = []
        for k, (fam, m) in enumerate(zip(self.fams, n)):
            if m:
                _check(_lib().pacuda_uw_decide(self.family_seed(k), _ptr(fam.cand), m, self.final_state, _ptr(out[k]),
                                               fam.helicities, _ptr(fam.jac), None, w_max[k], 0.0, 0.0,
                                               _ptr(fam.keep), _ptr(fam.weight), None, _stream()), "decide")
            events.append(Events(fam.cand[:m], fam.keep[:m], fam.weight[:m]))
        return events, sum(n)

    def two_stage(self, net, first, counts, mu, sigma, s_max, r_max):
        """Two-stage unweighting of the same candidates: the kept events per family and the number
        of exact evaluations."""
        nf = len(self.fams)
        n = self.candidates(first, counts)
        self.counters[nf:].zero_()
        segs = (Segment * nf)()
        for k, (fam, m) in enumerate(zip(self.fams, n)):
            segs[k] = Segment(self.family_seed(k), fam.cand.data_ptr(), m, k, s_max[k], fam.kept.data_ptr(),
                              fam.kept_s.data_ptr(), self.counters[nf + k:nf + k + 1].data_ptr())
        _check(_lib().pacuda_uw_stage1_segments(net.handle, segs, nf, self.final_state, mu, sigma, self.capacity,
                                                _stream()), "stage 1")
        kept = [int(v) for v in self.counters[nf:].tolist()]
        if max(kept) > self.capacity:
            raise S.SurrogateError(f"{max(kept)} first-stage events exceed the capacity {self.capacity}")
        out = self.exact([f.kept for f in self.fams], kept)
        events = []
        for k, (fam, m) in enumerate(zip(self.fams, kept)):
            if m:
                _check(_lib().pacuda_uw_decide(self.family_seed(k), _ptr(fam.kept), m, self.final_state, _ptr(out[k]),
                                               fam.helicities, _ptr(fam.jac), _ptr(fam.kept_s), 0.0, s_max[k],
                                               r_max[k], _ptr(fam.keep), _ptr(fam.weight), None, _stream()), "decide")
            events.append(Events(fam.kept[:m], fam.keep[:m], fam.weight[:m]))
        return events, sum(kept)

    def surrogate_values(self, net, x, mu, sigma):
        """s = exp(mu + sigma net(x)), the network's estimate of w = |M|^2 J, for points of known
        inputs (the fused inference kernel)."""
        out = net.forward(x)
        return (mu + sigma * out.double()).exp()


def train(net, x, y, epochs, batch=16384, lr=2e-3, lr_end=2e-5, seed=0, importance=None):
    """Adam on (x, y) for `epochs` passes in batches (whole batches only), the learning rate
    falling geometrically from lr to lr_end; each pass a random order of the points or, with
    `importance` (non-negative per-point weights), as many points drawn with replacement in
    proportion to it (the network then spends its accuracy where the drawn points are). Returns the
    mean loss of each epoch."""
    import torch

    n = (x.shape[0] // batch) * batch
    steps = epochs * (n // batch)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    history = []
    step = 0
    if importance is not None:
        # draws by inverse CDF (the cumulative sum once, in f64 on the host; uniforms from the
        # seeded generator; a sorted search): the same draws on every run, which torch's
        # multinomial sampling on the device does not give
        cdf = torch.cumsum(importance.detach().double().cpu(), 0)
        cdf = (cdf / cdf[-1]).to(x.device)
    for _ in range(epochs):
        if importance is None:
            perm = torch.randperm(x.shape[0], device="cuda", generator=gen)[:n]
        else:
            u = torch.rand(n, dtype=torch.float64, device="cuda", generator=gen)
            perm = torch.searchsorted(cdf, u).clamp_(max=x.shape[0] - 1)
        xs, ys = x[perm].contiguous(), y[perm].contiguous()
        loss.zero_()
        for b in range(n // batch):
            rate = lr * (lr_end / lr) ** (step / max(1, steps - 1))
            net.train_step(xs[b * batch:(b + 1) * batch], ys[b * batch:(b + 1) * batch], rate, loss)
            step += 1
        history.append(float(loss.item()) / n)
    return history


def train_data_parallel(net, x, y, dist, epochs, batch=16384, lr=2e-3, lr_end=2e-5, seed=0):
    """Data-parallel training over the ranks of `dist` (torch.distributed): each rank holds its own
    shard (x, y) of the labelled points (equal sizes), computes the gradient of its batch of `batch`
    points, the ranks average the gradients (one all-reduce of the parameter vector per step) and
    every rank applies the same Adam step, so their networks stay identical. Returns the mean loss
    of each epoch over all ranks."""
    import torch

    world = dist.get_world_size()
    n = (x.shape[0] // batch) * batch
    steps = epochs * (n // batch)
    gen = torch.Generator(device=x.device)
    gen.manual_seed(seed)
    history, step = [], 0
    for _ in range(epochs):
        perm = torch.randperm(x.shape[0], device=x.device, generator=gen)[:n]
        xs, ys = x[perm].contiguous(), y[perm].contiguous()
        total = torch.zeros(1, dtype=torch.float64, device=x.device)
        for b in range(n // batch):
            rate = lr * (lr_end / lr) ** (step / max(1, steps - 1))
            grad, loss = net.gradients(xs[b * batch:(b + 1) * batch], ys[b * batch:(b + 1) * batch])
            dist.all_reduce(grad)
            grad /= world
            net.apply_gradients(grad, rate)
            total += loss.double()
            step += 1
        dist.all_reduce(total)
        history.append(float(total.item()) / (n * world))
    return history


def maxima(values, weights=None, overweight=1e-3):
    """A reduced maximum for unweighting: the smallest threshold t such that the part of the
    total above it, sum(weights * max(0, values - t)), is at most `overweight` of
    sum(weights * values) (weights default to 1). Values above t become events of weight above 1
    (kept, not clipped), so the choice sets the efficiency, not the result; overweight=0 gives the
    largest value."""
    v = values.double().cpu().numpy() if hasattr(values, "cpu") else np.asarray(values, dtype=np.float64)
    w = np.ones_like(v) if weights is None else (
        weights.double().cpu().numpy() if hasattr(weights, "cpu") else np.asarray(weights, dtype=np.float64))
    keep = v > 0
    v, w = v[keep], w[keep]
    if v.size == 0:
        return 0.0
    order = np.argsort(-v)
    v, w = v[order], w[order]
    total = float((v * w).sum())
    # excess above v[i]: sum_{j < i} w_j (v_j - v_i) = (prefix of w v) - v_i (prefix of w)
    cwv = np.concatenate([[0.0], np.cumsum(w * v)[:-1]])
    cw = np.concatenate([[0.0], np.cumsum(w)[:-1]])
    excess = cwv - v * cw
    ok = np.nonzero(excess <= overweight * total)[0]
    return float(v[ok[-1]])


def chi2_against(weighted_values, weights, event_values, event_weights, edges, min_expected=5.0):
    """chi^2 and the number of bins between the normalised histogram of unweighted events (with
    their weights) and the exact weighted distribution it estimates (`weights` of every
    candidate). Each bin's variance is the one expected from the reference: the events' share
    p_b times sum(event_weights^2) / sum(event_weights)^2, plus the reference's own; neighbouring
    bins are merged until each expects at least `min_expected` events."""
    ref, _ = np.histogram(weighted_values, bins=edges, weights=weights)
    ref_var, _ = np.histogram(weighted_values, bins=edges, weights=weights ** 2)
    ev, _ = np.histogram(event_values, bins=edges, weights=event_weights)
    rt, et = ref.sum(), event_weights.sum()
    n_events = len(event_weights)
    if rt <= 0 or et <= 0:
        return float("nan"), 0
    # merge bins (in order) until each expects min_expected events
    groups, cur = [], []
    for b in range(len(ref)):
        cur.append(b)
        if ref[cur].sum() / rt * n_events >= min_expected:
            groups.append(cur)
            cur = []
    if cur:
        if groups:
            groups[-1] += cur
        else:
            groups.append(cur)
    w2 = float((event_weights ** 2).sum()) / et ** 2
    chi2 = 0.0
    for g in groups:
        p = ref[g].sum() / rt
        h = ev[g].sum() / et
        var = p * w2 + ref_var[g].sum() / rt ** 2
        if var > 0:
            chi2 += (h - p) ** 2 / var
    return float(chi2), len(groups)


def observables(p):
    """Per event: pT of the three final partons' hardest one, its rapidity, and m23 (of legs 3, 4)."""
    fin = p[:, 2:]
    pt = np.hypot(fin[..., 1], fin[..., 2])
    lead = np.argmax(pt, axis=1)
    rows = np.arange(p.shape[0])
    eta = np.arcsinh(fin[rows, lead, 3] / pt[rows, lead])
    q = fin[:, 1] + fin[:, 2]
    m23 = np.sqrt(np.maximum(0.0, q[:, 0] ** 2 - (q[:, 1:] ** 2).sum(axis=1)))
    return {"pt_lead": pt[rows, lead], "eta_lead": eta, "m23": m23}


def log_edges(v, bins=20):
    lo, hi = np.quantile(v, 0.01), np.quantile(v, 0.99)
    return np.concatenate([[-math.inf], np.linspace(lo, hi, bins - 1), [math.inf]])
