"""Benchmark: matrix-element points/s of p p -> 3 jets (leading colour, f64) on B200, and the
learned part's unweighted events/s against plain unweighting.

Workload (one step): 2^20 seeded RAMBO points at sqrt(s) = 13 TeV with jet cuts (pT > 20 GeV,
|eta| < 5, Delta R > 0.4), split over the subprocess families gg>ggg, qg>qgg, qq~>ggg and
gg>qq~g in proportion to seeded random weights; every point's |M|^2 resolved per helicity, all
colour orderings summed, in f64 (bit for bit the reference runner's f64 arithmetic).

* value: the batched device API, every family in one CUDA-graph replay (a persistent launch per
  blocks-per-SM choice the tuner made), momenta resident in HBM (168 MB of inputs: larger than
  L2, so no flush is needed); clocks: nvidia-smi samples taken inside the timed region;
* e2e: the call a generator makes, umami_matrix_element of the p p -> 3 jets UMAMI library
  (pacuda_b200/umami), one call per step over all events from pinned host momenta to |M|^2 in
  host memory, the copies in the timed region (under torchrun every rank's call on its shard,
  started together, the slowest rank's time); e2e_abi: the runner's own C ABI
  (pacman_recurrence_v1_run + _reduce_resolved per tile of 2^16 points) the same way;
* reference_gpu: the reference's own runner (recurrence_runner.cu built from its sources for
  sm_100a, unmodified) through its C ABI on the same points, per kernel kind (f64, df64, mixed),
  each in its own process; vs_reference_gpu: this library's rates over its f64 rate;
* parity: the timed outputs of the first 2048 points of every family bit for bit against the
  oracle and the reference runner's f64 outputs (the 6-leg lines check 256 points per plan);
* roofline: the dominant kernel's algorithmic flops (fixed per-op counts) per launch over its
  CUDA-event time, against this GPU's f64 FMA throughput measured in the same run; the
  algorithmic bytes (momenta in, outputs out) beside the DRAM traffic of an ncu capture;
* cpu_baseline: the CPU oracle (the runner's arithmetic restated in C++, OpenMP over all cores)
  on a bounded sample of the same families;
* precision (f64fma, mixed, mixed64, df64), precision_gg4g (with the stability check), pp4j:
  the other kinds and the 6-leg configurations (--no-precision skips them);
* surrogate: a network of log w (w = |M|^2 J) trained by this library's tensor-core kernels on
  2^22 points labelled by the f64 runner, then two-stage unweighting (network first, f64 runner
  second) against plain unweighting (f64 runner on every candidate) of the same 2^22 candidates:
  events/s of each, their ratio, efficiencies, the events' agreement with the exact weighted
  distribution (--no-surrogate skips it).
--impl reference prints the reference arm's line: the CPU oracle on the same sample per step.

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FAMILIES = ["gg>ggg", "qg>qgg", "qq~>ggg", "gg>qq~g"]
POINTS = 1 << 20
ECM = 13000.0
SEED = 20261203
TILE = 1 << 16
OVERWEIGHT = 1e-3  # reduced unweighting maxima: at most this share of the total above them


def split_points(total, seed):
    """The points per family: seeded random weights (Dirichlet), at least 1024 each."""
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.ones(len(FAMILIES)))
    n = np.maximum(1024, np.floor(w * total).astype(int))
    rem = total - n.sum()
    n[0 if n[0] + rem >= 1024 else int(np.argmax(n))] += rem
    if total < 1024 * len(FAMILIES) or n.min() < 1024:
        raise ValueError(f"{total} points do not give every family 1024")
    return [int(x) for x in n]


def workload(rank=0):
    from pacuda_b200 import phase_space, processes

    counts = split_points(POINTS, SEED)
    fams = []
    for k, (name, n) in enumerate(zip(FAMILIES, counts)):
        t = processes.template(name)
        p = phase_space.sample(len(processes.PROCESSES[name]), n, SEED + 1000 * rank + k, ecm=ECM)
        fams.append((name, t, p))
    return fams


class Clocks:
    """nvidia-smi samples (every 50 ms) during the timed region: the sampler starts before it and
    has written its first sample when `mark()` is called at the region's start; `stop()` at its
    end keeps only the samples written in between (at least the first one after the mark)."""

    def __init__(self, index=0):
        self.path = f"/tmp/bench_clocks_{os.getpid()}.csv"
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self.first = 0
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "50",
                                          "-i", str(index)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        t0 = time.time()
        while self.proc and self.proc.poll() is None and self._lines() == 0 and time.time() - t0 < 10:
            time.sleep(0.02)

    def _lines(self):
        try:
            with open(self.path) as f:
                return sum(1 for line in f if line.endswith("\n"))
        except OSError:
            return 0

    def mark(self):
        self.first = self._lines()

    def stop(self):
        if not self.proc:
            return None
        last = self._lines()
        if last <= self.first:  # a region shorter than the sampling interval: the next sample
            t0 = time.time()
            while self.proc.poll() is None and self._lines() <= self.first and time.time() - t0 < 1:
                time.sleep(0.01)
            last = self.first + 1
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], 0.0, set()
        with open(self.path) as f:
            lines = [line for line in f if line.endswith("\n")][self.first:last]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def fp64_peak(torch, lib):
    import ctypes as C

    sink = torch.zeros(1 << 16, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    blocks, threads = C.c_uint32(), C.c_uint32()
    iters = 20000
    fn = lib.pacuda_b200_measure_fp64
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
    for _ in range(2):
        fn(C.c_void_p(sink.data_ptr()), iters, C.byref(blocks), C.byref(threads), C.c_void_p(s.cuda_stream))
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn(C.c_void_p(sink.data_ptr()), iters, C.byref(blocks), C.byref(threads), C.c_void_p(s.cuda_stream))
        e1.record()
        e1.synchronize()
        flops = 2.0 * 8 * iters * blocks.value * threads.value
        best = max(best, flops / (e0.elapsed_time(e1) * 1e-3))
    return best / 1e12


def reduce_over_ranks(dist, ms, sums, squares=None, peak=None):
    """The job's step time is the slowest rank's; each family's |M|^2 total and sum of squares
    add up over the ranks, its largest |M|^2 is the largest of any rank (the points are sharded:
    the only exchange is this reduction of small tensors)."""
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=sums.device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total = sums.clone()
    dist.all_reduce(total)
    out = [float(t.item()), total]
    if squares is not None:
        sq = squares.clone()
        dist.all_reduce(sq)
        mx = peak.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        out += [sq, mx]
    return tuple(out)


def precision_line(torch, B, fams, ext, ref_out, steps, warmup, kind="mixed"):
    """The same points in another kernel kind (mixed: f32 currents, df64 denominators and
    amplitudes): its points/s on the device, and each point's relative error in its helicity sum
    against the f64 run."""
    plans, outs = [], []
    for (name, t, p), e in zip(fams, ext):
        plans.append(B.Plan(t, kind))
        outs.append(torch.empty(p.shape[0] * t.outputs, dtype=torch.float64, device="cuda"))
    batch = B.Batch(plans, ext, outs)
    batch.tune()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        batch.capture(stream)
    for _ in range(warmup):
        batch.run(stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        batch.run(stream)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    rel = []
    for (name, t, p), o, r in zip(fams, outs, ref_out):
        x = o.view(p.shape[0], t.outputs).sum(dim=1)
        y = r.view(p.shape[0], t.outputs).sum(dim=1)
        rel.append(((x - y).abs() / y.abs().clamp_min(1e-300)).cpu().numpy())
    rel = np.concatenate(rel)
    n = rel.size
    return {"kind": kind, "value": n / (ms * 1e-3), "unit": "points/s", "ms_per_step": ms,
            "rel_error_vs_f64": {"median": float(np.median(rel)), "q999": float(np.quantile(rel, 0.999)),
                                 "max": float(rel.max()), "frac_le_1e-10": float((rel <= 1e-10).mean())},
            "lanes_per_point": {nm: batch.lanes_per_point(k) for k, (nm, _, _) in enumerate(fams)},
            "blocks_per_sm": {nm: batch.plan_blocks_per_sm(k) for k, (nm, _, _) in enumerate(fams)}}


def surrogate_line(torch, families=None, train_points=1 << 22, candidates=1 << 22, epochs=300, batch=16384, steps=3,
                   alpha=0.5, lr=2e-3, overweight=None):
    """The learned part: a surrogate of the weight w = |M|^2 J of p p -> 3 jets candidates (or of
    the p p -> 4 jets families with families=processes.PP4J: eight unit-cube numbers; one
    network, the unit-cube numbers and a subprocess one-hot as inputs, 4 x 256 SiLU, BF16
    tensor-core products, trained on the standardized log w), trained by this library's kernels
    on `train_points` points inside the cuts labelled by the f64 recurrence (a training stream of
    candidates), then two-stage unweighting of `candidates` seeded candidates (split over the
    families as the benchmark's points are) against plain unweighting of the same candidates with
    the f64 runner alone. Reports the training, the surrogate's relative errors on held-out
    points, both pipelines' efficiencies and unweighted events/s (device time, CUDA events around
    each step, the host's reads of the kept counts inside), the events' agreement with the exact
    weighted distribution (chi^2 per bin of three observables), and the fused first-stage
    kernel's tensor throughput."""
    from pacuda_b200 import surrogate as S
    from pacuda_b200 import unweight as UW

    fams = list(families or FAMILIES)
    final_state = UW.final_state_of(fams[0])
    counts = split_points(candidates, SEED)
    # a training stream of candidates: about 28 % of 2 -> 3 candidates pass the cuts, 5.6 % of 2 -> 4
    stream, share = (4, 0.4) if final_state == 3 else (24, 0.1)
    train_counts = split_points(stream * train_points, SEED + 1)
    pl = UW.Pipeline(families=fams, capacity=int(share * max(max(counts), max(train_counts))) + 4096)
    res = {"workload": f"pp>{final_state}j LC: {', '.join(fams)}; 13 TeV, pT>20 GeV, |eta|<5, dR>0.4; network "
                       f"4 x 256 SiLU, inputs {pl.numbers} + {len(fams)} one-hot; {train_points} labelled points, "
                       f"{candidates} candidates unweighted", "candidates_per_family": dict(zip(fams, counts))}
    # labels: the f64 recurrence on the candidates of a training stream (from 2^40 on) inside the cuts
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    data = [pl.labelled(k, 1 << 40, c) for k, c in enumerate(train_counts)]
    e1.record()
    e1.synchronize()
    label_ms = e0.elapsed_time(e1)
    # the runner's launch choices timed on every family's points (the plain pipeline's load)
    listed = pl.candidates(1 << 40, train_counts)
    pl.exact([f.cand for f in pl.fams], [min(a, max(1, int(0.28 * c))) for a, c in zip(listed, counts)])
    pl.tune()
    x = torch.cat([d[0] for d in data])
    w = torch.cat([d[1] * d[2] for d in data])
    fam_of = torch.cat([torch.full((d[0].shape[0],), k, dtype=torch.int64, device="cuda") for k, d in enumerate(data)])
    labelled = int(x.shape[0])
    pick = torch.randperm(labelled, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
    n_hold = 1 << 16
    hold, train = pick[:n_hold], pick[n_hold:n_hold + train_points]
    logw = w.log()
    mu, sigma = float(logw[train].mean()), float(logw[train].std())
    y = ((logw - mu) / sigma).float()
    tx, ty = x[train].contiguous(), y[train].contiguous()
    net = S.Network(pl.inputs, max_batch=batch, seed=7)
    e0.record()
    # training points drawn in proportion to w^alpha: the accuracy goes where the events come from
    imp = (logw[train] - logw[train].max()).mul(alpha).exp().float() if alpha else None
    hist = UW.train(net, tx, ty, epochs=epochs, batch=batch, lr=lr, lr_end=1e-5, importance=imp)
    e1.record()
    e1.synchronize()
    train_ms = e0.elapsed_time(e1)
    if net.error():
        raise RuntimeError(f"surrogate kernels reported error {net.error()}")
    sv_hold = pl.surrogate_values(net, x[hold], mu, sigma)
    rel = (sv_hold / w[hold] - 1.0).abs().cpu().numpy()
    res["training"] = {"labelled_points": labelled, "train_points": int(tx.shape[0]), "epochs": epochs,
                       "importance": f"points drawn in proportion to w^{alpha}" if alpha else "uniform", "lr": lr,
                       "batch": batch, "loss_per_epoch": [round(v, 6) for v in hist], "label_ms": label_ms,
                       "train_ms": train_ms, "train_steps": epochs * (tx.shape[0] // batch),
                       "sigma_log_w": sigma, "held_out_points": n_hold,
                       "surrogate_rel_error": {q: float(np.quantile(rel, float(q))) for q in ("0.5", "0.9", "0.99")},
                       "log_error_rms": float((sv_hold.log() - w[hold].log()).pow(2).mean().sqrt())}
    # maxima per family from its labelled points (reduced: at most `overweight` of the total above)
    overweight = OVERWEIGHT if overweight is None else overweight
    maxima = []
    sv_all = pl.surrogate_values(net, x, mu, sigma)
    for k in range(len(fams)):
        sel = fam_of == k
        wk, sk = w[sel], sv_all[sel]
        maxima.append((UW.maxima(wk, overweight=overweight), UW.maxima(sk, overweight=overweight),
                       UW.maxima(wk / sk, sk, overweight=overweight)))
    res["maxima"] = {"overweight_share": overweight, "per_family": {nm: {"w_max": m[0], "s_max": m[1], "r_max": m[2]}
                                                                    for nm, m in zip(fams, maxima)}}
    del data, x, w, tx, ty, sv_all, fam_of
    # the two pipelines on the same candidates (stream from 0), timed per step
    first = 0

    w_maxes = [m[0] for m in maxima]
    s_maxes = [m[1] for m in maxima]
    r_maxes = [m[2] for m in maxima]

    def run(kind):
        if kind == "plain":
            events, exact = pl.plain(first, counts, w_maxes)
        else:
            events, exact = pl.two_stage(net, first, counts, mu, sigma, s_maxes, r_maxes)
        return events, exact

    lines = {}
    for kind in ("plain", "two_stage"):
        run(kind)  # warm-up (and the batch plans' first launches)
        e0.record()
        for _ in range(steps):
            events, exact = run(kind)
            counts_dev = torch.stack([e.count() for e in events])  # the step's kept events, on the device
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        per_family = [int(v) for v in counts_dev.tolist()]
        kept = sum(per_family)
        compact = [e.compact() for e in events]
        lines[kind] = {"ms_per_step": ms, "events": kept, "exact_evaluations": exact,
                       "events_per_s": kept / (ms * 1e-3), "candidates_per_s": candidates / (ms * 1e-3),
                       "efficiency_per_exact": kept / max(1, exact), "efficiency_per_candidate": kept / candidates,
                       "overweight_events": int(sum(int((w > 1).sum()) for _, w in compact)),
                       "events_per_family": dict(zip(fams, per_family))}
        lines[kind]["_events"] = compact
    res["plain"] = {k: v for k, v in lines["plain"].items() if not k.startswith("_")}
    res["two_stage"] = {k: v for k, v in lines["two_stage"].items() if not k.startswith("_")}
    res["events_per_s_ratio"] = lines["two_stage"]["events_per_s"] / lines["plain"]["events_per_s"]
    res["exact_error"] = ("0: the kept events' |M|^2 and weights come from the f64 runner (bit for bit the reference "
                          "runner's f64 arithmetic); the surrogate only decides which candidates are evaluated")
    # unbiasedness: each sample's histograms against the exact weighted distribution of all candidates
    from oracle import unweight_oracle as UO

    chi, xsec = {}, {}
    for k, name in enumerate(fams):
        seed = pl.family_seed(k)
        idx_all = pl.passing(k, first, counts[k])
        _, ma, ja, _ = pl.labelled(k, first, counts[k])
        wa = (ma * ja).cpu().numpy()
        # the total each sample estimates: sum of weights x its maxima, against the exact sum of w
        w_max, s_max, r_max = maxima[k]
        exact = float(wa.sum())
        for kind, scale in (("plain", w_max), ("two_stage", s_max * r_max)):
            wts = lines[kind]["_events"][k][1].double().cpu().numpy()
            est = float(wts.sum()) * scale
            err = float(np.sqrt((wts ** 2).sum())) * scale
            xsec.setdefault(kind, {})[name] = {"ratio_to_exact": est / exact, "stat_error": err / exact,
                                               "events": int(len(wts))}

        def moms(index):
            u = UO.uniforms(seed, index.cpu().numpy().astype(np.uint64), final_state)
            return UO.momenta(u, ECM, final_state)[0]

        ref = UW.observables(moms(idx_all))
        for kind in ("plain", "two_stage"):
            idx, wts = lines[kind]["_events"][k]
            ev = UW.observables(moms(idx))
            for obs in ref:
                edges = UW.log_edges(ref[obs], 16)
                c2, bins = UW.chi2_against(ref[obs], wa, ev[obs], wts.cpu().numpy(), edges)
                chi.setdefault(kind, {}).setdefault(name, {})[obs] = round(c2 / max(1, bins), 3)
    res["chi2_per_bin_vs_exact"] = chi
    res["total_vs_exact"] = xsec
    # the fused first stage alone: tensor throughput (algorithmic flops of the network per candidate)
    flops = 2 * (64 * 256 + 3 * 256 * 256 + 256)
    k0 = int(np.argmax(counts))
    w_max, s_max, r_max = maxima[k0]
    cand = pl.passing(k0, first, counts[k0]).clone()
    f0 = pl.fams[k0]
    e0.record()
    for _ in range(steps):
        pl.counters.zero_()
        UW._check(UW._lib().pacuda_uw_stage1(net.handle, pl.family_seed(k0), UW._ptr(cand), cand.numel(),
                                             pl.final_state, k0, mu, sigma, s_max, UW._ptr(f0.kept),
                                             UW._ptr(f0.kept_s), pl.capacity, UW._ptr(pl.counters), UW._stream()),
                  "stage 1")
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    peak, source = bf16_peak()
    tf = cand.numel() * flops / (ms * 1e-3) / 1e12
    res["stage1_kernel"] = {"candidates_inside_cuts": int(cand.numel()), "ms": ms,
                            "candidates_per_s": cand.numel() / (ms * 1e-3), "flops_per_candidate": flops,
                            "tflops": tf, "roofline": {"bound": "tensor", "achieved": tf, "peak": peak,
                                                       "unit": "TFLOP/s", "frac": tf / peak, "peak_source": source}}
    return res


def surrogate_kernels(torch, count=1 << 21, steps=5):
    """The surrogate's kernels alone on a random network (a small, self-contained case for
    profiling): the fused inference kernel on `count` points of given inputs, and the fused first
    stage on `count` candidates; time per launch and tensor throughput (algorithmic flops of the
    network per point: 2 (64 x 256 + 3 x 256 x 256 + 256))."""
    from pacuda_b200 import surrogate as S
    from pacuda_b200 import unweight as UW

    flops = 2 * (64 * 256 + 3 * 256 * 256 + 256)
    net = S.Network(9, max_batch=1024, seed=3)
    x = torch.rand(count, 9, device="cuda")
    out = torch.empty(count, device="cuda")
    pl = UW.Pipeline(families=FAMILIES[:1], capacity=count)
    cand = torch.arange(count, dtype=torch.int64, device="cuda")  # a candidate list (the weights do not matter)
    res = {}
    for what, blocks in (("forward", 2), ("stage1", 2), ("forward_1_block_per_sm", 1), ("stage1_1_block_per_sm", 1)):
        S.set_inference_blocks(blocks)
        def launch():
            if what.startswith("forward"):
                net.forward(x, out)
            else:
                pl.counters.zero_()
                UW._check(UW._lib().pacuda_uw_stage1(net.handle, 11, UW._ptr(cand), count, 3, 0, -3.0, 1.0, 1e30,
                                                     UW._ptr(pl.fams[0].kept), UW._ptr(pl.fams[0].kept_s),
                                                     pl.capacity, UW._ptr(pl.counters), UW._stream()), "stage 1")
        for _ in range(2):
            launch()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            launch()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        res[what] = {"points": count, "ms": ms, "points_per_s": count / (ms * 1e-3),
                     "tflops": count * flops / (ms * 1e-3) / 1e12, "blocks_per_sm": blocks}
    S.set_inference_blocks(2)
    # training steps (forward, backward and weight-gradient products, gradient reduction, Adam):
    # three products per layer per point, 3 x the inference flops
    batch = 16384
    tnet = S.Network(9, max_batch=batch, seed=5)
    tx = torch.rand(batch, 9, device="cuda")
    ty = torch.randn(batch, device="cuda")
    for _ in range(3):
        tnet.train_step(tx, ty, 1e-4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(4 * steps):
        tnet.train_step(tx, ty, 1e-4)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / (4 * steps)
    res["train_step"] = {"batch": batch, "ms": ms, "launches": S.last_launches(),
                         "tflops": 3 * batch * flops / (ms * 1e-3) / 1e12}
    if net.error() or tnet.error():
        raise RuntimeError(f"surrogate kernels reported error {net.error() or tnet.error()}")
    return res


def listing_case(torch, steps=5):
    """The candidate listing alone (a small, self-contained case for profiling): every family's
    candidates of one step listed inside the cuts, the p p -> 3 jets step's 2^22 candidates
    (1 + steps launches) and then the p p -> 4 jets step's 2^25 (1 + steps); time per call with
    its count read."""
    from pacuda_b200 import processes
    from pacuda_b200 import unweight as UW

    res = {}
    for name, fams, cand in (("pp3j", processes.PP3J, 1 << 22), ("pp4j", processes.PP4J, 1 << 25)):
        counts = split_points(cand, SEED)
        pl = UW.Pipeline(families=list(fams), capacity=int(0.4 * max(counts)) + 4096)
        n = pl.candidates(0, counts)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            pl.candidates(0, counts)
        e1.record()
        e1.synchronize()
        res[name] = {"candidates": cand, "ms": e0.elapsed_time(e1) / steps, "listed": n}
        del pl
    return res


def oracle_parity(cases):
    """Bitwise parity of device outputs with the oracle: cases (label, template, point-major
    momenta, device outputs [point][helicity])."""
    from oracle import oracle as O

    pairs = []
    for label, t, p, o in cases:
        _, want = O.evaluate(t, p, kernel=1)
        pairs.append((label, o.cpu().numpy(), want))
    return parity(pairs)


def six_gluon_line(torch, B, points=1 << 20, steps=3, warmup=2, check=256):
    """The precision configuration: g g -> 4 g, leading colour (60 orderings x 64 helicities, as
    the plan parts that fit 64-bit words), `points` seeded RAMBO points at 13 TeV with the loosened
    cuts pT > 5 GeV and Delta R > 0.1; points/s in f64 and in mixed precision, and the histogram of
    each point's relative error in |M|^2 (mixed against f64). The f64 outputs of the first `check`
    points of every plan are compared bit for bit with the oracle's."""
    from pacuda_b200 import phase_space, processes

    parts = processes.parts("gg>gggg")
    p = phase_space.sample(6, points, SEED + 6, ecm=ECM, pt_min=5.0, dr_min=0.1)
    ext = torch.tensor(phase_space.source_major(p), dtype=torch.float64, device="cuda")
    res, totals = {"workload": f"gg>gggg LC: 60 orderings x 64 helicities as {len(parts)} plans, {points} points, "
                               "13 TeV, pT>5 GeV, |eta|<5, dR>0.1"}, {}
    for kind in ("f64", "mixed"):
        plans = [B.Plan(t, kind) for t in parts]
        outs = [torch.empty(points * t.outputs, dtype=torch.float64, device="cuda") for t in parts]
        batch = B.Batch(plans, [ext] * len(parts), outs)
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            batch.tune(stream)
            batch.capture(stream)
        for _ in range(warmup):
            batch.run(stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            batch.run(stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        flops = sum(pl.flops for pl in plans) * points
        res[kind] = {"value": points / (ms * 1e-3), "unit": "points/s", "ms_per_step": ms,
                     "tflops": flops / (ms * 1e-3) / 1e12, "launches_per_step": batch.launches,
                     "lanes_per_point": [batch.lanes_per_point(k) for k in range(len(plans))],
                     "blocks_per_sm": [batch.plan_blocks_per_sm(k) for k in range(len(plans))]}
        totals[kind] = sum(o.view(points, t.outputs).sum(dim=1) for o, t in zip(outs, parts))
        if kind == "f64":
            res["parity"] = oracle_parity([(f"gg>gggg part {k}", t, p[:check], o.view(points, t.outputs)[:check])
                                           for k, (t, o) in enumerate(zip(parts, outs))])
        del batch, outs
    rel = ((totals["mixed"] - totals["f64"]).abs() / totals["f64"].abs().clamp_min(1e-300)).cpu().numpy()
    edges = [0.0] + [10.0 ** e for e in range(-16, 1)] + [np.inf]
    hist, _ = np.histogram(rel, bins=edges)
    res["mixed"]["rel_error_vs_f64"] = {
        "median": float(np.median(rel)), "q999": float(np.quantile(rel, 0.999)), "max": float(rel.max()),
        "frac_le_1e-10": float((rel <= 1e-10).mean()),
        "histogram": {"edges_log10": list(range(-16, 1)), "counts": [int(c) for c in hist]}}
    res["stability"] = stability_line(torch, parts, ext, totals["f64"], points, steps, warmup)
    return res


def stability_line(torch, templates, ext, want, points, steps, warmup, tols=(1e-10, 1e-6)):
    """The mixed kernel with the rotated-momentum stability check (pacuda_b200/stability.py):
    per tolerance, the whole pipeline's points/s (two mixed evaluations, the check, the f64
    evaluation of the points that fail it), the fraction of points sent back to f64, and the
    relative error of the result's |M|^2 against f64."""
    from pacuda_b200 import stability

    lines = []
    for tol in tols:
        s = stability.StableMixed(templates, points, tol)
        for _ in range(warmup):
            s.run(ext)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            outs, m = s.run(ext)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        total = sum(o.view(points, t.outputs).sum(dim=1) for o, t in zip(outs, templates))
        rel = ((total - want).abs() / want.abs().clamp_min(1e-300)).cpu().numpy()
        lines.append({"tol": tol, "value": points / (ms * 1e-3), "unit": "points/s", "ms_per_step": ms,
                      "fraction_to_f64": m / points,
                      "rel_error_vs_f64": {"median": float(np.median(rel)), "q999": float(np.quantile(rel, 0.999)),
                                           "max": float(rel.max()), "frac_le_1e-10": float((rel <= 1e-10).mean())}})
        del s, outs
    return lines


def pp4j_line(torch, B, points=1 << 22, steps=3, warmup=2, check=256):
    """p p -> 4 jets, every massless family the intrinsic ops express (gg>gggg as its plan parts,
    qg>qggg, qq~>gggg, gg>qq~gg), `points` seeded RAMBO points at 13 TeV with pT > 20 GeV and
    Delta R > 0.4 split over the families by seeded random weights, all in one persistent launch:
    points/s in f64 and in mixed precision, with the mixed kernel's relative error in |M|^2; the f64
    outputs of the first `check` points of every plan bit for bit against the oracle's."""
    from pacuda_b200 import phase_space, processes

    names = processes.PP4J
    rng = np.random.default_rng(SEED + 4)
    w = rng.dirichlet(np.ones(len(names)))
    counts = np.maximum(1024, np.floor(w * points).astype(int))
    counts[int(np.argmax(counts))] += points - counts.sum()
    fams, moms = [], {}
    for k, (name, n) in enumerate(zip(names, counts)):
        p = phase_space.sample(6, int(n), SEED + 40 + k, ecm=ECM)
        moms[name] = p[:check]
        e = torch.tensor(phase_space.source_major(p), dtype=torch.float64, device="cuda")
        for t in processes.parts(name):
            fams.append((name, t, int(n), e))
    res, totals = {"workload": f"pp>4j LC f64: {', '.join(names)}; {points} points, 13 TeV, pT>20 GeV, |eta|<5, "
                               f"dR>0.4; {len(fams)} plans in one launch",
                   "points_per_family": {nm: int(c) for nm, c in zip(names, counts)}}, {}
    for kind in ("f64", "mixed"):
        plans = [B.Plan(t, kind) for _, t, _, _ in fams]
        outs = [torch.empty(n * t.outputs, dtype=torch.float64, device="cuda") for _, t, n, _ in fams]
        batch = B.Batch(plans, [e for *_, e in fams], outs)
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            batch.tune(stream)
            batch.capture(stream)
        for _ in range(warmup):
            batch.run(stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            batch.run(stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        flops = sum(pl.flops * n for pl, (_, _, n, _) in zip(plans, fams))
        res[kind] = {"value": points / (ms * 1e-3), "unit": "points/s", "ms_per_step": ms,
                     "tflops": flops / (ms * 1e-3) / 1e12, "launches_per_step": batch.launches,
                     "blocks_per_sm": [batch.plan_blocks_per_sm(k) for k in range(len(plans))]}
        per_family = {}
        for (name, t, n, _), o in zip(fams, outs):
            x = o.view(n, t.outputs).sum(dim=1)
            per_family[name] = per_family[name] + x if name in per_family else x
        totals[kind] = torch.cat([per_family[nm] for nm in names])
        if kind == "f64":
            # the oracle on the first `check` points of every plan: the parity check, and timed, the
            # CPU recurrence's rate (each family's plans on its sample, weighted by its share)
            from oracle import oracle as O

            pairs, secs = [], {}
            for k, ((name, t, n, _), o) in enumerate(zip(fams, outs)):
                t0 = time.perf_counter()
                _, want = O.evaluate(t, moms[name][:check], kernel=1)
                secs[name] = secs.get(name, 0.0) + time.perf_counter() - t0
                pairs.append((f"{name} plan {k}", o.view(n, t.outputs)[:check].cpu().numpy(), want))
            res["parity"] = parity(pairs)
            total_s = sum(secs[nm] * int(c) / min(check, int(c)) for nm, c in zip(names, counts))
            res["cpu_baseline"] = {"value": points / total_s, "unit": "points/s", "cores": os.cpu_count(),
                                   "kind": "port",
                                   "sample": f"first {check} points of each family through all its plans, OpenMP "
                                             f"over all host cores, rates weighted by the families' shares"}
        del batch, outs
    rel = ((totals["mixed"] - totals["f64"]).abs() / totals["f64"].abs().clamp_min(1e-300)).cpu().numpy()
    res["mixed"]["rel_error_vs_f64"] = {"median": float(np.median(rel)), "q999": float(np.quantile(rel, 0.999)),
                                        "max": float(rel.max())}
    res["f64_vs_cpu"] = res["f64"]["value"] / res["cpu_baseline"]["value"]
    return res


def dram_bytes_per_point():
    """DRAM bytes per point of the batch kernel, from the committed ncu summary (one capture of the
    same family mix), or None."""
    import re

    try:
        text = open(os.path.join(ROOT, "profiles", "launches_pp3j_bench.md")).read()
    except OSError:
        return None
    m = re.search(r"^dram_bytes_per_point = ([0-9.]+)", text, re.M)
    return float(m.group(1)) if m else None


def hbm_peak():
    """(HBM GB/s of this pool's B200s, its source): MEASURED_PEAKS.json's copy bandwidth, else the
    earlier measurement on this pool (6650)."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback (no MEASURED_PEAKS.json)"


def bf16_peak():
    """(dense BF16 TFLOP/s of this pool's B200s, its source): the burst figure of
    MEASURED_PEAKS.json, else the earlier measurement on this pool (1590)."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]), "MEASURED_PEAKS.json"
    except (OSError, ValueError, KeyError):
        return 1590.0, "fallback (no MEASURED_PEAKS.json)"


def cpu_baseline(fams, sample=2048, keep=None):
    """The oracle on the first `sample` points of each family, all host cores; points/s of the
    family mix (each family's rate weighted by its share of the workload). With a dict `keep`,
    each family's oracle outputs [point][helicity] are kept there by name (the parity check)."""
    from oracle import oracle as O

    counts = [p.shape[0] for _, _, p in fams]
    total = sum(counts)
    secs = 0.0
    for (name, t, p), n in zip(fams, counts):
        m = min(sample, n)
        t0 = time.perf_counter()
        _, out = O.evaluate(t, p[:m], kernel=1)
        dt = time.perf_counter() - t0
        secs += dt * (n / m)  # the time of the family's full share at this rate
        if keep is not None:
            keep[name] = out
    return {"value": total / secs, "unit": "points/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"first {sample} points of each family (of {total}), OpenMP over all host cores, "
                      f"rates weighted by the families' shares"}


def same_bits(a, b):
    a, b = np.ascontiguousarray(a, dtype=np.float64), np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and bool(np.all((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))))


def parity(pairs):
    """Bitwise comparison of (label, got, want) arrays: values checked and values that differ."""
    checked, bad, where = 0, 0, []
    for label, got, want in pairs:
        got = np.ascontiguousarray(got, dtype=np.float64)
        want = np.ascontiguousarray(want, dtype=np.float64)
        checked += want.size
        if got.shape != want.shape:
            bad += want.size
            where.append(label)
            continue
        diff = ~((got.view(np.uint64) == want.view(np.uint64)) | (np.isnan(got) & np.isnan(want)))
        if diff.any():
            bad += int(diff.sum())
            where.append(label)
    return {"values_checked": checked, "mismatches": bad, "differing": where}


def e2e_abi(fams, steps, warmup, lib=None, kernel="f64", events=None):
    """points/s through the C ABI: per tile one run (forms on the device, amplitudes kept) and one
    resolved reduction, from pinned host buffers. With `events` (two CUDA events), also the rate
    between them recorded on the default stream around the timed steps."""
    import ctypes as C

    from pacuda_b200 import abi, phase_space
    from pacuda_b200.runner import Runner

    r = Runner(lib)
    assert r.configure(kernel) == 0
    jobs, h2d, d2h = [], 0, 0
    for name, t, p in fams:
        n = p.shape[0]
        for s in range(0, n, TILE):
            m = min(TILE, n - s)
            ext = phase_space.source_major(p[s:s + m])
            pin = r.lib.pacman_recurrence_v1_host_alloc(ext.nbytes)
            hext = np.ctypeslib.as_array((C.c_double * ext.size).from_address(pin))
            hext[:] = ext
            args = t.call(hext, m, stride=TILE)
            outp = r.lib.pacman_recurrence_v1_host_alloc(8 * m * t.outputs)
            out = np.ctypeslib.as_array((C.c_double * (m * t.outputs)).from_address(outp))
            red, keep = abi.reduce_resolved_args(t.planes, t.weights, t.offsets, out, m, 1, t.outputs, abi.OUTPUT_ZERO)
            jobs.append((args, red, keep, out, name))
            h2d += ext.nbytes
            d2h += out.nbytes

    def step():
        for args, red, keep, out, _ in jobs:
            if r.run(args) != 0 or r.reduce_resolved(red) != 0:
                raise RuntimeError("runner call failed")

    for _ in range(warmup):
        step()
    if events:
        events[0].record()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    if events:
        events[1].record()
        events[1].synchronize()
    dt = (time.perf_counter() - t0) / steps
    total = sum(p.shape[0] for _, _, p in fams)
    res = {"value": total / dt, "unit": "points/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "tile": TILE, "calls_per_step": 2 * len(jobs), "steps": steps}
    if events:
        ms = events[0].elapsed_time(events[1]) / steps
        res["device_value"] = total / (ms * 1e-3)
        res["device_ms_per_step"] = ms
    return res, [(j[4], j[3]) for j in jobs]  # (family, outputs) per tile, the families' tiles in order


REF_LIB = os.path.join(ROOT, "oracle", "_ref", "librecurrence.so")


def reference_gpu_worker(kind, steps, warmup, keep_path):
    """In its own process (a runner takes its kernel kind once, before its first run): the
    reference's runner built from its own sources for sm_100a (oracle/_ref/librecurrence.so,
    recurrence_runner.cu unmodified) through its stock C ABI, the same points as this benchmark,
    per tile of 2^16 points one run (forms on the device, amplitudes kept) and one resolved
    reduction from pinned host buffers. Prints one JSON line: points/s from CUDA events on the
    default stream (which the reference runner's synchronous copies and launches use) and from
    the host clock; with `keep_path`, the first 2048 outputs of each family go there."""
    import torch

    fams = workload(0)
    torch.cuda.init()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    line, outs = e2e_abi(fams, steps, warmup, lib=REF_LIB, kernel=kind, events=(e0, e1))
    line["kernel"] = kind
    if keep_path:
        first = {}
        tmpl = {name: (t, p) for name, t, p in fams}
        for name, o in outs:  # a family's first tile holds its first points
            if name not in first:
                t, p = tmpl[name]
                first[name] = np.array(o[: min(2048, p.shape[0]) * t.outputs]).reshape(-1, t.outputs)
        np.savez(keep_path, **first)
    print(json.dumps(line))


def reference_gpu(kinds=("f64", "df64", "mixed"), steps=2, warmup=1, keep_path=None):
    """The reference runner's rate per kernel kind (one worker process each; see
    reference_gpu_worker). None when the reference runner is not built."""
    if not os.path.exists(REF_LIB):
        return None
    res = {}
    for kind in kinds:
        cmd = [sys.executable, os.path.abspath(__file__), "--reference-gpu-kind", kind, "--steps", str(steps),
               "--warmup", str(warmup), "--points", str(POINTS)] + (["--keep", keep_path] if keep_path and kind == "f64" else [])
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        if p.returncode != 0:
            res[kind] = {"error": (p.stderr or p.stdout).strip().splitlines()[-1:]}
            continue
        res[kind] = json.loads(p.stdout.strip().splitlines()[-1])
    return res


def e2e_umami(fams, steps, warmup, outs=None, sync=None):
    """points/s through the UMAMI call a generator makes (umami_matrix_element, the reference's
    production entry point): every step one call over all events, from pinned host momenta (copied
    to the device inside the call) to |M|^2 in host memory (copied back inside the call). `sync`,
    when given, is called right before the timed calls (the ranks' barrier); the line's `seconds`
    is this process's time per step."""
    import ctypes as C
    import tempfile

    from pacuda_b200 import pacuda_file
    from pacuda_b200.runner import Runner
    from pacuda_b200.umami import build as ub

    lib = C.CDLL(ub.pp3j_library())
    lib.umami_initialize.argtypes = [C.POINTER(C.c_void_p), C.c_char_p]
    lib.umami_matrix_element.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                                         C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.c_size_t,
                                         C.POINTER(C.c_int), C.POINTER(C.c_void_p)]
    lib.umami_free.argtypes = [C.c_void_p]
    art = os.path.join(tempfile.mkdtemp(prefix="pp3j_"), "artifact")
    os.makedirs(art)
    pacuda_file.write(pacuda_file.from_processes(ub.PP3J, kernel=1, reference_points=0), art + ".pacuda")
    h = C.c_void_p()
    if lib.umami_initialize(C.byref(h), art.encode()) != 0:
        raise RuntimeError("umami_initialize failed")
    r = Runner(None)
    n = sum(p.shape[0] for _, _, p in fams)
    legs = 5

    def pinned(count, ctype):
        ptr = r.lib.pacman_recurrence_v1_host_alloc(count * C.sizeof(ctype))
        return ptr, np.ctypeslib.as_array((ctype * count).from_address(ptr))

    mom_p, mom = pinned(legs * 4 * n, C.c_double)
    fl_p, flavour = pinned(n, C.c_int)
    me_p, me = pinned(n, C.c_double)
    rows = mom.reshape(legs * 4, n)
    start = 0
    for name, _, p in fams:
        m = p.shape[0]
        for k in range(4):
            for leg in range(legs):
                rows[legs * k + leg, start:start + m] = p[:, leg, k]
        flavour[start:start + m] = ub.PP3J.index(name)
        start += m
    keys_in = (C.c_int * 2)(0, 2)
    ptr_in = (C.c_void_p * 2)(mom_p, fl_p)
    keys_out = (C.c_int * 1)(0)
    ptr_out = (C.c_void_p * 1)(me_p)

    def step():
        if lib.umami_matrix_element(h, n, n, 0, 2, keys_in, ptr_in, 1, keys_out, ptr_out) != 0:
            raise RuntimeError("umami_matrix_element failed")

    for _ in range(warmup):
        step()
    if sync:
        sync()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = (time.perf_counter() - t0) / steps
    # the helicity sums agree with the device-resident run's outputs (a sanity check)
    if outs is not None:
        start = 0
        for (name, t, p), o in zip(fams, outs):
            m = p.shape[0]
            num, den = t.meta["group_factor"]
            want = (o.reshape(m, t.outputs)[:64] * float(num) / float(den)).sum(axis=1)
            if not np.allclose(me[start:start + min(64, m)], want, rtol=1e-12, atol=0):
                raise RuntimeError(f"{name}: UMAMI |M|^2 differs from the batched run")
            start += m
    lib.umami_free(h)
    for ptr in (mom_p, fl_p, me_p):
        r.lib.pacman_recurrence_v1_host_free(ptr)
    return {"value": n / dt, "unit": "points/s", "h2d_bytes_per_step": n * legs * 4 * 8 + n * 24,
            "d2h_bytes_per_step": n * 8, "api": "umami_matrix_element (helicity sum, one call per step)",
            "calls_per_step": 1, "seconds": dt}


def main():
    global POINTS, FAMILIES
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--family", default=None, help="one subprocess family alone (profiling cases)")
    ap.add_argument("--points", type=int, default=POINTS, help="points per GPU")
    ap.add_argument("--no-tune", action="store_true", help="keep the default points per warp")
    ap.add_argument("--lanes-per-point", type=int, default=0)
    ap.add_argument("--no-precision", action="store_true", help="skip the mixed-precision lines")
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="1, 2, 3, 4, 5, 8 or 16 (with --no-tune or --lanes-per-point)")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip timing the reference's own GPU runner")
    ap.add_argument("--no-graph", action="store_true", help="plain launches instead of a CUDA-graph replay "
                                                             "(profiling cases: ncu does not replay the graph)")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate and two-stage unweighting line")
    ap.add_argument("--surrogate-only", action="store_true", help="only the surrogate line (development runs)")
    ap.add_argument("--surrogate-args", default="", help="key=value,... for the surrogate line (development runs)")
    ap.add_argument("--surrogate-kernels", action="store_true", help="only the surrogate kernels on a random network "
                                                                      "(the profiling case)")
    ap.add_argument("--listing", action="store_true", help="only the candidate listing of the two learned-part "
                                                            "workloads (the profiling case)")
    ap.add_argument("--reference-gpu-kind", default=None, help=argparse.SUPPRESS)  # the worker of reference_gpu()
    ap.add_argument("--keep", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    POINTS = args.points
    if args.reference_gpu_kind:
        reference_gpu_worker(args.reference_gpu_kind, args.steps, args.warmup, args.keep)
        return
    if args.family:
        FAMILIES = [args.family]
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    metric = "matrix-element points/s (p p -> 3 jets, LC, f64)"
    config = {"workload": "pp>3j LC f64: " + ", ".join(FAMILIES), "points_per_gpu": POINTS,
              "sqrt_s_gev": ECM, "cuts": "pT>20 GeV, |eta|<5, dR>0.4", "seed": SEED,
              "l2": f"inputs {POINTS * 160 / 1e6:.0f} MB per GPU" + (" > 126 MB L2 (no flush)" if POINTS * 160 > 126e6 else ""),
              "parallelism": f"points sharded, {world} GPU(s)"}

    if args.impl == "reference":
        # the reference's path on the host: its arithmetic restated (the oracle, f64), all cores
        if rank != 0:
            return
        fams = workload(0)
        for _ in range(max(0, args.warmup)):
            cpu_baseline(fams, sample=2048)
        vals = []
        for _ in range(args.steps):
            vals.append(cpu_baseline(fams, sample=2048)["value"])
        v = statistics.median(vals)
        cb = {"value": v, "unit": "points/s", "cores": os.cpu_count(), "kind": "port",
              "sample": "first 2048 points of each family per step (as the GPU arm's cpu_baseline), OpenMP over "
                        "all host cores, rates weighted by the families' shares"}
        print(json.dumps({"impl": "reference", "metric": metric, "value": v, "unit": "points/s", "n_gpus": 1,
                          "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                          "cpu_baseline": cb,
                          "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch

    from pacuda_b200 import batch as B
    from pacuda_b200 import build

    build.build()
    if args.surrogate_kernels:
        print(json.dumps({"surrogate_kernels": surrogate_kernels(torch)}))
        return
    if args.listing:
        print(json.dumps({"listing": listing_case(torch)}))
        return
    if args.surrogate_only:
        kw = {}
        for item in args.surrogate_args.split(",") if args.surrogate_args else []:
            key, val = item.split("=")
            if key == "families":
                from pacuda_b200 import processes

                kw[key] = processes.PP4J if val == "pp4j" else processes.PP3J
                continue
            kw[key] = float(val) if "." in val or "e" in val else int(val)
        print(json.dumps({"surrogate": surrogate_line(torch, **kw)}))
        return
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    fams = workload(rank)
    plans, ext, out = [], [], []
    flops = 0.0
    for name, t, p in fams:
        pl = B.Plan(t, "f64")
        plans.append(pl)
        ext.append(torch.tensor(phase_space_major(p), dtype=torch.float64, device="cuda"))
        out.append(torch.empty(p.shape[0] * t.outputs, dtype=torch.float64, device="cuda"))
        flops += pl.flops * p.shape[0]
    if args.lanes_per_point:
        for pl in plans:
            pl.lanes_per_point = args.lanes_per_point
    batch = B.Batch(plans, ext, out)
    if not args.no_tune and not args.lanes_per_point:
        batch.tune()
    if args.blocks_per_sm:
        batch.blocks_per_sm = args.blocks_per_sm
    stream = torch.cuda.Stream()
    if not args.no_graph:
        with torch.cuda.stream(stream):
            batch.capture(stream)
    for _ in range(args.warmup):
        batch.run(stream)
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", 0))) if rank == 0 else None
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.mark()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        batch.run(stream)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop() if clocks else None
    # per family: the total |M|^2, its sum of squares and its largest value (per point, summed
    # over the helicities)
    m2 = [o.view(p.shape[0], t.outputs).sum(dim=1) for o, (_, t, p) in zip(out, fams)]
    sums = torch.stack([x.sum() for x in m2])
    squares = torch.stack([(x * x).sum() for x in m2])
    peak_m2 = torch.stack([x.max() for x in m2])
    if world > 1:
        ms, sums, squares, peak_m2 = reduce_over_ranks(dist, ms, sums, squares, peak_m2)
        dist.barrier()
    points = sum(p.shape[0] for _, _, p in fams) * world
    value = points / (ms * 1e-3)
    peak = fp64_peak(torch, B.lib())
    achieved = flops / (ms * 1e-3) / 1e12  # this rank's launch: its flops over its device time
    alg_bytes = sum(p.shape[0] * (32 * t.external_count + 8 * t.outputs) for _, t, p in fams)
    per_point = dram_bytes_per_point() if not args.family else None
    traffic = per_point * sum(p.shape[0] for _, _, p in fams) if per_point else None
    res = {"metric": metric, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
           "gpu_launches": args.steps * batch.launches,
           "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak, "traffic": traffic,
                        "peak_source": "f64 FMA throughput measured in this run (2 flops per DFMA); the "
                                       "reference's arithmetic has no FMA, so half of it is the ceiling",
                        "frac_of_no_fma_ceiling": achieved / (peak / 2),
                        "traffic_source": "dram read+write bytes per point from one ncu capture of the same mix "
                                          "at its full 2^20 points in one launch "
                                          "(profiles/launches_pp3j_bench.md), times this launch's points",
                        "hbm": {"achieved_gbs": traffic / (ms * 1e-3) / 1e9 if traffic else None,
                                "algorithmic_bytes": alg_bytes,
                                "algorithmic_gbs": alg_bytes / (ms * 1e-3) / 1e9,
                                "algorithmic_bytes_note": "momenta in (legs x 4 x 8 B) and every helicity output out "
                                                          "(8 B each) per point",
                                "peak_gbs": hbm_peak()[0], "peak_source": hbm_peak()[1]},
                        "flops_per_point": {n: pl.flops for (n, _, _), pl in zip(fams, plans)}},
           "points_per_family": {n: p.shape[0] for n, _, p in fams},
           "lanes_per_point": {n: batch.lanes_per_point(k) for k, (n, _, _) in enumerate(fams)},
           "blocks_per_sm": {n: batch.plan_blocks_per_sm(k) for k, (n, _, _) in enumerate(fams)},
           "sum_m2_per_family": [float(x) for x in sums.cpu()],
           "sum_m2_squared_per_family": [float(x) for x in squares.cpu()],
           "max_m2_per_family": [float(x) for x in peak_m2.cpu()]}
    if clk:
        res["clocks"] = clk
    if world > 1 and not args.no_e2e and not args.family:
        # end to end at N GPUs: every rank's UMAMI call on its own shard from its pinned host
        # momenta, the ranks started together; the job's time per step is the slowest rank's
        from pacuda_b200.umami import build as ub

        if rank == 0:
            ub.pp3j_library()  # built once, before the other ranks look for it
        dist.barrier()
        line = e2e_umami(fams, max(3, args.steps // 2), 2, [o.cpu().numpy() for o in out], sync=dist.barrier)
        slowest = torch.tensor([line["seconds"]], dtype=torch.float64, device="cuda")
        dist.all_reduce(slowest, op=dist.ReduceOp.MAX)
        line["value"] = points / float(slowest)
        line["seconds"] = float(slowest)
        line["h2d_bytes_per_step"] *= world  # the whole job's copies
        line["d2h_bytes_per_step"] *= world
        line["api"] += f", one call per rank on its shard, {world} ranks, the slowest rank's time"
        res["e2e"] = line
    if rank == 0 and world == 1:
        if not args.no_e2e:
            outs = [o.cpu().numpy() for o in out]
            res["e2e"] = e2e_umami(fams, max(3, args.steps // 2), 2, outs)
            abi_line, _ = e2e_abi(fams, max(1, args.steps // 5), 1)
            abi_line["api"] = "pacman_recurrence_v1_run + _reduce_resolved per tile of 2^16 points"
            res["e2e_abi"] = abi_line
        oracle_out = {}
        if not args.no_cpu:
            res["cpu_baseline"] = cpu_baseline(fams, keep=oracle_out)
        # parity of what was timed: the first 2048 points of every family, bit for bit
        first = {name: o.view(p.shape[0], t.outputs)[: min(2048, p.shape[0])].cpu().numpy()
                 for o, (name, t, p) in zip(out, fams)}
        if not oracle_out:
            from oracle import oracle as O

            for name, t, p in fams:
                oracle_out[name] = O.evaluate(t, p[: min(2048, p.shape[0])], kernel=1)[1]
        pairs = [(f"{name} vs oracle", first[name], oracle_out[name]) for name, _, _ in fams]
        if not args.no_reference_gpu and not args.family:
            import tempfile

            keep = os.path.join(tempfile.mkdtemp(prefix="bench_ref_"), "ref_f64.npz")
            ref = reference_gpu(steps=2, warmup=1, keep_path=keep)
            if ref:
                res["reference_gpu"] = ref
                res["reference_gpu"]["runner"] = ("the reference's recurrence_runner.cu built from its own sources for "
                                                  "sm_100a (oracle/Makefile, runner/build.sh flags), unmodified, through its "
                                                  "C ABI: per tile of 2^16 points a run and a resolved reduction from pinned "
                                                  "host buffers")
                f64 = ref.get("f64", {})
                if "device_value" in f64:
                    res["vs_reference_gpu"] = {"value_over_device_f64": value / f64["device_value"],
                                               "e2e_over_e2e_f64": (res["e2e"]["value"] / f64["value"]) if "e2e" in res else None,
                                               "e2e_abi_over_e2e_f64": (res["e2e_abi"]["value"] / f64["value"])
                                               if "e2e_abi" in res else None}
                if os.path.exists(keep):
                    ref_out = dict(np.load(keep))
                    pairs += [(f"{name} vs reference runner f64", first[name], ref_out[name]) for name, _, _ in fams]
        res["parity"] = parity(pairs)
        res["parity"]["what"] = ("the timed run's outputs of the first 2048 points of each family against the oracle "
                                 "and the reference runner's f64 kernel, bit for bit")
        if not args.no_precision:
            res["precision"] = [precision_line(torch, B, fams, ext, out, args.steps, args.warmup, k)
                                for k in ("f64fma", "mixed", "mixed64", "df64")]
            res["precision_gg4g"] = six_gluon_line(torch, B)
            res["pp4j"] = pp4j_line(torch, B)
        if not args.no_surrogate:
            from pacuda_b200 import processes

            res["surrogate"] = surrogate_line(torch)
            if not args.no_precision:
                # p p -> 4 jets: the combined configuration's learned part (2^25 candidates: 5.6 % pass
                # the cuts and plain unweighting keeps 7e-4 of those, so 2^22 would give ~160 events)
                res["surrogate_pp4j"] = surrogate_line(torch, families=processes.PP4J, candidates=1 << 25,
                                                       epochs=600)
    if world > 1:
        import torch.distributed as dist

        del batch
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


def phase_space_major(p):
    from pacuda_b200 import phase_space

    return phase_space.source_major(p)


if __name__ == "__main__":
    main()
