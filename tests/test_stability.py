"""The rotated-momentum stability check (pacuda_b200/stability.py): the rotation is a rotation of
every leg's spatial momentum in the runner's source-major layout (the oracle's |M|^2 does not
change under it), and on the GPU every point carries either its mixed outputs or, when its check
fails, the f64 kernel's outputs, bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O
from pacuda_b200 import phase_space, processes, stability


def test_rotation_is_proper_and_leaves_the_oracles_m2_unchanged():
    import torch

    r = stability.rotation(7)
    assert np.allclose(r @ r.T, np.eye(3), atol=1e-15) and abs(np.linalg.det(r) - 1.0) < 1e-14
    t = processes.template("gg>ggg")
    n = 40
    p = phase_space.sample(5, n, 3)
    ext = torch.tensor(phase_space.source_major(p), dtype=torch.float64)
    q = stability.rotate(ext, 5, r).numpy().reshape(5, 4, n).transpose(2, 0, 1)
    assert np.array_equal(q[:, :, 0], p[:, :, 0])
    assert np.allclose(q[:, :, 1:], np.einsum("ij,nlj->nli", r, p[:, :, 1:]), rtol=0, atol=1e-9)
    _, a = O.evaluate(t, p, kernel=1)
    _, b = O.evaluate(t, np.ascontiguousarray(q), kernel=1)
    ta, tb = a.sum(axis=1), b.sum(axis=1)
    assert np.max(np.abs(tb / ta - 1.0)) < 1e-11


def _setup(names_or_parts, n, seed):
    import torch

    templates = names_or_parts
    legs = templates[0].external_count
    p = phase_space.sample(legs, n, seed, ecm=13000.0, pt_min=5.0, dr_min=0.1) if legs == 6 else \
        phase_space.sample(legs, n, seed)
    ext = torch.tensor(phase_space.source_major(p), dtype=torch.float64, device="cuda")
    return templates, p, ext


def _reference_outputs(templates, ext, n, kind):
    import torch
    from pacuda_b200 import batch as B

    plans = [B.Plan(t, kind) for t in templates]
    outs = [torch.full((n * t.outputs,), float("nan"), dtype=torch.float64, device="cuda") for t in templates]
    b = B.Batch(plans, [ext] * len(plans), outs)
    b.run()
    torch.cuda.synchronize()
    return [o.cpu().numpy().reshape(n, t.outputs) for o, t in zip(outs, templates)]


@pytest.mark.gpu
@pytest.mark.parametrize("tol", [0.0, 1e-7, float("inf")])
@pytest.mark.parametrize("process", ["gg>ggg", "gg>gggg"])
def test_points_carry_mixed_or_f64_bits_as_their_check_decides(process, tol):
    import torch

    templates = processes.parts(process) if process == "gg>gggg" else [processes.template(process)]
    n = 96 if process == "gg>gggg" else 700
    templates, p, ext = _setup(templates, n, 29)
    mixed = _reference_outputs(templates, ext, n, "mixed")
    f64 = _reference_outputs(templates, ext, n, "f64")
    s = stability.StableMixed(templates, n, tol)
    for repeat in range(2):  # the second run re-points the batches it made
        outs, m = s.run(ext)
        torch.cuda.synchronize()
        bad = s.unstable.cpu().numpy()
        assert m == int(bad.sum())
        if tol == float("inf"):
            assert m == 0
        for o, t, mx, fx in zip(outs, templates, mixed, f64):
            got = o.cpu().numpy().reshape(n, t.outputs)
            want = np.where(bad[:, None], fx, mx)
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), repeat
    if tol == 0.0:
        assert m > n // 2  # two f32 evaluations rarely agree to the bit


@pytest.mark.gpu
@pytest.mark.parametrize("tol", [1e-6, 1e-5])
def test_kept_points_are_within_ten_tolerances_of_f64(tol):
    """The points the check keeps in mixed precision: their |M|^2 within 10 tol of f64 (the check
    estimates a point's error from two evaluations that round alike; it is not a bound, so the
    margin is stated and tested), and a tolerance below the floor sends every point to f64."""
    import torch

    templates, p, ext = _setup([processes.template("gg>ggg")], 2000, 31)
    f64 = _reference_outputs(templates, ext, 2000, "f64")[0].sum(axis=1)
    s = stability.StableMixed(templates, 2000, tol)
    outs, m = s.run(ext)
    torch.cuda.synchronize()
    got = outs[0].cpu().numpy().reshape(2000, -1).sum(axis=1)
    kept = ~s.unstable.cpu().numpy()
    rel = np.abs(got - f64) / np.abs(f64)
    assert kept.sum() > 0
    assert np.all(rel[kept] <= 10 * tol), (rel[kept].max(), tol)
    low = stability.StableMixed(templates, 2000, stability.FLOOR / 10)
    outs, m = low.run(ext)
    torch.cuda.synchronize()
    assert m == 2000
    assert np.array_equal(outs[0].cpu().numpy().reshape(2000, -1).sum(axis=1), f64)
