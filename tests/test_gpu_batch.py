"""The batched device API: several plans in one persistent launch, each plan's resolved outputs
equal to the oracle's bit for bit, for every points-per-warp choice and kernel kind; the tuned and
graph-captured runs give the same bits."""
import numpy as np
import pytest

from tests import scenarios as S
from oracle import oracle as O
from pacuda_b200 import abi, phase_space, processes

NAMES = ["gg>ggg", "qg>qgg", "qq~>ggg", "gg>qq~g"]


def setup(kind, counts):
    import torch
    from pacuda_b200 import batch as B

    plans, ext, out, want = [], [], [], []
    for name, n in zip(NAMES, counts):
        t = processes.template(name)
        p = phase_space.sample(len(processes.PROCESSES[name]), n, 17 + n)
        _, w = O.evaluate(t, p, kernel=abi.KERNELS[kind])
        plans.append(B.Plan(t, kind))
        ext.append(torch.tensor(phase_space.source_major(p), dtype=torch.float64, device="cuda"))
        out.append(torch.full((n * t.outputs,), float("nan"), dtype=torch.float64, device="cuda"))
        want.append(w)
    return plans, ext, out, want


def check(out, want):
    for o, w in zip(out, want):
        got = o.cpu().numpy().reshape(w.shape)
        assert np.array_equal(got.view(np.uint64), w.view(np.uint64)), np.abs(got - w).max()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["f64", "df64", "mixed", "mixed64"])
def test_batch_matches_oracle_bitwise(kind):
    from pacuda_b200 import batch as B
    import torch

    plans, ext, out, want = setup(kind, [70, 33, 129, 5])
    b = B.Batch(plans, ext, out)
    b.run()
    torch.cuda.synchronize()
    check(out, want)


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [8, 16, 25, 32, 64, 96, 128, 170, 256, 512])
def test_every_lanes_per_point_gives_the_same_bits(lanes):
    """Blocks of 1 to 32 points, with idle threads where the points do not divide a warp;
    plans whose points do not fit keep their default."""
    from pacuda_b200 import batch as B
    import torch

    plans, ext, out, want = setup("f64", [70, 33, 129, 5])
    taken = 0
    for p in plans:
        try:
            p.lanes_per_point = lanes
            taken += 1
        except Exception:
            pass
    if not taken:
        pytest.skip(f"{lanes} lanes per point fit no plan")
    given = min(16 * (32 // n) for n in range(1, 33) if 16 * (32 // n) >= lanes)  # 16 warps
    assert any(p.lanes_per_point == given for p in plans)
    b = B.Batch(plans, ext, out)
    b.run()
    torch.cuda.synchronize()
    check(out, want)


@pytest.mark.gpu
def test_tuned_and_captured_runs_give_the_same_bits():
    from pacuda_b200 import batch as B
    import torch

    plans, ext, out, want = setup("f64", [300, 200, 100, 50])
    b = B.Batch(plans, ext, out)
    b.tune()
    for o in out:
        o.fill_(float("nan"))
    b.capture()
    b.run()
    torch.cuda.synchronize()
    check(out, want)
    assert b.launches == len({b.plan_blocks_per_sm(k) for k in range(len(plans))})


@pytest.mark.gpu
def test_plans_of_different_blocks_per_sm_run_as_launches_of_one_batch():
    """Plans with 1, 2 and 4 blocks per SM in one batch: three launches, each plan's bits."""
    from pacuda_b200 import batch as B
    import torch

    plans, ext, out, want = setup("f64", [300, 200, 100, 50])
    b = B.Batch(plans, ext, out)
    for k, blocks in enumerate([4, 2, 1, 2]):
        b.set_plan_blocks_per_sm(k, blocks)
    assert [b.plan_blocks_per_sm(k) for k in range(4)] == [4, 2, 1, 2] and b.launches == 3
    b.run()
    torch.cuda.synchronize()
    check(out, want)
    for o in out:
        o.fill_(float("nan"))
    b.capture()
    b.run()
    torch.cuda.synchronize()
    check(out, want)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["f64", "mixed"])
@pytest.mark.parametrize("blocks", [0, 2, 4])
def test_several_blocks_per_sm_give_the_same_bits(kind, blocks):
    """Independent blocks per SM (each with its share of the SM's shared memory and warps)."""
    from pacuda_b200 import batch as B
    import torch

    plans, ext, out, want = setup(kind, [70, 33, 129, 5])
    b = B.Batch(plans, ext, out)
    b.blocks_per_sm = blocks
    assert b.blocks_per_sm == blocks
    b.run()
    torch.cuda.synchronize()
    check(out, want)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["f64", "mixed"])
@pytest.mark.parametrize("blocks", [3, 5, 8, 16])
def test_blocks_of_fewer_warps_give_the_same_bits(kind, blocks):
    """3 and 5 blocks per SM (5 and 3 warps each, one warp of 16 unused), 8 and 16 (2 warps and
    1): every plan whose points fit such a block runs there, the others keep one block per SM;
    the plans then run as two launches, each plan's bits unchanged."""
    from pacuda_b200 import batch as B
    import torch

    plans, ext, out, want = setup(kind, [70, 33, 129, 5])
    b = B.Batch(plans, ext, out)
    moved = []
    for k in range(len(plans)):
        try:
            b.set_plan_blocks_per_sm(k, blocks)
            moved.append(k)
        except B.RunnerError:
            assert b.plan_blocks_per_sm(k) == 1
    assert moved and all(b.plan_blocks_per_sm(k) == blocks for k in moved)
    assert b.launches == (1 if len(moved) == len(plans) else 2)
    b.run()
    torch.cuda.synchronize()
    check(out, want)


@pytest.mark.gpu
def test_other_block_counts_are_refused():
    from pacuda_b200 import batch as B

    plans, ext, out, _ = setup("f64", [7, 7, 7, 7])
    b = B.Batch(plans, ext, out)
    for blocks in (6, 7, 9, 17, 32):
        with pytest.raises(B.RunnerError):
            b.blocks_per_sm = blocks
        with pytest.raises(B.RunnerError):
            b.set_plan_blocks_per_sm(1, blocks)
    assert b.blocks_per_sm == 1 and b.plan_blocks_per_sm(1) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["f64", "mixed"])
def test_six_gluon_parts_match_oracle_bitwise(kind):
    """gg>gggg as its parts (subsets of the colour orderings), in one batch: each part's outputs
    equal the oracle's bit for bit (one point per block, 512 lanes, 5 levels)."""
    from pacuda_b200 import batch as B
    import torch

    parts = processes.parts("gg>gggg")
    plans, ext, out, want = [], [], [], []
    for k, t in enumerate(parts):
        n = 40 + 13 * k
        p = phase_space.sample(6, n, 31 + k, ecm=13000.0)
        _, w = O.evaluate(t, p, kernel=abi.KERNELS[kind])
        plans.append(B.Plan(t, kind))
        ext.append(torch.tensor(phase_space.source_major(p), dtype=torch.float64, device="cuda"))
        out.append(torch.full((n * t.outputs,), float("nan"), dtype=torch.float64, device="cuda"))
        want.append(w)
    b = B.Batch(plans, ext, out)
    b.run()
    torch.cuda.synchronize()
    check(out, want)


@pytest.mark.gpu
def test_fma_kind_within_1e13_of_the_oracle():
    """The batched API's f64 kind with contracted multiply-adds: every point's |M|^2 (the sum of
    its helicity outputs) within 1e-13 relative of the f64 oracle, each helicity output within
    1e-13 of the point's largest; and not the same bits everywhere (the contraction happened)."""
    from pacuda_b200 import batch as B
    import torch

    counts = [300, 200, 200, 100]
    plans, ext, out, want = setup("f64", counts)
    fma = [B.Plan(p.template, "f64fma") for p in plans]
    b = B.Batch(fma, ext, out)
    b.run()
    torch.cuda.synchronize()
    differ = 0
    for o, w in zip(out, want):
        got = o.cpu().numpy().reshape(w.shape)
        tot_g, tot_w = got.sum(axis=1), w.sum(axis=1)
        assert np.all(np.abs(tot_g - tot_w) <= 1e-13 * np.abs(tot_w))
        assert np.all(np.abs(got - w) <= 1e-13 * np.abs(w).max(axis=1, keepdims=True))
        differ += int((got.view(np.uint64) != w.view(np.uint64)).sum())
    assert differ > 0
