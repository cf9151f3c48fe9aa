"""pacuda_b200_run_static, the entry point that allocates nothing, through the C ABI: two calls in a
row give the bits a batch of the same plans gives (the same executor, so the tolerance is zero),
and more plans than its fixed array holds are refused. The file is named to be collected last, so
the entry point also runs after every other test has used the library."""
import ctypes as C

import numpy as np
import pytest

from pacuda_b200 import phase_space, processes

NAMES = ["gg>ggg", "qg>qgg", "qq~>ggg", "gg>qq~g"]
COUNTS = [300, 77, 1025, 9]
INVALID = 2


def _static(lib):
    f = lib.pacuda_b200_run_static
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _arrays(values):
    n = len(values)
    return (C.c_void_p * n)(*values)


@pytest.mark.gpu
def test_run_static_equals_batch_run_on_two_calls():
    import torch
    from pacuda_b200 import batch as B

    plans, ext, ref, out = [], [], [], []
    for name, n in zip(NAMES, COUNTS):
        t = processes.template(name)
        p = phase_space.sample(len(processes.PROCESSES[name]), n, 41 + n)
        plans.append(B.Plan(t, "f64"))
        ext.append(torch.tensor(phase_space.source_major(p), dtype=torch.float64, device="cuda"))
        ref.append(torch.full((n * t.outputs,), float("nan"), dtype=torch.float64, device="cuda"))
        out.append(torch.full((n * t.outputs,), float("nan"), dtype=torch.float64, device="cuda"))
    b = B.Batch(plans, ext, ref)
    b.run()
    torch.cuda.synchronize()
    want = [r.cpu().numpy() for r in ref]
    assert all(np.isfinite(w).all() for w in want)

    run = _static(B.lib())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    handles = _arrays([p.handle for p in plans])
    eptr = _arrays([e.data_ptr() for e in ext])
    optr = _arrays([o.data_ptr() for o in out])
    cnt = (C.c_uint32 * len(COUNTS))(*COUNTS)
    for call in range(2):
        for o in out:
            o.fill_(float("nan"))
        assert run(handles, len(plans), eptr, cnt, optr, stream) == 0
        torch.cuda.synchronize()
        for o, w in zip(out, want):
            got = o.cpu().numpy()
            assert np.array_equal(got.view(np.uint64), w.view(np.uint64)), (call, np.abs(got - w).max())


@pytest.mark.gpu
def test_run_static_refuses_more_plans_than_its_array_holds():
    import torch
    from pacuda_b200 import batch as B

    t = processes.template("qg>qgg")
    n = 4
    p = phase_space.sample(len(processes.PROCESSES["qg>qgg"]), n, 5)
    plan = B.Plan(t, "f64")
    e = torch.tensor(phase_space.source_major(p), dtype=torch.float64, device="cuda")
    o = torch.zeros(n * t.outputs, dtype=torch.float64, device="cuda")
    run = _static(B.lib())
    k = 9  # PACUDA_B200_STATIC_MAX_PLANS + 1
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    status = run(_arrays([plan.handle] * k), k, _arrays([e.data_ptr()] * k), (C.c_uint32 * k)(*[n] * k),
                 _arrays([o.data_ptr()] * k), stream)
    assert status == INVALID
    assert run(_arrays([plan.handle]), 0, _arrays([e.data_ptr()]), (C.c_uint32 * 1)(n), _arrays([o.data_ptr()]),
               stream) == INVALID
    # a call at the limit still works afterwards, every plan into its own output
    outs = [torch.full((n * t.outputs,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(8)]
    assert run(_arrays([plan.handle] * 8), 8, _arrays([e.data_ptr()] * 8), (C.c_uint32 * 8)(*[n] * 8),
               _arrays([x.data_ptr() for x in outs]), stream) == 0
    torch.cuda.synchronize()
    first = outs[0].cpu().numpy()
    assert np.isfinite(first).all()
    for x in outs[1:]:
        assert np.array_equal(x.cpu().numpy().view(np.uint64), first.view(np.uint64))
