"""The .pacuda v2 file (convert/src/format.rs:1-29): write, read back, and the byte layout."""
import os
import struct

import numpy as np

from pacuda_b200 import pacuda_file as PF


def test_roundtrip_of_generated_plans(tmp_path):
    f = PF.from_processes(["gg>ggg", "qg>qgg"], kernel=1, batch=4096, reference_points=3)
    f.symjit_sha256 = ["ab" * 32]
    f.processes[1].crossing = [(1, -1.0), (0, -1.0), (2, 1.0), (3, 1.0), (4, 1.0)]
    f.processes[0].parameters = [("aS", 0.118, 0.0), ("MT", 173.0, 0.0)]
    path = tmp_path / "plans.pacuda"
    PF.write(f, path)
    g = PF.read(path)
    assert (g.kernel, g.batch, g.symjit_sha256) == (1, 4096, ["ab" * 32])
    assert [p.key for p in g.processes] == ["gg>ggg", "qg>qgg"]
    assert g.processes[1].crossing == f.processes[1].crossing
    assert g.processes[0].parameters == f.processes[0].parameters
    for p, q in zip(f.processes, g.processes):
        assert (p.legs, p.helicities, p.qcd_power, p.factor) == (q.legs, q.helicities, q.qcd_power, q.factor)
        for c, d in zip(p.colours, q.colours):
            a, b = c.template, d.template
            assert np.array_equal(a.words, b.words) and list(a.width) == list(b.width)
            for name in ("scale_re", "scale_im", "factor_re", "factor_im", "zero_amplitude", "download_amplitude",
                         "form_terms", "term_slots", "term_coefficients", "offsets", "planes", "weights"):
                assert np.array_equal(getattr(a, name), getattr(b, name)), name
            assert np.array_equal(c.reference_momenta, d.reference_momenta)
    assert PF.to_bytes(g) == PF.to_bytes(f)


def test_header_layout():
    b = PF.to_bytes(PF.PacudaFile(kernel=3, batch=7))
    assert b[:8] == b"PACUDA\x00\x01"
    assert struct.unpack("<IIIII", b[8:28]) == (2, 3, 7, 0, 0)
    assert len(b) == 28


def test_rejects_truncated_and_trailing_bytes():
    b = PF.to_bytes(PF.from_processes(["gg>gg"], reference_points=0))
    for bad in (b[:-3], b + b"\x00"):
        try:
            PF.from_bytes(bad)
        except ValueError:
            continue
        raise AssertionError("accepted a malformed file")


def test_summary_dump(tmp_path):
    """The debugging dump (python -m pacuda_b200.pacuda_file FILE): sizes, op counts, reduction."""
    import json
    import subprocess
    import sys

    from pacuda_b200 import pacuda_file as PF

    f = PF.from_processes(["gg>ggg"], reference_points=0)
    path = str(tmp_path / "a.pacuda")
    PF.write(f, path)
    out = subprocess.run([sys.executable, "-m", "pacuda_b200.pacuda_file", path, "--arrays"], capture_output=True,
                         text=True, check=True, cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    d = json.loads(out.stdout)
    c = d["processes"][0]["colours"][0]
    t = f.processes[0].colours[0].template
    assert c["words"] == len(t.words) and len(c["words_hex"]) == len(t.words)
    assert sum(c["ops"].values()) == len(t.words) and c["outputs"] == 32 and c["live_outputs"] > 0
