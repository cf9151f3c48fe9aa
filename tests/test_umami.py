"""The UMAMI library's host parts on CPU: its `.pacuda` reader agrees with the Python reader (and
rejects what the reference's rejects), the program key is the reference's FNV-1a, and the library
builds against a provider header and exports exactly the nine UMAMI functions."""
import ctypes as C
import os
import struct
import subprocess

import pytest

from pacuda_b200 import pacuda_file
from tests import umami_fixture as U

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "tests", "harness")
UMAMI_FUNCTIONS = {"umami_get_meta", "umami_supported_inputs", "umami_required_inputs", "umami_supported_outputs",
                   "umami_initialize", "umami_free", "umami_get_parameter", "umami_set_parameter",
                   "umami_matrix_element"}


def reader():
    subprocess.run(["make", "-s", "-C", HARNESS, "libreader_harness.so"], check=True)
    lib = C.CDLL(os.path.join(HARNESS, "libreader_harness.so"))
    lib.reader_dump.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t]
    return lib


def dump(path):
    buf = C.create_string_buffer(1 << 22)
    n = reader().reader_dump(path.encode(), buf, len(buf))
    return n, buf.value.decode()


def fnv(widths, words):
    h = 1469598103934665603
    for b in bytes(widths[:8]) + b"".join(struct.pack("<Q", int(w)) for w in words):
        h = ((h ^ b) * 1099511628211) & (2 ** 64 - 1)
    return h or 1


def python_dump(f):
    g = lambda v, fmt: "".join(fmt % x for x in v)
    s = f"file kernel {f.kernel} batch {f.batch} shas {len(f.symjit_sha256)}\n"
    for p in f.processes:
        s += (f"process {p.key} legs {p.legs} helicities {p.helicities} alpha {p.alpha_s_name} {p.alpha_s:.17g} "
              f"power {p.qcd_power} factor {p.factor[0]}/{p.factor[1]}\n")
        for nm, re, im in p.parameters:
            s += f"parameter {nm} {re:.17g} {im:.17g}\n"
        s += "crossing" + g([l for l, _ in p.crossing or []], " %u") + "\n"
        s += "signs" + g([x for _, x in p.crossing or []], " %.17g") + "\n"
        for c in p.colours:
            t = c.template
            w = (list(t.width) + [0] * 8)[:8]
            live = [h for h in range(len(t.offsets) - 1) if t.offsets[h + 1] > t.offsets[h]]
            s += (f"colour {c.id} tile {t.tile} words {len(t.words)} key {fnv(w, t.words):016x} planes "
                  f"{t.current_planes} {t.amplitude_planes} {t.momentum_planes} external {t.external_count} "
                  f"outputs {len(t.offsets) - 1}\n")
            s += "width" + g(w, " %u") + "\n"
            s += "scale_re" + g(t.scale_re, " %.17g") + "\n"
            s += "factor_im" + g(t.factor_im, " %.17g") + "\n"
            s += "zero" + g(list(t.zero_amplitude), " %u") + "\n"
            s += "download" + g(list(t.download_amplitude), " %u") + "\n"
            s += "form_terms" + g(list(t.form_terms), " %u") + "\n"
            s += "term_slots" + g(list(t.term_slots), " %u") + "\n"
            s += "offsets" + g(list(t.offsets), " %u") + "\n"
            s += "live" + g(live, " %u") + "\n"
            s += "live_offsets" + g([t.offsets[h] for h in live] + [t.offsets[-1]], " %u") + "\n"
            s += f"reference {c.reference_points} {len(c.reference_momenta)} {len(c.reference_values)}\n"
    return s


def test_reader_agrees_with_the_python_reader(tmp_path):
    d = U.make_artifact(str(tmp_path / "artifact"))
    f = pacuda_file.read(d + ".pacuda")
    f.processes[0].parameters = [("MT", 173.0, 0.0)]
    f.processes[0].colours[0].reference_points = 2
    f.processes[0].colours[0].reference_momenta = [0.5] * (2 * 5 * 4)
    f.processes[0].colours[0].reference_values = [1.5] * (2 * 32)
    pacuda_file.write(f, d + ".pacuda")
    n, text = dump(d + ".pacuda")
    assert n > 0, text
    assert text == python_dump(pacuda_file.read(d + ".pacuda"))


def test_reader_rejects_malformed_files(tmp_path):
    d = U.make_artifact(str(tmp_path / "artifact"))
    data = open(d + ".pacuda", "rb").read()
    cases = {"truncated": data[:-3], "trailing": data + b"\0", "magic": b"PACUDX" + data[6:],
             "version": data[:8] + struct.pack("<I", 3) + data[12:], "empty": b""}
    for name, bad in cases.items():
        path = str(tmp_path / f"{name}.pacuda")
        open(path, "wb").write(bad)
        n, why = dump(path)
        assert n == -1 and why, name
    assert dump(str(tmp_path / "missing.pacuda"))[0] == -1


def test_umami_library_builds_and_exports_the_nine_functions(tmp_path):
    from pacuda_b200 import build
    from pacuda_b200.umami import build as ubuild, provider

    build.build()
    hdr = tmp_path / "provider_test.h"
    hdr.write_text(provider.header(U.SPEC))
    so = ubuild.build(str(hdr), str(tmp_path / "libumami_test.so"))
    names = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in names.splitlines() if " T " in line}
    assert exported == UMAMI_FUNCTIONS
    lib = C.CDLL(so)  # loads without a GPU; the metadata needs none
    n = C.c_int()
    assert lib.umami_get_meta(3, C.byref(n)) == 0 and n.value == 32
    assert lib.umami_get_meta(1, C.byref(n)) == 0 and n.value == 5
    assert lib.umami_get_meta(99, C.byref(n)) != 0
