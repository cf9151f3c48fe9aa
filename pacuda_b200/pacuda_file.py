"""The `.pacuda` plan file, version 2: reader and writer.

The format is the reference converter's (convert/src/format.rs:1-29; read by
umami/umami_pacuda.c:149-279): little endian, sequential, no padding; arrays are preceded by
their count, strings by their byte length (u32, no NUL); run lists by their number of
(first, count) pairs.

    file      magic "PACUDA\\0\\x01", u32 version 2, u32 kernel, u32 batch, u32 n, n x 64 hex bytes
              (symjit kernel SHA-256s), u32 processes, the processes
    process   str key, u32 legs, u32 helicities, str alpha_s name, f64 alpha_s, i32 QCD power,
              u32 parameters, (str name, f64 re, f64 im) each, i64 group numerator,
              i64 denominator, u32 crossing (0 or legs; then (u32 leg, f64 sign) each),
              u32 colours, the colours
    colour    str id, template, reduction, reference
    template  u32 tile, u32 words, u64 words[], u8 width[8], u32 current, amplitude and momentum
              planes, u32 scales, f64 re[], f64 im[], u32 factors, f64 re[], f64 im[], runs zero,
              runs download, u32 external count, runs form terms, u32 terms, u32 slots[],
              f64 coefficients[]
    reduction u32 outputs, u32 offsets[outputs + 1], u32 planes[..], f64 weights[..]
    reference u32 points, f64 momenta[points x legs x 4], f64 values[points x helicities]
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

from .plan import Template

MAGIC = b"PACUDA\x00\x01"
VERSION = 2


@dataclass
class Colour:
    id: str
    template: Template
    reference_momenta: np.ndarray = field(default_factory=lambda: np.zeros(0))
    reference_values: np.ndarray = field(default_factory=lambda: np.zeros(0))
    reference_points: int = 0


@dataclass
class Process:
    key: str
    legs: int
    helicities: int
    alpha_s_name: str = ""
    alpha_s: float = 0.0
    qcd_power: int = 0
    parameters: list = field(default_factory=list)  # (name, re, im)
    factor: tuple = (1, 1)
    crossing: list | None = None                     # [(leg, sign)] or None
    colours: list = field(default_factory=list)


@dataclass
class PacudaFile:
    kernel: int = 1
    batch: int = 0
    symjit_sha256: list = field(default_factory=list)
    processes: list = field(default_factory=list)


class _Out:
    def __init__(self):
        self.b = bytearray()

    def u32(self, v):
        self.b += struct.pack("<I", int(v))

    def i32(self, v):
        self.b += struct.pack("<i", int(v))

    def i64(self, v):
        self.b += struct.pack("<q", int(v))

    def f64(self, v):
        self.b += struct.pack("<d", float(v))

    def s(self, text):
        data = text.encode()
        self.u32(len(data))
        self.b += data

    def arr(self, a, dtype):
        self.b += np.ascontiguousarray(a, dtype=dtype).astype(np.dtype(dtype).newbyteorder("<")).tobytes()

    def runs(self, a):
        a = np.asarray(a, dtype=np.uint32).reshape(-1)
        self.u32(len(a) // 2)
        self.arr(a, np.uint32)


def to_bytes(f: PacudaFile) -> bytes:
    o = _Out()
    o.b += MAGIC
    o.u32(VERSION)
    o.u32(f.kernel)
    o.u32(f.batch)
    o.u32(len(f.symjit_sha256))
    for sha in f.symjit_sha256:
        data = sha.encode()
        if len(data) != 64:
            raise ValueError("a SHA-256 is 64 hex digits")
        o.b += data
    o.u32(len(f.processes))
    for p in f.processes:
        o.s(p.key)
        o.u32(p.legs)
        o.u32(p.helicities)
        o.s(p.alpha_s_name)
        o.f64(p.alpha_s)
        o.i32(p.qcd_power)
        o.u32(len(p.parameters))
        for name, re, im in p.parameters:
            o.s(name)
            o.f64(re)
            o.f64(im)
        o.i64(p.factor[0])
        o.i64(p.factor[1])
        if p.crossing is None:
            o.u32(0)
        else:
            o.u32(len(p.crossing))
            for leg, sign in p.crossing:
                o.u32(leg)
                o.f64(sign)
        o.u32(len(p.colours))
        for c in p.colours:
            t = c.template
            o.s(c.id)
            o.u32(t.tile)
            o.u32(len(t.words))
            o.arr(t.words, np.uint64)
            o.b += bytes(bytearray(int(x) & 0xFF for x in list(t.width)[:8]) + bytes(8 - min(8, len(t.width))))
            o.u32(t.current_planes)
            o.u32(t.amplitude_planes)
            o.u32(t.momentum_planes)
            o.u32(len(t.scale_re))
            o.arr(t.scale_re, np.float64)
            o.arr(t.scale_im, np.float64)
            o.u32(len(t.factor_re))
            o.arr(t.factor_re, np.float64)
            o.arr(t.factor_im, np.float64)
            o.runs(t.zero_amplitude)
            o.runs(t.download_amplitude)
            o.u32(t.external_count)
            o.runs(t.form_terms)
            o.u32(len(t.term_slots))
            o.arr(t.term_slots, np.uint32)
            o.arr(t.term_coefficients, np.float64)
            o.u32(len(t.offsets) - 1)
            o.arr(t.offsets, np.uint32)
            o.arr(t.planes, np.uint32)
            o.arr(t.weights, np.float64)
            o.u32(c.reference_points)
            o.arr(c.reference_momenta, np.float64)
            o.arr(c.reference_values, np.float64)
    return bytes(o.b)


class _In:
    def __init__(self, b):
        self.b, self.at = memoryview(b), 0

    def take(self, n):
        if n < 0 or self.at + n > len(self.b):
            raise ValueError("the file ends early")
        v = self.b[self.at:self.at + n]
        self.at += n
        return v

    def u32(self):
        return struct.unpack("<I", self.take(4))[0]

    def i32(self):
        return struct.unpack("<i", self.take(4))[0]

    def i64(self):
        return struct.unpack("<q", self.take(8))[0]

    def f64(self):
        return struct.unpack("<d", self.take(8))[0]

    def s(self):
        return bytes(self.take(self.u32())).decode()

    def arr(self, n, dtype):
        dt = np.dtype(dtype).newbyteorder("<")
        return np.frombuffer(bytes(self.take(n * dt.itemsize)), dtype=dt).astype(dtype)

    def runs(self):
        return self.arr(2 * self.u32(), np.uint32)


def from_bytes(data: bytes) -> PacudaFile:
    r = _In(data)
    if bytes(r.take(8)) != MAGIC:
        raise ValueError("not a .pacuda file")
    version = r.u32()
    if version != VERSION:
        raise ValueError(f".pacuda version {version}, this reader reads {VERSION}")
    f = PacudaFile(kernel=r.u32(), batch=r.u32())
    for _ in range(r.u32()):
        f.symjit_sha256.append(bytes(r.take(64)).decode())
    for _ in range(r.u32()):
        key = r.s()
        legs, hel = r.u32(), r.u32()
        p = Process(key=key, legs=legs, helicities=hel, alpha_s_name=r.s(), alpha_s=r.f64(), qcd_power=r.i32())
        p.parameters = [(r.s(), r.f64(), r.f64()) for _ in range(r.u32())]
        p.factor = (r.i64(), r.i64())
        nc = r.u32()
        if nc:
            if nc != legs:
                raise ValueError(f"process {key}: a crossing of {nc} legs, of {legs}")
            p.crossing = [(r.u32(), r.f64()) for _ in range(nc)]
        for _ in range(r.u32()):
            cid = r.s()
            tile = r.u32()
            words = r.arr(r.u32(), np.uint64)
            width = list(bytes(r.take(8)))
            cur, amp, mom = r.u32(), r.u32(), r.u32()
            ns = r.u32()
            sre, sim = r.arr(ns, np.float64), r.arr(ns, np.float64)
            nf = r.u32()
            fre, fim = r.arr(nf, np.float64), r.arr(nf, np.float64)
            zero, down = r.runs(), r.runs()
            ext = r.u32()
            form_terms = r.runs()
            nt = r.u32()
            slots, coef = r.arr(nt, np.uint32), r.arr(nt, np.float64)
            outputs = r.u32()
            offsets = r.arr(outputs + 1, np.uint32)
            count = int(offsets[-1])
            planes, weights = r.arr(count, np.uint32), r.arr(count, np.float64)
            t = Template(words=words, width=width, current_planes=cur, amplitude_planes=amp, momentum_planes=mom,
                         scale_re=sre, scale_im=sim, factor_re=fre, factor_im=fim, zero_amplitude=zero,
                         download_amplitude=down, external_count=ext, form_terms=form_terms, term_slots=slots,
                         term_coefficients=coef, offsets=offsets, planes=planes, weights=weights, tile=tile)
            npts = r.u32()
            moms = r.arr(npts * legs * 4, np.float64)
            vals = r.arr(npts * hel, np.float64)
            p.colours.append(Colour(cid, t, moms, vals, npts))
        f.processes.append(p)
    if r.at != len(data):
        raise ValueError(f"{len(data) - r.at} bytes after the last process")
    return f


def read(path) -> PacudaFile:
    with open(path, "rb") as fh:
        return from_bytes(fh.read())


def write(f: PacudaFile, path):
    with open(path, "wb") as fh:
        fh.write(to_bytes(f))


def from_processes(names, kernel=1, batch=0, reference_points=8, seed=7):
    """A file of generated plans (pacuda_b200.processes): one colour "lc" per process, or, for a
    process whose plan is split into parts of its colour orderings, one colour per part ("lc0",
    "lc1", ...: their values add up), with `reference_points` RAMBO points (their values left zero)."""
    from . import phase_space, processes

    f = PacudaFile(kernel=kernel, batch=batch)
    for name in names:
        legs = processes.PROCESSES[name]
        parts = processes.parts(name)
        t0 = parts[0]
        num, den = t0.meta["group_factor"]
        p = Process(key=name, legs=len(legs), helicities=t0.outputs, alpha_s_name="aS", alpha_s=t0.meta["alpha_s"],
                    qcd_power=t0.meta["qcd_power"], factor=(num, den))
        mom = phase_space.sample(len(legs), reference_points, seed) if reference_points else np.zeros((0, len(legs), 4))
        for k, t in enumerate(parts):
            t.tile = 1 << 16
            cid = "lc" if len(parts) == 1 else f"lc{k}"
            p.colours.append(Colour(cid, t, mom.reshape(-1), np.zeros(reference_points * t.outputs), reference_points))
        f.processes.append(p)
    return f


def summary(f: PacudaFile, arrays: bool = False) -> dict:
    """A JSON-ready description of a file (for debugging, as the reference's pac2json): per
    process its parameters and crossing, per colour its plan's sizes, its decoded rows' op counts
    and its reduction; with `arrays`, the tables themselves."""
    from . import plan as P

    def table(a):
        return [x.item() if hasattr(x, "item") else x for x in np.asarray(a).reshape(-1)]

    out = {"kernel": f.kernel, "batch": f.batch, "symjit_sha256": list(f.symjit_sha256), "processes": []}
    for p in f.processes:
        pd = {"key": p.key, "legs": p.legs, "helicities": p.helicities, "alpha_s": [p.alpha_s_name, p.alpha_s],
              "qcd_power": p.qcd_power, "parameters": [list(x) for x in p.parameters], "factor": list(p.factor),
              "crossing": [list(x) for x in p.crossing] if p.crossing else None, "colours": []}
        for c in p.colours:
            t = c.template
            ops = {}
            for row in P.decode(t.words, t.width):
                ops[int(row[0])] = ops.get(int(row[0]), 0) + 1
            offsets = np.asarray(t.offsets)
            cd = {"id": c.id, "tile": int(t.tile), "words": len(t.words), "width": [int(x) for x in t.width],
                  "current_planes": int(t.current_planes), "amplitude_planes": int(t.amplitude_planes),
                  "momentum_planes": int(t.momentum_planes), "scales": len(t.scale_re), "factors": len(t.factor_re),
                  "external_count": int(t.external_count), "terms": len(t.term_slots),
                  "ops": {str(k): v for k, v in sorted(ops.items())},
                  "outputs": len(offsets) - 1,
                  "live_outputs": int(np.count_nonzero(offsets[1:] > offsets[:-1])),
                  "reduction_terms": int(offsets[-1]), "reference_points": int(c.reference_points)}
            if arrays:
                cd.update({"words_hex": [f"{int(w):016x}" for w in t.words], "scale_re": table(t.scale_re),
                           "scale_im": table(t.scale_im), "factor_re": table(t.factor_re),
                           "factor_im": table(t.factor_im), "zero": table(t.zero_amplitude),
                           "download": table(t.download_amplitude), "form_terms": table(t.form_terms),
                           "term_slots": table(t.term_slots), "term_coefficients": table(t.term_coefficients),
                           "offsets": table(t.offsets), "planes": table(t.planes), "weights": table(t.weights)})
            pd["colours"].append(cd)
        out["processes"].append(pd)
    return out


if __name__ == "__main__":
    import json
    import sys

    if len(sys.argv) < 2:
        sys.exit("usage: python -m pacuda_b200.pacuda_file FILE.pacuda [--arrays]")
    print(json.dumps(summary(read(sys.argv[1]), arrays="--arrays" in sys.argv[2:]), indent=1))
