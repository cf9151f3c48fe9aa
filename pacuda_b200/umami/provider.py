"""Provider headers for the UMAMI library (include/umami_provider.h) from a plain description.

A subprocess's provider lists its processes (keys of the `.pacuda` file), and per channel and
flavour the contributions that make an event's |M|^2: (process, colour id, leg permutation,
factor, colour index). The reference takes these tables from the matrix-element artifact's
generated header; here they are written from a dict:

    {"particles": 5, "masses": [0.0] * 5, "colors": 1,
     "processes": [{"key": "gg>ggg", "helicities": 32,
                    "parameters": [("aS", 0.118, 0.0, False, True)]}],
     "channels": [[[{"process": 0, "colour": "lc", "permutation": [0, 1, 2, 3, 4],
                     "factor": 1.0, "color_index": 0}]]],
     "has_alpha_s": True, "has_color_flow": True}

(channels -> flavours -> contributions). Helicity labels map one to one onto every process's
helicities.
"""
from __future__ import annotations


def _c(x: float) -> str:
    return repr(float(x))


def header(spec: dict) -> str:
    n = int(spec["particles"])
    procs = spec["processes"]
    hel = max(int(p["helicities"]) for p in procs)
    out = ["/* generated by pacuda_b200/umami/provider.py */", "#include <stddef.h>", "#include <stdbool.h>",
           '#include "umami_provider.h"',
           f"#define UMAMI_HAS_ALPHA_S {1 if spec.get('has_alpha_s', True) else 0}",
           f"#define UMAMI_HAS_COLOR_FLOW {1 if spec.get('has_color_flow', True) else 0}"]
    out.append(f"static const double provider_masses[{n}] = {{{', '.join(_c(m) for m in spec['masses'])}}};")
    out.append(f"static const int provider_identity[{hel}] = {{{', '.join(str(h) for h in range(hel))}}};")
    for i, p in enumerate(procs):
        params = p.get("parameters", [])
        rows = ", ".join(f'{{"{nm}", {_c(re)}, {_c(im)}, {str(bool(cx)).lower()}, {str(bool(mu)).lower()}}}'
                         for nm, re, im, cx, mu in params) or '{"", 0.0, 0.0, false, false}'
        out.append(f"static const UmamiParameter provider_parameters_{i}[] = {{{rows}}};")
    out.append("static const UmamiProcess provider_processes[] = {" + ", ".join(
        f'{{"{p["key"]}", {int(p["helicities"])}, {len(p.get("parameters", []))}, provider_parameters_{i}}}'
        for i, p in enumerate(procs)) + "};")
    chans = []
    for c, channel in enumerate(spec["channels"]):
        flavs = []
        for f, contributions in enumerate(channel):
            rows = []
            for j, e in enumerate(contributions):
                perm = e["permutation"]
                assert sorted(perm) == list(range(n)), perm
                out.append(f"static const size_t provider_perm_{c}_{f}_{j}[{n}] = {{{', '.join(str(x) for x in perm)}}};")
                rows.append(f'{{{int(e["process"])}, "{e["colour"]}", provider_perm_{c}_{f}_{j}, {_c(e["factor"])}, '
                            f'provider_identity, provider_identity, {int(e.get("color_index", 0))}}}')
            out.append(f"static const UmamiContribution provider_contributions_{c}_{f}[] = {{{', '.join(rows)}}};")
            flavs.append(f"{{{len(contributions)}, provider_contributions_{c}_{f}}}")
        out.append(f"static const UmamiFlavour provider_flavours_{c}[] = {{{', '.join(flavs)}}};")
        chans.append(f"{{{len(channel)}, provider_flavours_{c}}}")
    out.append(f"static const UmamiChannel provider_channels[] = {{{', '.join(chans)}}};")
    out.append(f"static const UmamiProvider umami_provider = {{{n}, {hel}, {hel}, {int(spec.get('colors', 1))}, "
               f"provider_masses, {len(procs)}, provider_processes, {len(spec['channels'])}, provider_channels}};")
    return "\n".join(out) + "\n"
