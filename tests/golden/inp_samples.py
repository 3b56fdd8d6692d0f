"""Sample INP files in the layout Abaqus/CAE writes, for the INP reader's
tests: ``inp_hex.inp`` (a jittered 3x3x3 C3D8 block with list and
``generate`` sets, an element-based surface on an internal set, a section,
a Neo-Hookean material with density, and an assembly with a plain and a
translated + rotated instance) and ``inp_mixed.inp`` (one part holding a
2x2x2 C3D8 block and a separate C3D4 cube, two sections with two
materials, and a surface on both element types).

``make_golden.py --case inp`` writes these files and the fixtures of what
the reference reads from them; the tests read the committed files.
"""
from __future__ import annotations

import os

import numpy as np


def _rows(values, per=16):
    v = [int(x) for x in values]
    return ["".join("%d, " % x for x in v[i:i + per]).rstrip(", ") for i in range(0, len(v), per)]


def _part(name, X, blocks, nsets, elsets, surfaces, sections):
    out = ["*Part, name=%s" % name, "*Node"]
    out += ["%7d, %s" % (i + 1, ", ".join("%.17g" % c for c in x)) for i, x in enumerate(X)]
    for etype, first, el in blocks:
        out.append("*Element, type=%s" % etype)
        out += ["%d, %s" % (first + k, ", ".join("%d" % (n + 1) for n in row)) for k, row in enumerate(el)]
    for nm, members, gen in nsets:
        out.append("*Nset, nset=%s%s" % (nm, ", generate" if gen else ""))
        out += ["%d, %d, %d" % members] if gen else _rows(np.asarray(members) + 1)
    for nm, members, gen, internal in elsets:
        out.append("*Elset, elset=%s%s%s" % (nm, ", internal" if internal else "", ", generate" if gen else ""))
        out += ["%d, %d, %d" % members] if gen else _rows(np.asarray(members) + 1)
    for nm, lines in surfaces:
        out.append("*Surface, type=ELEMENT, name=%s" % nm)
        out += ["%s, S%d" % (s, f) for s, f in lines]
    for k, (elset, mat) in enumerate(sections):
        out += ["** Section: Section-%d" % (k + 1), "*Solid Section, elset=%s, material=%s" % (elset, mat), ","]
    out.append("*End Part")
    return out


def _materials(mats):
    out = ["**", "** MATERIALS", "**"]
    for nm, rho, c10, d1 in mats:
        out += ["*Material, name=%s" % nm, "*Density", "%.17g," % rho, "*Hyperelastic, neo hooke",
                "%.17g, %.17g" % (c10, d1)]
    return out + ["** ----------------------------------------------------------------"]


def hex_sample():
    from oracle import fea_oracle as O
    n = 3
    X, el = O.hex_block(n, jitter=0.1, seed=4)
    X, el = X.numpy(), el.numpy()
    clamp = np.nonzero(X[:, 0] < 0.5 / n)[0]          # the first node plane (jittered)
    end = np.arange(el.shape[0])[np.arange(el.shape[0]) // (n * n) == n - 1]
    lines = ["*Heading", "** Job name: inp_hex Model name: Model-1", "*Preprint, echo=NO, model=NO, history=NO",
             "**", "** PARTS", "**"]
    lines += _part("block", X, [("C3D8", 1, el)],
                   [("clamp", clamp, False), ("allnodes", (1, X.shape[0], 1), True)],
                   [("allelems", (1, el.shape[0], 1), True, False), ("_end_S4", end, False, True)],
                   [("end", [("_end_S4", 4)])], [("allelems", "Rubber")])
    lines += ["**", "** ASSEMBLY", "**", "*Assembly, name=Assembly", "**",
              "*Instance, name=block-1, part=block", "*End Instance", "**",
              "*Instance, name=block-2, part=block", "          2.,         0.5,          0.",
              "          0.,          0.,          0.,          0.,          0.,          1.,         30.",
              "*End Instance", "**", "*Nset, nset=fixA", "1, 2, 3", "*Elset, elset=EA, generate", "1, 9, 2",
              "*End Assembly"]
    lines += _materials([("Rubber", 2.5, 0.5, 0.04)])
    return "\n".join(lines) + "\n"


def mixed_sample():
    from oracle import fea_oracle as O
    Xh, eh = O.hex_block(2, jitter=0.05, seed=5)
    Xt, et = O.tet_block(1)
    Xh, eh, Xt, et = Xh.numpy(), eh.numpy(), Xt.numpy(), et.numpy()
    Xt = Xt + np.array([2.0, 0.0, 0.0])
    X = np.concatenate([Xh, Xt])
    et = et + Xh.shape[0]
    nh, nt = eh.shape[0], et.shape[0]
    top_hex = np.arange(nh)[Xh[eh[:, 4:], 2].min(1) > 0.9]
    lines = ["*Heading", "** Job name: inp_mixed Model name: Model-1", "**", "** PARTS", "**"]
    lines += _part("body", X, [("C3D8", 1, eh), ("C3D4", nh + 1, et)],
                   [("clamp", np.nonzero(X[:, 0] < 0.25)[0], False)],
                   [("hexes", (1, nh, 1), True, False), ("tets", np.arange(nh, nh + nt), False, False),
                    ("_top_S2", top_hex, False, True), ("_tet_S1", np.arange(nh, nh + 2), False, True)],
                   [("top", [("_top_S2", 2), ("_tet_S1", 1)])],
                   [("hexes", "Rubber"), ("tets", "Foam")])
    lines += _materials([("Rubber", 1.5, 0.5, 0.04), ("Foam", 0.25, 0.2, 0.1)])
    return "\n".join(lines) + "\n"


SAMPLES = {"inp_hex": hex_sample, "inp_mixed": mixed_sample}


def write_samples(out_dir):
    paths = {}
    for name, make in SAMPLES.items():
        p = os.path.join(out_dir, name + ".inp")
        with open(p, "w") as f:
            f.write(make())
        paths[name] = p
    return paths
