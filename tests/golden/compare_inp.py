"""Read every INP file of the reference's own test tree with both readers
(the reference's FEA_INP, imported unmodified as make_golden.py does, and
fea_b200.FEA_INP) and, where all elements are C3D4 / C3D8, build both models
with from_inp; write a per-file report of every difference.

    python tests/golden/compare_inp.py --ref <path of the reference source tree>

The INP files are read where they lie and are not copied; the report
(``inp_reference_report.json`` next to this script) is the record.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def parse_diffs(r, o):
    d = []
    if list(r.part) != list(o.part):
        d.append("part names")
    for pn in r.part:
        if pn not in o.part:
            continue
        a, b = r.part[pn], o.part[pn]
        if not torch.equal(a.nodes, b.nodes):
            d.append("%s: nodes" % pn)
        if list(a.elems) != list(b.elems):
            d.append("%s: element types" % pn)
        d += ["%s: elements %s" % (pn, t) for t in a.elems if t in b.elems and not np.array_equal(a.elems[t], b.elems[t])]
        for kind in ("sets_nodes", "sets_elems"):
            A, B = getattr(a, kind), getattr(b, kind)
            if set(A) != set(B):
                d.append("%s: %s names" % (pn, kind))
            d += ["%s: %s %s (%d vs %d)" % (pn, kind, k, len(A[k]), len(B[k])) for k in A if k in B and A[k] != B[k]]
        if list(a.surfaces) != list(b.surfaces):
            d.append("%s: surface names" % pn)
        for s in a.surfaces:
            ea, eb = a.surfaces[s], b.surfaces.get(s, [])
            if len(ea) != len(eb) or any(not np.array_equal(x[0], y[0]) or x[1] != y[1] for x, y in zip(ea, eb)):
                d.append("%s: surface %s" % (pn, s))
        if [list(x) for x in a.sections] != [list(x) for x in b.sections]:
            d.append("%s: sections" % pn)
        if not torch.equal(a.elems_material, b.elems_material):
            d.append("%s: element material table" % pn)
    for mn, ma in r.material.items():
        mb = o.material.get(mn)
        if mb is None or (ma.type, list(ma.mat_para), ma.density) != (mb.type, list(mb.mat_para), mb.density):
            d.append("material %s" % mn)
    ia, ib = getattr(r.assemble, "instances", {}), o.assemble.instances
    if set(ia) != set(ib):
        d.append("instance names")
    d += ["instance %s" % k for k in ia if k in ib and (ia[k][0] != ib[k][0] or not np.allclose(ia[k][1], ib[k][1],
                                                                                                atol=1e-12))]
    for kind in ("sets_nodes", "sets_elems"):
        A, B = getattr(r.assemble, kind, {}), getattr(o.assemble, kind)
        if set(A) != set(B):
            d.append("assembly %s names" % kind)
        d += ["assembly %s %s (%d vs %d)" % (kind, k, len(A[k]), len(B[k])) for k in A if k in B and A[k] != B[k]]
    return d


def model_diffs(fr, fo):
    d = []
    for pn, pr in fr.assembly._parts.items():
        po = fo.assembly._parts[pn]
        if not torch.equal(pr.nodes.to(torch.float64), po.nodes):
            d.append("%s: nodes" % pn)
        if set(pr.set_nodes) != set(po.set_nodes):
            d.append("%s: node set names" % pn)
        d += ["%s: node set %s" % (pn, k) for k in pr.set_nodes
              if k in po.set_nodes and not np.array_equal(np.asarray(pr.set_nodes[k]), po.set_nodes[k])]
        er, eo = list(pr.elems.values()), list(po.elems.values())
        if len(er) != len(eo):
            d.append("%s: element groups" % pn)
        for k, (a, b) in enumerate(zip(er, eo)):
            same = (type(a).__name__ == type(b).__name__
                    and np.array_equal(np.asarray(a._elems_index), b._elems_index.numpy())
                    and np.array_equal(np.asarray(a._elems), b._elems.numpy())
                    and (float(a.materials.mu), float(a.materials.kappa)) == b.materials.parameters()
                    and bool((torch.as_tensor(a.density) == float(b.density)).all()))
            if not same:
                d.append("%s: element group %d" % (pn, k))
        for s in po.surfaces.keys():
            fa = torch.cat([x._elems for x in pr.extract_surfaces(s)])
            fb = torch.cat([x._elems for x in po.extract_surfaces(s)])
            if not torch.equal(fa.to(torch.int64), fb):
                d.append("%s: surface %s faces" % (pn, s))
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the reference source tree (the directory holding FEA/)")
    a = ap.parse_args()
    from make_golden import import_reference
    FEA = import_reference(a.ref)
    import fea_b200 as F
    report = {}
    for path in sorted(glob.glob(os.path.join(a.ref, "tests", "**", "*.inp"), recursive=True)):
        key = os.path.relpath(path, a.ref)
        r, o = FEA.FEA_INP(), F.FEA_INP()
        entry = {}
        try:
            r.read_inp(path)
        except Exception as ex:                      # noqa: BLE001 (recorded)
            entry["reference_reader"] = "%s: %s" % (type(ex).__name__, ex)
        try:
            o.read_inp(path)
        except Exception as ex:                      # noqa: BLE001 (recorded)
            entry["fea_b200_reader"] = "%s: %s" % (type(ex).__name__, ex)
            report[key] = entry
            continue
        entry["elements"] = {t: int(e.shape[0]) for p in o.part.values() for t, e in p.elems.items()}
        if "reference_reader" not in entry:
            entry["parse_differences"] = parse_diffs(r, o)
            if set(entry["elements"]) <= {"C3D4", "C3D8"}:
                entry["model_differences"] = model_diffs(FEA.from_inp(r), F.from_inp(o))
        report[key] = entry
        print(key, json.dumps(entry))
    with open(os.path.join(HERE, "inp_reference_report.json"), "w") as f:
        json.dump(report, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
