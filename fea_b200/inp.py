"""Abaqus INP input: ``FEA_INP`` and ``from_inp``.

Mirrors the reader of sssnnn7119/FEA (FEA/inp.py:10-880) and its model
builder ``FEA.from_inp`` (FEA/__init__.py:10-79): the same attribute names
and layouts, so that code written against the reference reads a model the
same way.  Host code only (text parsing and the construction of ``Part`` /
``Assembly`` objects); nothing here runs on the device.

Layouts (all 0-based, as in the reference):

* ``part[name].nodes``: tensor [N, 4] in torch's default dtype, column 0 the
  node label - 1 and columns 1-3 the coordinates (inp.py:334-348);
* ``part[name].elems[type]``: int64 array [E, 1 + nodes per element], column
  0 the element label - 1 (inp.py:46-211);
* ``sets_nodes`` / ``sets_elems``: name -> set of labels - 1
  (inp.py:213-274);
* ``surfaces[name]``: list of (element labels - 1, face index - 1), one entry
  per data line and element type, in the element arrays' row order
  (inp.py:276-332);
* ``sections``: list of [element set, material] (inp.py:350-358);
* ``elems_material``: tensor [n, 5] = (label - 1, density, material type,
  parameter 0, parameter 1), -1 where no section applies (inp.py:367-368,
  870-879); material type 1 is Neo-Hookean with parameters
  (mu, kappa) = (2 C10, 2 / D1) (inp.py:460-466), type 0 linear elastic.

The parser reads keyword lines with their parameters in any order and case,
skips comment and blank lines, takes every data line of a block (several
``generate`` lines, several node or element blocks, element data continued
on the next line, set names inside set data) and accepts surfaces declared
before the elements they name.  On the CAE-written files the reference
reads, the results are the same; where the reference's fixed-format
matching would skip or overwrite a block, this reader takes it.  A
``*Hyperelastic`` model other than neo-Hooke raises NotImplementedError (the
reference reads its constants as neo-Hooke ones).
"""
from __future__ import annotations

import numpy as np
import torch

# nodes per element of the element types the reference reads (inp.py:46-211)
ELEMENT_NODES = {"C3D4": 4, "C3D4H": 4, "C3D6": 6, "C3D8": 8, "C3D8R": 8, "C3D10": 10, "C3D10H": 10,
                 "C3D15": 15, "C3D20": 20, "S3": 3}
SHELL_TYPES = {"S3"}
MATERIAL_OPTIONS = {"density", "hyperelastic", "elastic", "expansion", "damping", "conductivity",
                    "specific heat", "plastic", "depvar", "user material", "viscoelastic"}


def _norm(s: str) -> str:
    return " ".join(s.lower().split())


def parse_keyword(line: str):
    """'*Name, key=value, flag' -> ('name', {'key': 'value', 'flag': True});
    keyword and parameter names lower-cased with single spaces."""
    fields = [f.strip() for f in line.strip()[1:].split(",")]
    params = {}
    for f in fields[1:]:
        if not f:
            continue
        if "=" in f:
            k, v = f.split("=", 1)
            params[_norm(k)] = v.strip()
        else:
            params[_norm(f)] = True
    return _norm(fields[0]), params


def blocks(lines):
    """The file as [keyword, params, data lines] blocks, in file order;
    comment ('**') and blank lines dropped."""
    out = []
    for raw in lines:
        s = raw.strip()
        if not s or s.startswith("**"):
            continue
        if s.startswith("*"):
            name, params = parse_keyword(s)
            out.append([name, params, []])
        elif out:
            out[-1][2].append(s)
    return out


def _tokens(data):
    return [t.strip() for row in data for t in row.split(",") if t.strip()]


def _label_set(params, data, known):
    """Members (labels - 1) of a *Nset / *Elset block; `generate` lines are
    start, end[, step]; a non-numeric entry names another set of `known`."""
    out = set()
    if params.get("generate"):
        for row in data:
            v = [int(t) for t in row.split(",") if t.strip()]
            step = v[2] if len(v) > 2 else 1
            out.update(range(v[0] - 1, v[1], step))
        return out
    for t in _tokens(data):
        try:
            out.add(int(t) - 1)
        except ValueError:
            out.update(known[t])
    return out


class FEA_INP:
    """Reader of an Abaqus INP file (inp.py:10-880)."""

    class Parts:
        def __init__(self) -> None:
            self.elems: dict = {}
            self.nodes: torch.Tensor = None
            self.sections: list = []
            self.sets_nodes: dict = {}
            self.sets_elems: dict = {}
            self.surfaces: dict = {}
            self.num_elems_3D = 0
            self.num_elems_2D = 0
            self.elems_material: torch.Tensor = None

        def read(self, part_blocks):
            """Fill the part from its blocks (those between *Part and *End Part)."""
            node_rows, surface_blocks = [], []
            for name, params, data in part_blocks:
                if name == "node":
                    node_rows += [[float(t) for t in row.split(",") if t.strip()] for row in data]
                elif name == "element":
                    etype = str(params.get("type", "")).upper()
                    nn = ELEMENT_NODES.get(etype)
                    if nn is None:
                        continue                  # element types the reference does not read
                    v = np.array([int(t) for t in _tokens(data)], dtype=np.int64)
                    if v.size % (nn + 1):
                        raise ValueError("*Element, type=%s: %d numbers are not whole elements of %d"
                                         % (etype, v.size, nn + 1))
                    arr = v.reshape(-1, nn + 1) - 1
                    self.elems[etype] = np.concatenate([self.elems[etype], arr]) if etype in self.elems else arr
                    # counted in data lines, as the reference does (two per C3D20
                    # element): they size elems_material
                    if etype in SHELL_TYPES:
                        self.num_elems_2D += len(data)
                    else:
                        self.num_elems_3D += len(data)
                    if "elset" in params:
                        self.sets_elems.setdefault(params["elset"], set()).update(arr[:, 0].tolist())
                elif name == "nset":
                    self.sets_nodes[params["nset"]] = _label_set(params, data, self.sets_nodes)
                elif name == "elset":
                    self.sets_elems[params["elset"]] = _label_set(params, data, self.sets_elems)
                elif name == "surface":
                    surface_blocks.append((params, data))
                elif name == "solid section":
                    self.sections.append([params["elset"], params["material"]])
            if node_rows:
                self.nodes = torch.tensor(node_rows)
                self.nodes[:, 0] -= 1
            for params, data in surface_blocks:
                if str(params.get("type", "ELEMENT")).upper() != "ELEMENT" or not self.elems:
                    continue
                entries = []
                for row in data:
                    f = [t.strip() for t in row.split(",")]
                    if f[0] in self.sets_elems:
                        members = list(self.sets_elems[f[0]])
                    else:
                        members = [int(f[0]) - 1]
                    face = int(f[1][1:])            # 'S3' -> 3
                    for key in self.elems:
                        el = self.elems[key]
                        rows = np.nonzero(np.isin(el[:, 0], members))[0]
                        entries.append((el[rows, 0], face - 1))
                self.surfaces[params["name"]] = entries

    class Materials:
        """Density, type (0 linear elastic, 1 Neo-Hookean) and parameters (inp.py:448-483)."""

        def __init__(self) -> None:
            self.type: int = None
            self.mat_para: list = None
            self.density: float = 0.0

        def read(self, material_blocks):
            for name, params, data in material_blocks:
                if name == "density":
                    self.density = float(data[0].split(",")[0])
                elif name == "hyperelastic":
                    model = [k for k in params if k not in ("neo hooke", "type", "moduli")]
                    if model:
                        raise NotImplementedError("*Hyperelastic, %s: only neo hooke is on the B200 path"
                                                  % ", ".join(model))
                    # every number of the line, the first two as (mu, kappa) = (2 C10, 2 / D1)
                    v = [float(t) for t in data[0].split(",") if t.strip()]
                    self.type = 1
                    self.mat_para = [2.0 * v[0], 2.0 / v[1]] + v[2:]
                elif name == "elastic":
                    self.type = 0
                    self.mat_para = [float(t) for t in data[0].split(",") if t.strip()]

    class Assembly:
        """Instances (part, 4x4 placement), assembly-level node and element
        sets and nodes (inp.py:508-701)."""

        def __init__(self) -> None:
            self.instances: dict = {}
            self.sets_nodes: dict = {}
            self.sets_elems: dict = {}
            self.nodes: torch.Tensor = None

        def read(self, assembly_blocks):
            for name, params, data in assembly_blocks:
                if name == "instance":
                    self.instances[params["name"]] = (params.get("part"), self._placement(data))
                elif name == "nset":
                    self.sets_nodes[params["nset"]] = _label_set(params, data, self.sets_nodes)
                elif name == "elset":
                    # keyed by the bare set name, `instance=` or not: the
                    # reference's split of the keyword line at every '='
                    # (inp.py:638-651) never sees an 'instance=' field
                    self.sets_elems[params["elset"]] = _label_set(params, data, self.sets_elems)
                elif name == "node" and data:
                    self.nodes = torch.tensor([[float(t) for t in row.split(",") if t.strip()] for row in data])
                    self.nodes[:, 0] -= 1

        @staticmethod
        def _placement(data):
            """4x4 placement of an instance: the optional first data line is a
            translation; the optional second, a rotation by an angle in degrees
            about the axis through two points (applied after the translation,
            about that axis)."""
            T = np.eye(4)
            if data:
                t = [float(x) for x in data[0].split(",") if x.strip()]
                T[:3, 3] = t[:3]
            if len(data) > 1:
                r = [float(x) for x in data[1].split(",") if x.strip()]
                a, b, deg = np.array(r[0:3]), np.array(r[3:6]), r[6]
                u = (b - a) / np.linalg.norm(b - a)
                th = np.radians(deg)
                K = np.array([[0.0, -u[2], u[1]], [u[2], 0.0, -u[0]], [-u[1], u[0], 0.0]])
                Rm = np.cos(th) * np.eye(3) + np.sin(th) * K + (1.0 - np.cos(th)) * np.outer(u, u)
                T[:3, :3] = Rm
                T[:3, 3] += a - Rm @ a
            return T

    def __init__(self) -> None:
        self.part: dict = {}
        self.material: dict = {}
        self.assemble = FEA_INP.Assembly()
        self.disp_result: list = []

    def read_inp(self, path):
        """Read the parts, materials and assembly of an INP file and assign
        each part's elements their section's material (inp.py:831-879)."""
        with open(path) as f:
            self.read_lines(f.readlines())

    def read_lines(self, lines):
        self.part, self.material = {}, {}
        bl = blocks(lines)
        i = 0
        while i < len(bl):
            name, params, _ = bl[i]
            if name == "part":
                j = i + 1
                while j < len(bl) and bl[j][0] != "end part":
                    j += 1
                p = FEA_INP.Parts()
                p.read(bl[i + 1:j])
                self.part[params["name"]] = p
                i = j + 1
                continue
            if name == "assembly":
                j = i + 1
                while j < len(bl) and bl[j][0] != "end assembly":
                    j += 1
                self.assemble = FEA_INP.Assembly()
                self.assemble.read(bl[i + 1:j])
                i = j + 1
                continue
            if name == "material":
                j = i + 1
                while j < len(bl) and bl[j][0] in MATERIAL_OPTIONS:
                    j += 1
                m = FEA_INP.Materials()
                m.read(bl[i + 1:j])
                self.material[params["name"]] = m
                i = j
                continue
            i += 1
        for p in self.part.values():
            # rows: the reference's count of element data lines, widened to
            # every label an element block or a section set names (the
            # reference fails on a section over elements it does not read)
            labels = [int(e[:, 0].max()) + 1 for e in p.elems.values() if e.size]
            labels += [max(p.sets_elems[es]) + 1 for es, _ in p.sections if p.sets_elems.get(es)]
            n = max([p.num_elems_2D + p.num_elems_3D] + labels)
            p.elems_material = -torch.ones([n, 5])
            for elset, mat_name in p.sections:
                index = torch.tensor(sorted(p.sets_elems[elset]), dtype=torch.int64)
                mat = self.material[mat_name]
                if mat.type is None:
                    raise ValueError("material %s of section %s defines no elastic behaviour" % (mat_name, elset))
                p.elems_material[index, 0] = index.to(p.elems_material.dtype)
                p.elems_material[index, 1] = mat.density
                p.elems_material[index, 2] = mat.type
                p.elems_material[index, 3] = mat.mat_para[0]
                p.elems_material[index, 4] = mat.mat_para[1]


def from_inp(inp: FEA_INP, create_instance=True):
    """Build the model of a read INP file (FEA/__init__.py:10-79): one Part
    per INP part with its node sets and element-based surface sets, one
    element group per (element type, material type) with that type's
    elements and the section's material and density, an Instance per part
    when asked, all in a new FEAController's Assembly.  As in the reference,
    a group takes every element of its type (one material type per element
    type is the supported case)."""
    from . import elements, materials
    from .assembly import Assembly
    from .controller import FEAController
    from .part import Instance, Part

    asm = Assembly()
    for part_name, pin in inp.part.items():
        part = Part(pin.nodes[:, 1:])
        for set_name, members in pin.sets_nodes.items():
            part.set_nodes[set_name] = np.unique(np.array(sorted(members), dtype=np.int64))
        asm.add_part(part=part, name=part_name)
        if create_instance:
            asm.add_instance(instance=Instance(part), name=part_name)
        for etype, el in pin.elems.items():
            if etype not in elements.BaseElement._subclasses:
                raise NotImplementedError("element type %s is outside the B200 element path" % etype)
            em = pin.elems_material[torch.from_numpy(el[:, 0])]
            for mtype in em[:, 2].to(torch.int32).unique():
                rows = torch.nonzero(em[:, 2].to(torch.int32) == mtype).reshape(-1)
                mat = materials.initialize_materials(int(mtype), em[rows][:, 3:])
                grp = elements.initialize_element(element_type=etype, elems_index=torch.from_numpy(el[:, 0]),
                                                  elems=torch.from_numpy(el[:, 1:]), part=part)
                grp.set_materials(mat)
                grp.set_density(em[rows][:, 1])
                part.add_element(grp)
        for surface_name, entries in pin.surfaces.items():
            part.add_surface_set(surface_name, [(labels, face) for labels, face in entries])
    fe = FEAController()
    fe.assembly = asm
    return fe
