"""INP reader and from_inp (CPU): the committed sample files
(tests/golden/inp_samples.py) read by ``fea_b200.FEA_INP`` agree with what
the reference's FEA_INP.read_inp and from_inp produced from the same files
(fixtures written by make_golden.py --case inp); the model they build runs
through the host plan to the oracle's CSR; format variants the reference's
fixed-format matching skips are read; unsupported inputs raise.
"""
import contextlib
import os

import numpy as np
import pytest
import torch

from oracle import fea_oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SAMPLES = ["inp_hex", "inp_mixed"]


@contextlib.contextmanager
def default_dtype(dt):
    old = torch.get_default_dtype()
    torch.set_default_dtype(dt)
    try:
        yield
    finally:
        torch.set_default_dtype(old)


def read(name, dt=torch.float64):
    from fea_b200 import FEA_INP
    inp = FEA_INP()
    with default_dtype(dt):
        inp.read_inp(os.path.join(HERE, name + ".inp"))
    return inp


def fixture(name):
    return np.load(os.path.join(HERE, name + ".npz"))


@pytest.mark.parametrize("name", SAMPLES)
def test_reader_matches_reference(name):
    inp, g = read(name), fixture(name)
    for pn, p in inp.part.items():
        assert np.array_equal(p.nodes.numpy(), g["nodes:%s" % pn])
        assert list(p.elems.keys()) == list(g["elemtypes:%s" % pn])
        for t, e in p.elems.items():
            assert e.dtype == np.int64 and np.array_equal(e, g["elems:%s:%s" % (pn, t)])
        want = {k.split(":", 2)[2] for k in g.files if k.startswith("nset:%s:" % pn)}
        assert set(p.sets_nodes) == want
        for sn, m in p.sets_nodes.items():
            assert np.array_equal(np.array(sorted(m)), g["nset:%s:%s" % (pn, sn)])
        want = {k.split(":", 2)[2] for k in g.files if k.startswith("elset:%s:" % pn)}
        assert set(p.sets_elems) == want
        for sn, m in p.sets_elems.items():
            assert np.array_equal(np.array(sorted(m)), g["elset:%s:%s" % (pn, sn)])
        assert list(p.surfaces.keys()) == list(g["surfaces:%s" % pn])
        for sn, entries in p.surfaces.items():
            assert len(entries) == int(g["surfn:%s:%s" % (pn, sn)])
            for k, (labels, face) in enumerate(entries):
                assert np.array_equal(labels, g["surf:%s:%s:%d:labels" % (pn, sn, k)])
                assert face == int(g["surf:%s:%s:%d:face" % (pn, sn, k)])
        assert [list(s) for s in p.sections] == g["sections:%s" % pn].tolist()
        assert np.array_equal(p.elems_material.numpy(), g["elems_material:%s" % pn])
    mats = {k.split(":", 1)[1] for k in g.files if k.startswith("material:")}
    assert set(inp.material) == mats
    for mn, m in inp.material.items():
        assert [m.type, m.mat_para[0], m.mat_para[1], m.density] == g["material:%s" % mn].tolist()
    inst = {k.split(":", 1)[1] for k in g.files if k.startswith("instance:")}
    assert set(inp.assemble.instances) == inst
    for iname, (pname, T) in inp.assemble.instances.items():
        assert pname == str(g["instancepart:%s" % iname])
        assert np.allclose(T, g["instance:%s" % iname], rtol=0, atol=1e-14)
    for kind, sets in (("asm_nset", inp.assemble.sets_nodes), ("asm_elset", inp.assemble.sets_elems)):
        assert set(sets) == {k.split(":", 1)[1] for k in g.files if k.startswith(kind + ":")}
        for sn, m in sets.items():
            assert np.array_equal(np.array(sorted(m)), g["%s:%s" % (kind, sn)])


def test_nodes_follow_the_default_dtype():
    """As in the reference, coordinates are parsed in torch's default dtype."""
    g = fixture("inp_hex")
    p = read("inp_hex", torch.float32).part["block"]
    assert p.nodes.dtype == torch.float32
    assert np.array_equal(p.nodes.numpy(), g["nodes:block"].astype(np.float32))


@pytest.mark.parametrize("name", SAMPLES)
def test_from_inp_builds_the_reference_model(name):
    import fea_b200 as F
    g = fixture(name)
    with default_dtype(torch.float64):
        fe = F.from_inp(read(name))
    for pn, part in fe.assembly._parts.items():
        assert torch.equal(part.nodes, torch.from_numpy(g["nodes:%s" % pn][:, 1:]))
        assert set(part.set_nodes) == {k.split(":", 2)[2] for k in g.files if k.startswith("pset:%s:" % pn)}
        for sn, m in part.set_nodes.items():
            assert np.array_equal(m, g["pset:%s:%s" % (pn, sn)])
        assert len(part.elems) == int(g["ngroups:%s" % pn])
        for k, e in enumerate(part.elems.values()):
            gk = "group:%s:%d" % (pn, k)
            assert type(e).__name__ == str(g[gk + ":type"])
            assert np.array_equal(e._elems_index.numpy(), g[gk + ":elems_index"])
            assert np.array_equal(e._elems.numpy(), g[gk + ":elems"])
            mu, kappa = e.materials.parameters()
            assert (mu, kappa) == (float(g[gk + ":mu"]), float(g[gk + ":kappa"]))
            assert np.all(g[gk + ":density"] == float(e.density))
        assert pn in fe.assembly._instances


def test_surface_of_the_hex_sample_is_the_x_max_face():
    """The element-based surface 'end' (set _end_S4, face S4) extracts the
    Q4 faces on x = max, outward (C3D8 face 3: nodes 1, 2, 6, 5)."""
    import fea_b200 as F
    with default_dtype(torch.float64):
        fe = F.from_inp(read("inp_hex"))
    part = fe.assembly._parts["block"]
    (surf,) = part.extract_surfaces("end")
    n = 3
    X, el = O.hex_block(n, jitter=0.1, seed=4)
    end = torch.arange(el.shape[0])[torch.arange(el.shape[0]) // (n * n) == n - 1]
    assert surf.kind == "Q4" and torch.equal(surf._elems, el[end][:, [1, 2, 6, 5]])


def test_parsed_model_plans_the_oracle_csr():
    """The mesh and clamp set read from the hex sample give, through the host
    plan, the reduced CSR the oracle assembles for the same model."""
    from fea_b200.plan import HostPlan, KIND
    p = read("inp_hex").part["block"]
    X = p.nodes[:, 1:].to(torch.float64)
    el = torch.from_numpy(p.elems["C3D8"][:, 1:])
    clamp = np.array(sorted(p.sets_nodes["clamp"]))
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 50.0)], [], [(clamp, (0, 1, 2))])
    from fea_b200 import _lib as L
    mask = np.full(X.shape[0], 7, np.uint8)
    mask[clamp] = 0
    hp = HostPlan(X.shape[0], mask, [(KIND["C3D8"], el.numpy())], [])
    _, (ip, ix, _) = m.assemble(m.initial_gc())
    assert clamp.size == 16 and hp.scalar(L.FEA_S_NDOF) == 3 * (X.shape[0] - 16)
    assert np.array_equal(hp.array(L.FEA_A_INDPTR), ip.numpy())
    assert np.array_equal(hp.array(L.FEA_A_INDICES), ix.numpy())


VARIANT = """** keyword case, parameter order, blank and comment lines
*HEADING
*Part, NAME=p

*NODE
1, 0., 0., 0.
2, 1., 0., 0.
3, 0., 1., 0.
4, 0., 0., 1.
5, 1., 1., 1.
** a second node block
*Node
6, 2., 2., 2.
*element, type=c3d4, elset=first
1, 1, 2, 3,
4
*Element, type=C3D4
2, 2, 3, 4, 5
*Nset, generate, nset=gen
1, 3, 2
5, 6
*Elset, elset=both
first, 2
*Surface, name=s, type=ELEMENT
2, S3
*Solid Section, material=m, elset=both
*End Part
*Material, name=m
*Density
3.,
*Hyperelastic, neo hooke
0.25, 0.5
*Step, name=Step-1
"""


def test_format_variants_the_reference_skips():
    from fea_b200 import FEA_INP
    inp = FEA_INP()
    with default_dtype(torch.float64):
        inp.read_lines(VARIANT.splitlines(True))
    p = inp.part["p"]
    assert p.nodes.shape == (6, 4) and p.nodes[5, 0] == 5 and p.nodes[5, 1] == 2.0
    assert np.array_equal(p.elems["C3D4"], np.array([[0, 0, 1, 2, 3], [1, 1, 2, 3, 4]]))
    assert p.sets_elems["first"] == {0} and p.sets_elems["both"] == {0, 1}
    assert p.sets_nodes["gen"] == {0, 2, 4, 5}
    assert len(p.surfaces["s"]) == 1
    labels, face = p.surfaces["s"][0]
    assert labels.tolist() == [1] and face == 2
    assert p.sections == [["both", "m"]]
    m = inp.material["m"]
    assert (m.type, m.mat_para, m.density) == (1, [0.5, 4.0], 3.0)
    # rows = element data lines (3: the first element takes two), as the reference counts them
    assert p.elems_material[:, 1:].tolist() == [[3.0, 1.0, 0.5, 4.0]] * 2 + [[-1.0] * 4]


def test_unsupported_inputs_raise():
    import fea_b200 as F
    inp = F.FEA_INP()
    with pytest.raises(NotImplementedError):
        inp.read_lines(["*Material, name=m\n", "*Hyperelastic, mooney-rivlin\n", "0.3, 0.1, 0.02\n"])
    inp.read_lines(["*Part, name=p\n", "*Node\n"] + ["%d, %d., 0., 0.\n" % (i + 1, i) for i in range(10)]
                   + ["*Element, type=C3D10\n", "1, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10\n",
                      "*Elset, elset=all\n", "1\n", "*Solid Section, elset=all, material=m\n", "*End Part\n",
                      "*Material, name=m\n", "*Hyperelastic, neo hooke\n", "0.5, 0.1\n"])
    assert inp.part["p"].elems["C3D10"].shape == (1, 11)
    with pytest.raises(NotImplementedError):
        F.from_inp(inp)
    with pytest.raises(ValueError):
        inp.read_lines(["*Part, name=p\n", "*Node\n", "1, 0., 0., 0.\n", "*Element, type=C3D4\n",
                        "1, 1, 1, 1, 1\n", "*Elset, elset=all\n", "1\n",
                        "*Solid Section, elset=all, material=m\n", "*End Part\n",
                        "*Material, name=m\n", "*Density\n", "1.,\n"])
