"""A model read from an Abaqus INP file runs through the CUDA path: the
committed CAE-layout hex sample (tests/golden/inp_hex.inp) read by FEA_INP
and built by from_inp, clamped on its node set and pulled on its
element-based surface, solved by StaticImplicitSolver, gives the
displacements of the oracle's Newton on the same mesh, set, faces and
material (<= 1e-8 relative, both converged to ||R|| <= 1e-11 ||R0||)."""
import os

import numpy as np
import pytest
import torch

from oracle import fea_oracle as O
from tests.helpers import rel

pytestmark = pytest.mark.gpu

SAMPLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "inp_hex.inp")


def test_inp_model_solves_like_the_oracle():
    import fea_b200 as F
    from fea_b200.elements import FACES
    old = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        inp = F.FEA_INP()
        inp.read_inp(SAMPLE)
    finally:
        torch.set_default_dtype(old)
    fe = F.from_inp(inp)
    p = -0.02
    fe.assembly.add_load(F.loads.Pressure(instance_name="block", surface_set="end", pressure=p), "pull")
    fe.assembly.add_boundary(F.boundarys.Boundary_Condition(instance_name="block", set_nodes_name="clamp"), "clamp")
    fe.solver = F.solver.StaticImplicitSolver(rtol=1e-11, maximum_iteration=60)
    gc = fe.solve()
    assert not isinstance(gc, bool)

    part = inp.part["block"]
    X = part.nodes[:, 1:].to(torch.float64)
    el = torch.from_numpy(part.elems["C3D8"][:, 1:])
    (labels, face), = part.surfaces["end"]
    faces = el[torch.from_numpy(labels)][:, FACES["C3D8"][face]]
    clamp = np.array(sorted(part.sets_nodes["clamp"]))
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 50.0, 2.5)], [O.PressureLoad(faces, p)], [(clamp, (0, 1, 2))])
    ref, _ = O.newton_solve(m, m.initial_gc(), rtol=1e-11, max_iter=60)
    assert rel(gc, ref) < 1e-8
