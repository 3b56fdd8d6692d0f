"""Couple constraint (nodes tied to a reference point, couple.py:7-282) with a
concentrated force and a moment on the point, through the CUDA path, against
the reference's own run (tests/golden/couple_hex3.npz): the reduced R, K
(pattern bit-exact, values <= 1e-12), energy, the tied nodes' displacement,
and the converged Newton solution (<= 1e-8)."""
import numpy as np
import pytest
import torch

from tests.helpers import csr_from_api, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


def couple_fea(g, solver=None):
    import fea_b200 as F
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(float(g["mu"]), float(g["kappa"])))
    part.add_element(e)
    part.set_nodes["bottom"] = g["fixed"]
    part.set_nodes["top"] = g["top"]
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    rp = asm.add_reference_point(F.ReferencePoint(g["rp"].tolist()))
    asm.add_constraint(F.constraints.Couple(instance_name="p", set_nodes_name="top", rp_name=rp))
    asm.add_load(F.loads.Concentrate_Force(rp_name=rp, force=g["force"].tolist()), "f")
    asm.add_load(F.loads.Moment(rp_name=rp, moment=g["moment"].tolist()), "m")
    asm.add_boundary(F.boundarys.Boundary_Condition(instance_name="p", set_nodes_name="bottom"), "bc")
    c = F.FEAController()
    c.assembly = asm
    c.solver = solver if solver is not None else F.solver.StaticImplicitSolver()
    c.initialize()
    return c


def test_couple_reduced_system_vs_reference(golden):
    g = golden("couple_hex3")
    c = couple_fea(g)
    asm = c.assembly
    np.testing.assert_array_equal(asm.GC.cpu().numpy(), g["gc0"])
    S = asm.system
    np.testing.assert_array_equal(S.indptr.cpu().numpy(), g["indptr"])
    np.testing.assert_array_equal(S.indices.cpu().numpy(), g["indices"])
    state = torch.from_numpy(g["state"]).cuda()
    rgc = torch.cat([r.reshape(-1) for r in asm._GC2RGC(state)])
    assert float((rgc.cpu() - torch.from_numpy(g["rgc_state"])).abs().max()) < 1e-15
    R, Kidx, Kv = asm.assemble_Stiffness_Matrix(GC=state)
    assert rel(R, g["R"]) < TOL and rel(Kv, g["values"]) < TOL
    assert rel(asm.assemble_force(GC=state), g["force_R"]) < TOL
    E = float(asm._total_Potential_Energy(GC=state))
    assert abs(E - float(g["energy"])) <= TOL * abs(float(g["energy"]))


def test_couple_newton_converges_to_reference(golden):
    import fea_b200 as F
    g = golden("couple_hex3")
    c = couple_fea(g, solver=F.solver.StaticImplicitSolver(rtol=1e-11, maximum_iteration=60))
    gc = c.solver.solve()
    assert not isinstance(gc, bool)
    assert rel(gc, g["gc_converged"]) < 1e-8
