"""Rotated instances and explicit dynamics with loads, through the CUDA path,
against fixtures produced by running the reference itself.

- rot_hex3: two instances of one jittered C3D8 part, one rotated and
  translated; reduced R, K, energy and residual (<= 1e-12), the converged
  Newton solution (<= 1e-8), the element-level outputs with the instance's
  rotation matrix, the Instance API's energy and mass, and the residual VJP
  against the reference's autograd (<= 1e-12).
- explicit_loaded: DynamicExplicitSolver with two element groups and a
  pressure load (the reference's loop, dynamic_explicit.py:66-145), <= 1e-12.
"""
import numpy as np
import pytest
import torch

from tests.helpers import csr_from_api, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rotated_fea(g, solver=None):
    import fea_b200 as F
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(float(g["mu"]), float(g["kappa"])))
    part.add_element(e)
    part.set_nodes["clamp"] = g["fixed"]
    part.add_surface_set("end", [(g["end_elems"], 3)])
    asm = F.Assembly()
    asm.add_part(part, "p")
    ia, ib = F.Instance(part), F.Instance(part)
    ib._rotation = torch.from_numpy(g["rotation"])
    ib._translation = torch.from_numpy(g["translation"])
    asm.add_instance(ia, "a")
    asm.add_instance(ib, "b")
    for nm in ("a", "b"):
        asm.add_load(F.loads.Pressure(instance_name=nm, surface_set="end", pressure=float(g["p"])), "p_" + nm)
        asm.add_boundary(F.boundarys.Boundary_Condition(instance_name=nm, set_nodes_name="clamp"), "bc_" + nm)
    c = F.FEAController()
    c.assembly = asm
    c.solver = solver if solver is not None else F.solver.StaticImplicitSolver()
    c.initialize()
    return c, e, ib


def test_rotated_instance_reduced_system(golden):
    g = golden("rot_hex3")
    c, e, ib = rotated_fea(g)
    asm = c.assembly
    assert torch.allclose(ib.rotation_matrix, torch.from_numpy(g["rotation_matrix"]), rtol=0, atol=1e-15)
    np.testing.assert_array_equal(asm.GC.cpu().numpy(), g["gc0"])
    ip, ix = csr_from_api(asm)
    np.testing.assert_array_equal(ip, g["indptr"])
    np.testing.assert_array_equal(ix, g["indices"])
    state = torch.from_numpy(g["state"]).cuda()
    R, Kidx, Kv = asm.assemble_Stiffness_Matrix(GC=state)
    assert rel(R, g["R"]) < TOL and rel(Kv, g["values"]) < TOL
    assert rel(asm.assemble_force(GC=state), g["force"]) < TOL
    E = float(asm._total_Potential_Energy(GC=state))
    assert abs(E - float(g["energy"])) <= TOL * abs(float(g["energy"]))


def test_rotated_instance_newton_converges_to_reference(golden):
    import fea_b200 as F
    g = golden("rot_hex3")
    c, e, ib = rotated_fea(g, solver=F.solver.StaticImplicitSolver(rtol=1e-11, maximum_iteration=60))
    gc = c.solver.solve()
    assert not isinstance(gc, bool)
    assert rel(gc, g["gc_converged"]) < 1e-8


def test_rotated_instance_element_and_instance_api(golden):
    g = golden("rot_hex3")
    c, e, ib = rotated_fea(g)
    Ub = torch.from_numpy(g["Ub"]).cuda()
    fi, Re, Kidx, Kval = e.structural_Force(Ub, ib.rotation_matrix)
    np.testing.assert_array_equal(fi.cpu().numpy(), g["elem_force_index"])
    np.testing.assert_array_equal(Kidx.cpu().numpy(), g["elem_K_indices"])
    assert rel(Re, g["elem_R"]) < TOL and rel(Kval, g["elem_K_values"]) < TOL
    fi2, Re2 = e.structural_Force(Ub, ib.rotation_matrix, if_onlyforce=True)
    assert rel(Re2, g["elem_R"]) < TOL
    RGC = c.assembly._GC2RGC(torch.from_numpy(g["state"]).cuda())
    Eb = float(ib.potential_energy(RGC))
    assert abs(Eb - float(g["inst_energy"])) <= TOL * abs(float(g["inst_energy"]))
    ri, rv, ki, kv = ib.structural_stiffness(RGC)
    assert rel(rv, g["elem_R"]) < TOL and rel(kv, g["elem_K_values"]) < TOL
    assert int(ri.min()) == ib._index_start
    Mi, Mv = ib.get_mass_matrix()
    np.testing.assert_array_equal(Mi.cpu().numpy(), g["inst_mass_indices"])
    assert rel(Mv, g["inst_mass_values"]) < 1e-13


def test_rotated_instance_residual_vjp(golden):
    """lam . dR/dX with respect to the part's nodes (shared by both
    instances: the sum of the two instance blocks) and lam . dR/dmu."""
    from fea_b200 import adjoint
    g = golden("rot_hex3")
    c, e, ib = rotated_fea(g)
    gc = torch.from_numpy(g["gc_converged"]).cuda()
    lam = torch.from_numpy(g["adj_lambda"]).cuda()
    dX, dmu = adjoint.residual_vjp(c.assembly, gc, lam)
    N = g["X"].shape[0]
    assert rel(dX[:N] + dX[N:], g["adj_gX"]) < TOL
    assert abs(float(sum(dmu)) - float(g["adj_gmu"])) <= TOL * abs(float(g["adj_gmu"]))


def test_explicit_with_pressure_and_two_groups(golden):
    import fea_b200 as F
    g = golden("explicit_loaded")
    X = torch.from_numpy(g["X"])
    part = F.Part(X)
    cell = g["cell"]
    for k, key in enumerate(("elems0", "elems1")):
        mu, kappa = g["mats"][k]
        e = F.elements.C3D4(elems=torch.from_numpy(g[key]), elems_index=torch.from_numpy(np.nonzero(cell % 2 == k)[0]),
                            part=part)
        e.set_materials(F.materials.NeoHookean(float(mu), float(kappa)))
        e.set_density(float(g["rho"]))
        part.add_element(e, "g%d" % k)
    fid = g["face_id"]
    part.add_surface_set("top", [(g["face_elem"][fid == f], int(f)) for f in np.unique(fid)])
    part.set_nodes["bottom"] = g["fixed"]
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    asm.add_load(F.loads.Pressure(instance_name="p", surface_set="top", pressure=float(g["p"])), "pressure")
    asm.add_boundary(F.boundarys.Boundary_Condition(instance_name="p", set_nodes_name="bottom"), "bc")
    dt, steps = float(g["dt"]), int(g["steps"])
    T = dt * steps
    c = F.FEAController()
    c.assembly = asm
    c.solver = F.solver.DynamicExplicitSolver(time_end=T * (1 - 1e-9), time_per_storage=0.5 * dt)
    c.initialize()
    P = asm.plan
    assert [tuple(f.conn.shape) for f in P.faces] == [tuple(g["pressure_faces"].shape)]
    assert rel(asm.lumped_mass_inv(), g["minv"]) < 1e-14
    c.solver._deltaT = dt
    c.solver.solve(GC0=torch.zeros_like(asm.GC), GV0=torch.from_numpy(g["gv0"]).cuda())
    s = c.solver
    assert len(s._GC_list) == int(g["n_stored"])
    assert abs(s._time_list[-1] - float(g["time_final"])) < 1e-15
    assert rel(s._GC_list[-1], g["u_final"]) < TOL
    assert rel(s._GV_list[-1], g["v_final"]) < TOL
    assert rel(s._GA_list[-1], g["a_final"]) < TOL
