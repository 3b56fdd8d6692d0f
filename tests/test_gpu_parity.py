"""CUDA path (through the C ABI) against the reference's golden fixtures and the oracle.

Tolerances: element R / K / energy <= 1e-12 relative (2-norm over all
entries); converged displacements <= 1e-8 relative; CSR pattern bit-exact.
"""
import numpy as np
import pytest
import torch

from oracle import fea_oracle as O
from tests.helpers import csr_from_api, fea_model, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12
CASES = [("cfg1", "C3D4"), ("tet3", "C3D4"), ("hex5", "C3D8")]


@pytest.mark.parametrize("name,kind", CASES)
def test_reduced_R_K_energy_vs_golden(golden, name, kind):
    g = golden(name)
    c, e, _ = fea_model(g, kind)
    c.initialize()
    asm = c.assembly
    ip, ix = csr_from_api(asm)
    np.testing.assert_array_equal(ip, g["indptr"])
    np.testing.assert_array_equal(ix, g["indices"])
    state = torch.from_numpy(g["state"]).cuda()
    R, Kidx, Kv = asm.assemble_Stiffness_Matrix(GC=state)
    assert rel(R, g["R"]) < TOL
    assert rel(Kv, g["values"]) < TOL
    assert Kidx.shape == (2, g["values"].shape[0])
    E = asm._total_Potential_Energy(GC=state)
    assert abs(float(E) - float(g["energy"])) <= TOL * abs(float(g["energy"]))
    Rf = asm.assemble_force(GC=state)
    assert rel(Rf, g["R"]) < TOL


@pytest.mark.parametrize("name,kind", [("tet3", "C3D4"), ("hex5", "C3D8")])
def test_element_level_structural_force(golden, name, kind):
    g = golden(name)
    c, e, _ = fea_model(g, kind)
    c.initialize()
    U = c.assembly._GC2RGC(torch.from_numpy(g["state"]).cuda())[0]
    fi, Re, Kidx, Kval = e.structural_Force(U, None)
    np.testing.assert_array_equal(fi.cpu().numpy(), g["elem_force_index"])
    np.testing.assert_array_equal(Kidx.cpu().numpy(), g["elem_K_indices"])
    assert rel(Re, g["elem_R"]) < TOL
    assert rel(Kval, g["elem_K_values"]) < TOL
    fi2, Re2 = e.structural_Force(U, torch.eye(3, dtype=torch.float64), if_onlyforce=True)
    assert rel(Re2, g["elem_R"]) < TOL
    Ee = float(e.potential_Energy(U))
    assert abs(Ee - float(g["elem_energy"])) <= TOL * abs(float(g["elem_energy"]))


def test_newton_hex_converges_to_reference(golden):
    import fea_b200 as F
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8", solver=F.solver.StaticImplicitSolver(rtol=1e-11, maximum_iteration=60))
    c.initialize()
    gc = c.solver.solve()
    assert not isinstance(gc, bool)
    assert rel(gc, g["gc_converged"]) < 1e-8


def test_newton_tet_increments_match_reference(golden):
    import fea_b200 as F
    g = golden("cfg1")
    c, e, load = fea_model(g, "C3D4", solver=F.solver.StaticImplicitSolver(rtol=1e-11, maximum_iteration=60))
    c.initialize()
    gc = c.assembly.GC.clone()
    np.testing.assert_array_equal(gc.cpu().numpy(), g["gc0"])
    for k in range(5):
        load.pressure = float(g["p"]) * (k + 1) / 5
        gc = c.solver.solve(GC0=gc)
        assert not isinstance(gc, bool)
        assert rel(gc, g["gc_increments"][k]) < 1e-8


def test_default_newton_stop_test(golden):
    """With the reference's absolute stop test the solve lands within its tolerance."""
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    gc = c.solver.solve()
    R = c.assembly.assemble_force(GC=gc)
    assert float(R.abs().max()) < 1e-6


def test_lumped_mass_and_explicit_vs_golden(golden):
    import fea_b200 as F
    g = golden("explicit_tet4")
    dt, steps = float(g["dt"]), int(g["steps"])
    T = dt * steps
    c, e, _ = fea_model(g, "C3D4", pressure=False, fixed=False,
                        solver=F.solver.DynamicExplicitSolver(time_end=T * (1 - 1e-9), time_per_storage=0.5 * dt))
    c.initialize()
    assert rel(c.assembly.lumped_mass_inv(), g["minv"]) < 1e-14
    c.solver._deltaT = dt
    c.solver.solve(GC0=torch.zeros_like(c.assembly.GC), GV0=torch.from_numpy(g["gv0"]).cuda())
    s = c.solver
    assert len(s._GC_list) == int(g["n_stored"])
    assert abs(s._time_list[-1] - float(g["time_final"])) < 1e-15
    assert rel(s._GC_list[-1], g["u_final"]) < TOL
    assert rel(s._GV_list[-1], g["v_final"]) < TOL
    assert rel(s._GA_list[-1], g["a_final"]) < TOL


def test_explicit_sparse_storage_matches_per_step_recurrence(golden):
    """Storing rarely advances the same recurrence as storing every step."""
    import fea_b200 as F
    g = golden("explicit_tet4")
    dt, steps = float(g["dt"]), int(g["steps"])
    T = dt * steps
    c, e, _ = fea_model(g, "C3D4", pressure=False, fixed=False,
                        solver=F.solver.DynamicExplicitSolver(time_end=T * (1 - 1e-9), time_per_storage=7.3 * dt))
    c.initialize()
    c.solver._deltaT = dt
    c.solver.solve(GC0=torch.zeros_like(c.assembly.GC), GV0=torch.from_numpy(g["gv0"]).cuda())
    assert rel(c.solver._GC_list[-1], g["u_final"]) < TOL
    assert rel(c.solver._GA_list[-1], g["a_final"]) < TOL


def test_explicit_fp32_variant_close(golden):
    import fea_b200 as F
    g = golden("explicit_tet4")
    dt, steps = float(g["dt"]), int(g["steps"])
    T = dt * steps
    c, e, _ = fea_model(g, "C3D4", pressure=False, fixed=False,
                        solver=F.solver.DynamicExplicitSolver(time_end=T * (1 - 1e-9), time_per_storage=T, fp32=True))
    c.initialize()
    c.solver._deltaT = dt
    c.solver.solve(GC0=torch.zeros_like(c.assembly.GC), GV0=torch.from_numpy(g["gv0"]).cuda())
    # FP32 element force with FP64 nodal sums: 1.35e-5 of the FP64 reference
    # run after the fixture's 40 steps (measured on a B200)
    assert rel(c.solver._GC_list[-1], g["u_final"]) < 3e-5


@pytest.mark.parametrize("kind,dofs", [("C3D8", (0, 1, 2)), ("C3D4", (2,)), ("C3D8", (0, 2))])
def test_random_state_vs_oracle_partial_bcs(kind, dofs):
    """Seeded states, partial Dirichlet sets (rows/cols of single DOFs removed)."""
    import fea_b200 as F
    from tests.helpers import top_faces
    n = 3
    X, el = O.hex_block(n, jitter=0.15, seed=7) if kind == "C3D8" else O.tet_block(n)
    top, faces = top_faces(kind, X.numpy(), el.numpy(), n)
    fixed = torch.nonzero(X[:, 2] < 0.5 / n).flatten().numpy() if kind == "C3D4" else \
        np.arange((n + 1) ** 3)[np.arange((n + 1) ** 3) % (n + 1) == 0]
    m = O.Model(X, [O.Group(kind, el, 1.3, 20.0)], [O.PressureLoad(faces, 0.07)], [(fixed, dofs)])
    part = F.Part(X)
    cls = F.elements.C3D4 if kind == "C3D4" else F.elements.C3D8
    e = cls(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.3, 20.0))
    part.add_element(e)
    part.add_surface_set("top", top)
    part.set_nodes["bottom"] = fixed
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    asm.add_load(F.loads.Pressure("p", "top", 0.07))
    asm.add_boundary(F.boundarys.Boundary_Condition("p", "bottom", indexDoF=list(dofs)))
    asm.initialize()
    gc = torch.randn(asm.GC.shape, generator=torch.Generator().manual_seed(11), dtype=torch.float64) * 0.02
    R, (ip, ix, vv) = m.assemble(gc)
    Rg, Kidx, Kg = asm.assemble_Stiffness_Matrix(GC=gc.cuda())
    np.testing.assert_array_equal(asm.plan.indptr.cpu().numpy(), ip.numpy())
    np.testing.assert_array_equal(asm.plan.indices.cpu().numpy(), ix.numpy())
    assert rel(Rg, R) < TOL
    assert rel(Kg, vv) < TOL
    assert abs(float(asm._total_Potential_Energy(GC=gc.cuda())) - float(m.energy(gc))) < TOL * abs(float(m.energy(gc)))


def test_assembly_deterministic_and_symmetric(golden):
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8", pressure=False)
    c.initialize()
    state = torch.from_numpy(g["state"]).cuda()
    R1, K1 = c.assembly.assemble_csr(state)
    R2, K2 = c.assembly.assemble_csr(state)
    assert torch.equal(R1, R2) and torch.equal(K1, K2)          # bitwise reproducible
    P = c.assembly.plan
    A = torch.sparse_csr_tensor(P.indptr, P.indices.long(), K1, (P.ndof, P.ndof)).to_dense()
    assert float((A - A.T).abs().max()) <= 1e-12 * float(A.abs().max())


@pytest.mark.parametrize("name,kind", [("tet3", "C3D4"), ("hex5", "C3D8")])
def test_tangent_is_derivative_of_residual(golden, name, kind):
    """Central differences of R along a random direction reproduce K d
    (follower pressure included)."""
    g = golden(name)
    c, e, _ = fea_model(g, kind)
    c.initialize()
    A = c.assembly
    x = torch.from_numpy(g["state"]).cuda()
    d = torch.randn(x.shape, generator=torch.Generator().manual_seed(5), dtype=torch.float64).cuda()
    _, K = A.assemble_csr(x)
    Kd = A.plan.spmv(K, d)
    h = 1e-6
    fd = (A.assemble_force(GC=x + h * d) - A.assemble_force(GC=x - h * d)) / (2 * h)
    assert rel(fd, Kd) < 1e-7


def test_rigid_translation_zero_residual(golden):
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8", pressure=False, fixed=False)
    c.initialize()
    t = torch.tensor([0.3, -0.2, 0.1], dtype=torch.float64)
    gc = t.repeat(c.assembly.plan.ndof // 3).cuda()
    R = c.assembly.assemble_force(GC=gc)
    assert float(R.abs().max()) < 1e-13


def test_pcg_solves_reduced_system(golden):
    g = golden("cfg1")
    c, e, _ = fea_model(g, "C3D4")
    c.initialize()
    A = c.assembly
    P = A.plan
    R, K = A.assemble_csr(torch.from_numpy(g["state"]).cuda())
    b = (-R).contiguous()
    x = torch.zeros_like(b)
    it, rr, st = P.pcg(K, b, x, 1e-24, 5000)
    assert st == 0 and rr < 1e-24
    xd = O.direct_solve(torch.from_numpy(g["indptr"]), torch.from_numpy(g["indices"]).long(),
                        K.cpu(), b.cpu())
    assert rel(x, xd) < 1e-9
    # FP32 SpMV inner iterations with FP64 refinement reach the same tolerance
    x2 = torch.zeros_like(b)
    it2, outer, rr2, st2 = P.pcg_mixed(K, P.to_f32(K), b, x2, 1e-24, 1e-6, 20000)
    assert st2 == 0 and rr2 < 1e-24 and outer >= 2
    assert rel(x2, xd) < 1e-9


@pytest.mark.parametrize("kind,dofs", [("C3D8", (0, 2)), ("C3D4", (1,)), ("C3D8", (0, 1, 2))])
def test_node_row_spmv_and_pcg_match_csr(kind, dofs):
    """The node-row SpMV / PCG (shared column list per node) against the plain
    CSR kernels and the oracle's CSR product, with partially fixed nodes
    (rows of 1 and 2 free DOFs) in the pattern."""
    import fea_b200 as F
    n = 4
    X, el = O.hex_block(n, jitter=0.1, seed=2) if kind == "C3D8" else O.tet_block(n)
    fixed = torch.nonzero(X[:, 0] < 1e-9).flatten().numpy()
    part = F.Part(X)
    cls = F.elements.C3D4 if kind == "C3D4" else F.elements.C3D8
    e = cls(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 10.0))
    part.add_element(e)
    part.set_nodes["x0"] = fixed
    part.set_nodes["x1"] = torch.nonzero(X[:, 0] > 1 - 1e-9).flatten().numpy()   # keeps K nonsingular
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    asm.add_boundary(F.boundarys.Boundary_Condition("p", "x0", indexDoF=list(dofs)), "bc0")
    asm.add_boundary(F.boundarys.Boundary_Condition("p", "x1"), "bc1")
    asm.initialize()
    P = asm.plan
    gc = torch.randn(asm.GC.shape, generator=torch.Generator().manual_seed(3), dtype=torch.float64) * 1e-3
    R, K = asm.assemble_csr(gc.cuda())
    v = torch.randn(P.ndof, generator=torch.Generator().manual_seed(4), dtype=torch.float64).cuda()
    y_node = P.spmv(K, v)
    y_csr = P.spmv(K, v, generic=True)
    y_o = O.csr_matvec(P.indptr.cpu(), P.indices.cpu().long(), K.cpu(), v.cpu())
    assert rel(y_node, y_o) < 1e-14 and rel(y_csr, y_o) < 1e-14
    b = (-R).contiguous()
    xs = {}
    for mode in ("node", "csr"):
        x = torch.zeros_like(b)
        it, rr, st = P.pcg(K, b, x, 1e-26, 20000, generic=(mode == "csr"))
        assert st == 0 and rr < 1e-26
        xs[mode] = x
    xd = O.direct_solve(P.indptr.cpu(), P.indices.cpu().long(), K.cpu(), b.cpu())
    assert rel(xs["node"], xd) < 1e-9 and rel(xs["csr"], xd) < 1e-9
    x2 = torch.zeros_like(b)
    it2, outer, rr2, st2 = P.pcg_mixed(K, P.to_f32(K), b, x2, 1e-24, 1e-6, 20000)
    assert st2 == 0 and rel(x2, xd) < 1e-9


def test_reference_conjugate_gradient_semantics(golden):
    """_linear_solver.conjugate_gradient: plain CG on a COO input, squared-ratio stop test."""
    import fea_b200 as F
    g = golden("hex5")
    ip = torch.from_numpy(g["indptr"]); ix = torch.from_numpy(g["indices"]).long(); vv = torch.from_numpy(g["values"])
    rows = torch.repeat_interleave(torch.arange(ip.numel() - 1), ip[1:] - ip[:-1])
    b = -torch.from_numpy(g["R"])
    x = F.solver._linear_solver.conjugate_gradient(torch.stack([rows, ix]).cuda(), vv.cuda(), b.cuda(),
                                                   torch.zeros(0), tol=1e-20, max_iter=20000)
    xo, _ = O.conjugate_gradient(ip, ix, vv, b, tol=1e-20, max_iter=20000)
    assert rel(x, xo) < 1e-8


def _free_block(kind, n, jitter=0.0, rho=1.0):
    """Unit block through the public API, without loads or boundary conditions."""
    import fea_b200 as F
    from tests.test_oracle_known_answers import KAPPA, MU
    X, el = O.hex_block(n, jitter=jitter, seed=9) if kind == "C3D8" else O.tet_block(n)
    part = F.Part(X)
    cls = F.elements.C3D4 if kind == "C3D4" else F.elements.C3D8
    e = cls(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(MU, KAPPA))
    e.set_density(rho)
    part.add_element(e)
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    asm.initialize()
    return asm, X, el


@pytest.mark.parametrize("kind", ["C3D8", "C3D4"])
def test_rigid_rotation_zero_residual(kind):
    """u = (Q - I) X with Q a rotation: F = Q, no stress, R = 0 and energy 0."""
    from tests.test_oracle_known_answers import rotation
    asm, X, _ = _free_block(kind, 3, jitter=0.1 if kind == "C3D8" else 0.0)
    u = (X @ rotation().T - X).reshape(-1).cuda()
    assert float(asm.assemble_force(GC=u).abs().max()) < 1e-13
    R, _, Kv = asm.assemble_Stiffness_Matrix(GC=u)
    assert float(R.abs().max()) < 1e-13 and bool(torch.isfinite(Kv).all())
    assert abs(float(asm._total_Potential_Energy(GC=u))) < 1e-13


@pytest.mark.parametrize("kind", ["C3D8", "C3D4"])
def test_uniaxial_stretch_closed_form(kind):
    """F = diag(lam, 1, 1): the x-force on the face x = 1 is the closed-form P11
    times the face area 1; the block as a whole is in equilibrium."""
    from tests.test_oracle_known_answers import uniaxial_P11, uniaxial_W
    lam = 1.05
    asm, X, _ = _free_block(kind, 3)
    u = torch.zeros_like(X)
    u[:, 0] = (lam - 1.0) * X[:, 0]
    R = asm.assemble_force(GC=u.reshape(-1).cuda()).cpu().reshape(-1, 3)
    P11 = uniaxial_P11(lam)
    face = (X[:, 0] - 1.0).abs() < 1e-12
    assert abs(float(R[face, 0].sum()) - P11) < 1e-12 * P11
    assert abs(float(R[:, 0].sum())) < 1e-12 * P11
    W = uniaxial_W(lam)
    assert abs(float(asm._total_Potential_Energy(GC=u.reshape(-1).cuda())) - W) < 1e-12 * W


def test_patch_test_jittered_c3d8():
    """u = (F - I) X is reproduced exactly by trilinear hexes on a jittered
    block: every interior node is in equilibrium, with and without K."""
    from tests.test_oracle_known_answers import PATCH_F, interior_nodes
    n = 4
    asm, X, _ = _free_block("C3D8", n, jitter=0.15)
    u = (X @ torch.tensor(PATCH_F, dtype=torch.float64).T - X).reshape(-1).cuda()
    R = asm.assemble_force(GC=u).cpu().reshape(-1, 3)
    scale = float(R.abs().max())
    assert scale > 1e-3
    assert float(R[interior_nodes(n)].abs().max()) < 1e-12 * scale
    R2, _, _ = asm.assemble_Stiffness_Matrix(GC=u)
    assert rel(R2, R.reshape(-1)) < TOL


@pytest.mark.parametrize("kind", ["C3D8", "C3D4"])
def test_lumped_mass_totals_rho_volume(kind):
    """Row-sum lumped mass summed per direction = rho * mesh volume, and equal
    to the oracle's lumped mass entry by entry."""
    rho = 2.5
    asm, X, el = _free_block(kind, 3, jitter=0.1 if kind == "C3D8" else 0.0, rho=rho)
    m = (1.0 / asm.lumped_mass_inv()).cpu().reshape(-1, 3)
    _, w, _ = O.preload_gaussian(kind, X, el)
    vol = float(w.sum())
    for d in range(3):
        assert abs(float(m[:, d].sum()) - rho * vol) < 1e-12 * rho * vol
    ref = O.Model(X, [O.Group(kind, el, 1.0, 1.0, rho)], [], []).lumped_mass_inv()
    assert rel(asm.lumped_mass_inv(), ref) < 1e-14


def test_hex_element_residual_stays_in_bounds(golden):
    """hex5 has 125 elements, not a multiple of the 8 elements of a C3D8 CTA:
    the element residual output must hold exactly the golden values and the
    memory after it must stay untouched, on every one of repeated calls."""
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    U = c.assembly._GC2RGC(torch.from_numpy(g["state"]).cuda())[0]
    P = e._group_plan()
    mu, kappa = e.materials.parameters()
    gc = e._gc(U)
    n = 8 * 3 * e._elems.shape[0]
    assert e._elems.shape[0] % 8 != 0
    for _ in range(20):
        buf = torch.full((n + 256,), -7.0, dtype=torch.float64, device="cuda")
        K = torch.full((P.nnz,), float("nan"), dtype=torch.float64, device="cuda")
        P.assemble_volume(0, mu, kappa, gc, K=K, elemR=buf[:n])
        assert bool((buf[n:] == -7.0).all())
        assert rel(buf[:n], g["elem_R"]) < TOL
        assert rel(K, g["elem_K_values"]) < TOL


def test_nvtx_ranges_do_not_change_results(golden):
    """The optional NVTX ranges wrap host calls only: the assembly and PCG
    give the same bits with them on."""
    import fea_b200._trace as T
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    asm = c.assembly
    st = torch.from_numpy(g["state"]).cuda()
    R0, K0 = asm.assemble_csr(st)
    x0 = torch.zeros_like(R0)
    asm.plan.pcg(K0, -R0, x0, 1e-20, 3000)
    old = T.ENABLED
    T.ENABLED = True
    try:
        R1, K1 = asm.assemble_csr(st)
        x1 = torch.zeros_like(R1)
        asm.plan.pcg(K1, -R1, x1, 1e-20, 3000)
    finally:
        T.ENABLED = old
    assert torch.equal(R0, R1) and torch.equal(K0, K1) and torch.equal(x0, x1)


def test_collapsed_c3d8_element_matches_oracle():
    """A C3D8 element with two corners on one node (its top edge collapsed):
    the element kernel stages both blocks the repeated node puts on the
    diagonal, and R, K equal the oracle's."""
    import fea_b200 as F
    X, el = O.hex_block(3, jitter=0.1, seed=5)
    el = el.clone()
    el[13, 6] = el[13, 7]
    fixed = torch.nonzero(X[:, 0] < 1e-9).flatten().numpy()
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 10.0)], [], [(fixed, (0, 1, 2))])
    nfree = int(m.free_mask().sum())
    gc = 0.01 * torch.randn(nfree, generator=torch.Generator().manual_seed(2), dtype=torch.float64)
    Rref, (ip, ix, vref) = m.assemble(gc)
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 10.0))
    part.add_element(e)
    part.set_nodes["fix"] = fixed
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    asm.add_boundary(F.boundarys.Boundary_Condition(instance_name="p", set_nodes_name="fix"), "bc")
    asm.initialize()
    R, K = asm.assemble_csr(gc.cuda())
    np.testing.assert_array_equal(asm.plan.indptr.cpu().numpy(), ip.numpy())
    assert rel(R, Rref) < TOL
    assert rel(K, vref) < TOL


def test_explicit_c3d8_with_partial_clamp_vs_oracle():
    """The explicit step on a jittered C3D8 block (one face clamped in x and
    z only), eight steps from a seeded velocity, against the oracle's
    central-difference loop; FP64 within 1e-12, the FP32 element math within
    1e-4."""
    import fea_b200 as F
    X, el = O.hex_block(4, jitter=0.15, seed=9)
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 20.0))
    e.set_density(1.3)
    part.add_element(e)
    fixed = torch.nonzero(X[:, 0] < 1e-9).flatten().numpy()
    part.set_nodes["fix"] = fixed
    asm = F.Assembly()
    asm.add_part(part, "b")
    asm.add_instance(F.Instance(part), "b")
    asm.add_boundary(F.boundarys.Boundary_Condition("b", "fix", indexDoF=[0, 2]))
    asm.initialize()
    P = asm.plan
    dt = 5e-3                  # h = 0.25, wave speed sqrt((kappa + 4 mu / 3) / rho) = 4.1: dt h^-1 c = 0.08
    v0 = 0.05 * torch.randn(P.ndof, generator=torch.Generator().manual_seed(4), dtype=torch.float64)
    minv = asm.lumped_mass_inv()
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 20.0, 1.3)], [], [(fixed, (0, 2))])
    assert rel(minv, m.lumped_mass_inv()) < 1e-14
    uo, vo, ao = O.explicit_run(m, torch.zeros(P.ndof, dtype=torch.float64), v0, dt, 8)
    for fp32, tol in ((False, TOL), (True, 1e-4)):
        u = torch.zeros(P.ndof, dtype=torch.float64, device="cuda")
        v = v0.cuda()
        vh, acc = torch.empty_like(u), torch.empty_like(u)
        P.explicit_run(0, 1.0, 20.0, minv, dt, 0, u, vh, acc, v, fp32=fp32, init=True)
        P.explicit_run(0, 1.0, 20.0, minv, dt, 8, u, vh, acc, v, fp32=fp32, init=False)
        assert rel(u, uo) < tol and rel(v, vo) < tol and rel(acc, ao) < tol, fp32
