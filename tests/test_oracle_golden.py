"""The CPU oracle against fixtures produced by running the reference itself."""
import numpy as np
import pytest
import torch

from oracle import fea_oracle as O

DT = torch.float64


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def tet_model(g):
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    faces = torch.from_numpy(g["pressure_faces"])
    return O.Model(X, [O.Group("C3D4", el, float(g["mu"]), float(g["kappa"]))],
                   [O.PressureLoad(faces, float(g["p"]))], [(g["fixed"], (0, 1, 2))])


def hex_model(g):
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    faces = torch.from_numpy(g["pressure_faces"])
    return O.Model(X, [O.Group("C3D8", el, float(g["mu"]), float(g["kappa"]))],
                   [O.PressureLoad(faces, float(g["p"]))], [(g["fixed"], (0, 1, 2))])


def test_pressure_faces_match_face_tables(golden):
    """The load's face node lists equal the element face tables (tetrahedral.py:45-64)."""
    g = golden("cfg1")
    el = torch.from_numpy(g["elems"])
    X = torch.from_numpy(g["X"])
    mine = torch.cat([f for _, _, f in O.boundary_faces("C3D4", el, X, 2, 1.0)])
    assert torch.equal(mine, torch.from_numpy(g["pressure_faces"]))


def test_initial_gc_quirk(golden):
    for name, mk in (("cfg1", tet_model), ("hex5", hex_model)):
        g = golden(name)
        m = mk(g)
        np.testing.assert_array_equal(m.initial_gc().numpy(), g["gc0"])


def test_element_pattern_bit_exact(golden):
    for name in ("tet3", "hex5"):
        g = golden(name)
        idx, slot, force = O.element_pattern(torch.from_numpy(g["elems"]))
        np.testing.assert_array_equal(idx.numpy(), g["elem_K_indices"])
        np.testing.assert_array_equal(slot.numpy(), g["elem_slot"])
        np.testing.assert_array_equal(force.numpy(), g["elem_force_index"])


def test_element_residual_tangent_energy(golden):
    for name, kind in (("tet3", "C3D4"), ("hex5", "C3D8")):
        g = golden(name)
        m = tet_model(g) if kind == "C3D4" else hex_model(g)
        U = m.gc_to_u(torch.from_numpy(g["state"]))
        Re, Ke = O.element_residual_tangent(kind, m.X, m.groups[0].elems, U, m.groups[0].mu, m.groups[0].kappa)
        assert rel(Re.reshape(-1), g["elem_R"]) < 1e-13
        idx, slot, _ = O.element_pattern(m.groups[0].elems)
        vals = torch.zeros(idx.shape[1], dtype=DT).scatter_add_(0, slot, Ke.reshape(-1))
        assert rel(vals, g["elem_K_values"]) < 1e-13
        e = O.element_energy(kind, m.X, m.groups[0].elems, U, m.groups[0].mu, m.groups[0].kappa)
        assert abs(float(e) - float(g["elem_energy"])) <= 1e-13 * abs(float(g["elem_energy"]))


def test_element_mass(golden):
    for name, kind in (("tet3", "C3D4"), ("hex5", "C3D8")):
        g = golden(name)
        el = torch.from_numpy(g["elems"])
        Me = O.element_mass(kind, torch.from_numpy(g["X"]), el, 1.0)
        full = torch.zeros(el.shape[1], 3, el.shape[1], 3, el.shape[0], dtype=DT)
        for d in range(3):
            full[:, d, :, d, :] = Me
        idx, slot, _ = O.element_pattern(el)
        vals = torch.zeros(idx.shape[1], dtype=DT).scatter_add_(0, slot, full.reshape(-1))
        np.testing.assert_array_equal(idx.numpy(), g["mass_indices"])
        assert rel(vals, g["mass_values"]) < 1e-14


def test_pressure_load(golden):
    g = golden("hex5")
    m = hex_model(g)
    x = m.X + m.gc_to_u(torch.from_numpy(g["state"]))
    f, k = O.pressure_force_tangent(x, m.pressures[0].faces, m.pressures[0].p)
    assert rel(f.reshape(-1), g["pressure_force"]) < 1e-13
    assert rel(k.reshape(-1), g["pressure_K"]) < 1e-13
    v = O.pressure_volume(x, m.pressures[0].faces)
    assert abs(float(-m.pressures[0].p * v) - float(g["pressure_energy"])) < 1e-13 * abs(float(g["pressure_energy"]))


def test_reduced_assembly_csr(golden):
    for name, mk in (("cfg1", tet_model), ("tet3", tet_model), ("hex5", hex_model)):
        g = golden(name)
        m = mk(g)
        state = torch.from_numpy(g["state"])
        R, (ip, ix, vv) = m.assemble(state)
        np.testing.assert_array_equal(ip.numpy(), g["indptr"])
        np.testing.assert_array_equal(ix.numpy(), g["indices"])
        assert rel(vv, g["values"]) < 1e-13
        assert rel(R, g["R"]) < 1e-13
        assert abs(float(m.energy(state)) - float(g["energy"])) <= 1e-13 * abs(float(g["energy"]))


def test_newton_converged_displacements(golden):
    """Oracle Newton (direct solve) lands on the reference's converged GC."""
    g = golden("hex5")
    m = hex_model(g)
    gc, _ = O.newton_solve(m, m.initial_gc(), rtol=1e-13, max_iter=30)
    assert rel(gc, g["gc_converged"]) < 1e-10
    g = golden("cfg1")
    m = tet_model(g)
    gc = m.initial_gc()
    for k in range(5):
        m.pressures[0].p = float(g["p"]) * (k + 1) / 5
        gc, _ = O.newton_solve(m, gc, rtol=1e-13, max_iter=30)
        assert rel(gc, g["gc_increments"][k]) < 1e-10


def test_explicit_run(golden):
    g = golden("explicit_tet4")
    X = torch.from_numpy(g["X"])
    m = O.Model(X, [O.Group("C3D4", torch.from_numpy(g["elems"]), float(g["mu"]), float(g["kappa"]), float(g["rho"]))])
    assert rel(m.lumped_mass_inv(), g["minv"]) < 1e-14
    n = X.shape[0] * 3
    u, v, a = O.explicit_run(m, torch.zeros(n, dtype=DT), torch.from_numpy(g["gv0"]), float(g["dt"]), int(g["steps"]))
    assert rel(u, g["u_final"]) < 1e-12
    assert rel(v, g["v_final"]) < 1e-12
    assert rel(a, g["a_final"]) < 1e-12


def test_cg_matches_reference_semantics(golden):
    """Jacobi-scaled CG solves the reduced system of the reference."""
    g = golden("hex5")
    ip = torch.from_numpy(g["indptr"]); ix = torch.from_numpy(g["indices"]).long(); vv = torch.from_numpy(g["values"])
    b = -torch.from_numpy(g["R"])
    x, it = O.jacobi_scaled_cg(ip, ix, vv, b, torch.zeros_like(b), tol=1e-24, max_iter=5000)
    r = b - O.csr_matvec(ip, ix, vv, x)
    assert r.norm() / b.norm() < 1e-10
    xd = O.direct_solve(ip, ix, vv, b)
    assert rel(x, xd) < 1e-9


def newmark_model(g):
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    faces = torch.from_numpy(g["pressure_faces"])
    return O.Model(X, [O.Group(str(g["kind"]), el, float(g["mu"]), float(g["kappa"]), float(g["rho"]))],
                   [O.PressureLoad(faces, float(g["p"]))], [(g["fixed"], (0, 1, 2))])


NEWMARK = ["newmark_tet2", "newmark_hex2"]


@pytest.mark.parametrize("name", NEWMARK)
def test_consistent_mass(golden, name):
    """Reduced consistent mass of the reference (assembly.py:421-443), summed."""
    g = golden(name)
    M = newmark_model(g).mass_matrix()
    M.sum_duplicates()
    M.sort_indices()
    np.testing.assert_array_equal(M.indptr, g["mass_indptr"])
    np.testing.assert_array_equal(M.indices, g["mass_indices"])
    assert rel(M.data, g["mass_values"]) < 1e-14


@pytest.mark.parametrize("name", NEWMARK)
def test_newmark_run(golden, name):
    """Implicit Newmark histories of the reference's DynamicImplicitSolver,
    including its initial acceleration M a0 = R(gc0)."""
    g = golden(name)
    m = newmark_model(g)
    n = g["GC"].shape[1]
    z = torch.zeros(n, dtype=DT)
    GC, GV, GA = O.newmark_run(m, z, z, float(g["dt"]), int(g["steps"]), tol_error=float(g["tol"]))
    assert len(GC) == g["GC"].shape[0]
    for k in range(len(GC)):
        assert rel(GC[k], g["GC"][k]) < 1e-10 or np.abs(g["GC"][k]).max() < 1e-15
        assert rel(GV[k], g["GV"][k]) < 1e-10 or np.abs(g["GV"][k]).max() < 1e-15
        assert rel(GA[k], g["GA"][k]) < 1e-10


def rotated_model(g):
    """Two instances of the rot_hex3 part as one oracle model: instance a at
    the part's nodes, instance b at R X + t (elements and pressure faces of
    b shifted by the part's node count)."""
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    R = torch.from_numpy(g["rotation_matrix"])
    Xb = X @ R.T + torch.from_numpy(g["translation"])
    N = X.shape[0]
    end = torch.from_numpy(g["end_elems"])
    fa = el[end][:, [1, 2, 6, 5]]
    mu, kappa, p = float(g["mu"]), float(g["kappa"]), float(g["p"])
    return O.Model(torch.cat([X, Xb]), [O.Group("C3D8", el, mu, kappa), O.Group("C3D8", el + N, mu, kappa)],
                   [O.PressureLoad(fa, p), O.PressureLoad(fa + N, p)],
                   [(g["fixed"], (0, 1, 2)), (g["fixed"] + N, (0, 1, 2))])


def test_rotated_instances_as_assembly_frame_coordinates(golden):
    """A rotated, translated instance evaluated on R X + t with the
    assembly-frame displacement gives the reference's rotated element
    outputs: reduced R, K and energy of the two-instance model."""
    g = golden("rot_hex3")
    m = rotated_model(g)
    state = torch.from_numpy(g["state"])
    R, (ip, ix, v) = m.assemble(state)
    np.testing.assert_array_equal(ip.numpy(), g["indptr"])
    np.testing.assert_array_equal(ix.numpy(), g["indices"])
    assert rel(R, g["R"]) < 1e-13 and rel(v, g["values"]) < 1e-13
    assert abs(float(m.energy(state)) - float(g["energy"])) <= 1e-13 * abs(float(g["energy"]))
    Rc, _ = m.assemble(torch.from_numpy(g["gc_converged"]), want_K=False)
    assert float(Rc.abs().max()) < 1e-12


def test_explicit_with_pressure_and_two_groups(golden):
    g = golden("explicit_loaded")
    X = torch.from_numpy(g["X"])
    (mu0, k0), (mu1, k1) = g["mats"]
    rho = float(g["rho"])
    m = O.Model(X, [O.Group("C3D4", torch.from_numpy(g["elems0"]), float(mu0), float(k0), rho),
                    O.Group("C3D4", torch.from_numpy(g["elems1"]), float(mu1), float(k1), rho)],
                [O.PressureLoad(torch.from_numpy(g["pressure_faces"]), float(g["p"]))], [(g["fixed"], (0, 1, 2))])
    assert rel(m.lumped_mass_inv(), g["minv"]) < 1e-14
    gv0 = torch.from_numpy(g["gv0"])
    u, v, a = O.explicit_run(m, torch.zeros_like(gv0), gv0, float(g["dt"]), int(g["steps"]))
    assert rel(u, g["u_final"]) < 1e-12 and rel(v, g["v_final"]) < 1e-12 and rel(a, g["a_final"]) < 1e-12


def couple_model(g):
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    base = O.Model(X, [O.Group("C3D8", el, float(g["mu"]), float(g["kappa"]))], [], [(g["fixed"], (0, 1, 2))])
    return O.CoupledModel(base, g["top"], torch.from_numpy(g["rp"]), torch.from_numpy(g["force"]),
                          torch.from_numpy(g["moment"]))


def test_couple_constraint_vs_reference(golden):
    """Tied nodes following a reference point (Couple), with a force and a
    moment on the point: reduced R, K and energy at a state with a finite
    rotation, and the reference's converged solution in equilibrium."""
    g = golden("couple_hex3")
    m = couple_model(g)
    state = torch.from_numpy(g["state"])
    np.testing.assert_allclose(m.node_u(state).numpy(), g["rgc_state"][:3 * g["X"].shape[0]], rtol=0, atol=1e-15)
    R, (ip, ix, v) = m.assemble(state)
    np.testing.assert_array_equal(ip.numpy(), g["indptr"])
    np.testing.assert_array_equal(ix.numpy(), g["indices"])
    assert rel(R, g["R"]) < 1e-13 and rel(v, g["values"]) < 1e-13
    assert abs(float(m.energy(state)) - float(g["energy"])) <= 1e-13 * abs(float(g["energy"]))
    Rc, _ = m.assemble(torch.from_numpy(g["gc_converged"]))
    assert float(Rc.abs().max()) < 1e-12
