"""Generate golden fixtures by running the reference package sssnnn7119/FEA.

Run in a container where the reference source tree is available:

    python tests/golden/make_golden.py --ref <path of the reference source tree>

The reference is imported unmodified, with three stub modules injected first:
``tkinter`` and ``turtle`` (stray imports at FEA/assemble/loads/contact.py:1-2)
and ``pypardiso`` (its CPU Newton path always calls ``pypardiso.spsolve``,
FEA/solver/static_implicit.py:384-387; the stub maps it to scipy's direct
solver).  Everything runs on CPU in float64.  The fixtures are small ``.npz``
files next to this script; the tests read them and never need the reference.
"""
from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def import_reference(path):
    import scipy.sparse.linalg as spla
    shim = types.ModuleType("pypardiso")
    shim.spsolve = lambda A, b: spla.spsolve(A.tocsc(), b)
    sys.modules["pypardiso"] = shim
    for name in ("tkinter", "turtle"):
        m = types.ModuleType(name)
        m.N = m.color = m.pd = None
        sys.modules[name] = m
    sys.path.insert(0, path)
    torch.set_default_dtype(torch.float64)
    import FEA  # noqa: E402
    return FEA


def build_reference(FEA, X, groups, pressures, fixed):
    """Build a reference controller: one part/instance 'p'.

    groups: list of (kind, elems, mu, kappa, rho); pressures: list of
    (surface list [(elem_idx np, face_id)], p); fixed: list of (nodes, dofs).
    """
    part = FEA.Part(X.clone())
    start = 0
    elems_objs = []
    for kind, el, mu, kappa, rho in groups:
        cls = getattr(FEA.elements, kind)
        e = cls(elems=el.clone(), elems_index=torch.arange(start, start + el.shape[0]), part=part)
        e.set_materials(FEA.materials.NeoHookean(torch.tensor(mu), torch.tensor(kappa)))
        e.set_density(torch.tensor([rho]))
        part.add_element(e)
        elems_objs.append(e)
        start += el.shape[0]
    for i, (nodes, dofs) in enumerate(fixed):
        part.set_nodes["fix%d" % i] = np.asarray(nodes)
    loads = []
    for i, (surf, p) in enumerate(pressures):
        part.add_surface_set("surf%d" % i, surf)
    asm = FEA.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(FEA.Instance(part), "p")
    for i, (surf, p) in enumerate(pressures):
        ld = FEA.loads.Pressure(instance_name="p", surface_set="surf%d" % i, pressure=p)
        asm.add_load(ld, "pressure%d" % i)
        loads.append(ld)
    for i, (nodes, dofs) in enumerate(fixed):
        asm.add_boundary(FEA.boundarys.Boundary_Condition(instance_name="p", set_nodes_name="fix%d" % i,
                                                          indexDoF=list(dofs)), "bc%d" % i)
    c = FEA.FEAController()
    c.assembly = asm
    return c, part, elems_objs, loads


def coalesced_csr(R, Ki, Kv):
    n = R.shape[0]
    A = torch.sparse_coo_tensor(Ki, Kv, (n, n)).coalesce().to_sparse_csr()
    return A.crow_indices().numpy(), A.col_indices().numpy().astype(np.int32), A.values().numpy()


def converge(FEA, c, gc0, tol=1e-10):
    """Reference Newton (CPU direct solve) to a tight residual.

    The reference stops on max|R| < 1e-6 measured before its last step
    (static_implicit.py:345-346); solve() is re-entered until the residual at
    the returned point is below ``tol``.
    """
    gc = gc0
    for _ in range(3):
        gc = c.solver.solve(GC0=gc)
        if isinstance(gc, bool):
            raise RuntimeError("reference Newton did not converge")
        R = c.assembly.assemble_Stiffness_Matrix(GC=gc)[0]
        if R.abs().max() < tol:
            break
    # The Armijo test stalls once energy changes reach round-off; finish with
    # plain Newton steps on the reference's own R and K (direct solve).
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    for _ in range(4):
        R, Ki, Kv = c.assembly.assemble_Stiffness_Matrix(GC=gc)
        if R.abs().max() < 1e-14:
            break
        n = R.shape[0]
        A = sp.coo_matrix((Kv.numpy(), (Ki[0].numpy(), Ki[1].numpy())), shape=(n, n)).tocsc()
        gc = gc + torch.from_numpy(spla.spsolve(A, -R.numpy()))
    R = c.assembly.assemble_Stiffness_Matrix(GC=gc)[0]
    return gc, float(R.abs().max())


def case_tet_cube(FEA, O, out, n=10, mu=1.0, kappa=10.0, p=0.05, full_element=False, name="cfg1"):
    """Config-1 style unit cube of Kuhn tets, bottom clamped, top pressure."""
    X, el = O.tet_block(n)
    bottom = torch.nonzero(X[:, 2].abs() < 1e-9).flatten().numpy()
    surf = [(idx.numpy(), fid) for idx, fid, _ in O.boundary_faces("C3D4", el, X, 2, 1.0)]
    c, part, (e,), (ld,) = build_reference(FEA, X, [("C3D4", el, mu, kappa, 1.0)], [(surf, p)], [(bottom, (0, 1, 2))])
    c.solver = FEA.solver.StaticImplicitSolver(tol_error=1e-10)
    c.initialize()
    gc0 = c.assembly.GC.clone()
    res = dict(X=X.numpy(), elems=el.numpy(), fixed=bottom, mu=mu, kappa=kappa, p=p, gc0=gc0.numpy())
    res["face_elem"] = np.concatenate([s[0] for s in surf])
    res["face_id"] = np.concatenate([np.full(len(s[0]), s[1]) for s in surf])
    # Reference pressure faces in the load's own order
    res["pressure_faces"] = torch.cat([s._elems for s in ld.surface_element]).numpy()
    # five load increments p*k/5, each re-entering solve() from the previous GC
    gcs, res_max = [], []
    gc = gc0
    for k in range(1, 6):
        ld.pressure = p * k / 5
        gc, rm = converge(FEA, c, gc)
        gcs.append(gc.numpy().copy())
        res_max.append(rm)
    res["gc_increments"] = np.stack(gcs)
    res["resid_increments"] = np.array(res_max)
    # reduced R, K (coalesced CSR) and energy at a seeded perturbed state
    g = torch.Generator().manual_seed(1)
    gcs_state = torch.from_numpy(gcs[-1]) + 1e-3 * torch.randn(gc0.shape, generator=g)
    R, Ki, Kv = c.assembly.assemble_Stiffness_Matrix(GC=gcs_state)
    ip, ix, vv = coalesced_csr(R, Ki, Kv)
    res.update(state=gcs_state.numpy(), R=R.numpy(), indptr=ip, indices=ix, values=vv,
               energy=float(c.assembly._total_Potential_Energy(GC=gcs_state)),
               force=c.assembly.assemble_force(GC=gcs_state).numpy())
    if full_element:
        U = c.assembly._GC2RGC(gcs_state)[0]
        fi, Re, Kidx, Kval = e.structural_Force(U, None)
        res.update(elem_force_index=fi.numpy(), elem_R=Re.numpy(), elem_K_indices=Kidx.numpy(),
                   elem_K_values=Kval.numpy(), elem_slot=e._index_matrix_coalesce.numpy(),
                   elem_energy=float(e.potential_Energy(U)))
        Mi, Mv = e.get_mass_matrix()
        res.update(mass_indices=Mi.numpy(), mass_values=Mv.numpy())
    np.savez_compressed(os.path.join(out, "%s.npz" % name), **res)
    print(name, "E", el.shape[0], "n", gc0.shape[0], "nnz", vv.shape[0], "final max|R|", res_max)


def case_hex_block(FEA, O, out, n=5, mu=1.0, kappa=50.0, p=-0.02, seed=0, name="hex5"):
    """Config-2 style jittered C3D8 block, x=0 clamped, pressure on x=1 (Q4)."""
    X, el = O.hex_block(n, jitter=0.1, seed=seed)
    h = 1.0 / n
    clamp = torch.nonzero(X[:, 0] < 0.5 * h).flatten().numpy()
    # x=1 face: face id 3 = nodes [1,2,6,5] of each end element (brick.py:192-193)
    xe = X[el][:, [1, 2, 6, 5], 0]
    endel = torch.nonzero(xe.min(dim=1).values > 1 - 0.5 * h).flatten().numpy()
    surf = [(endel, 3)]
    c, part, (e,), (ld,) = build_reference(FEA, X, [("C3D8", el, mu, kappa, 1.0)], [(surf, p)], [(clamp, (0, 1, 2))])
    c.solver = FEA.solver.StaticImplicitSolver(tol_error=1e-10)
    c.initialize()
    gc0 = c.assembly.GC.clone()
    res = dict(X=X.numpy(), elems=el.numpy(), fixed=clamp, mu=mu, kappa=kappa, p=p, gc0=gc0.numpy(),
               end_elems=endel, pressure_faces=torch.cat([s._elems for s in ld.surface_element]).numpy())
    gc, rm = converge(FEA, c, gc0)
    res.update(gc_converged=gc.numpy(), resid_converged=rm)
    g = torch.Generator().manual_seed(2)
    state = gc + 2e-3 * torch.randn(gc.shape, generator=g)
    R, Ki, Kv = c.assembly.assemble_Stiffness_Matrix(GC=state)
    ip, ix, vv = coalesced_csr(R, Ki, Kv)
    U = c.assembly._GC2RGC(state)[0]
    fi, Re, Kidx, Kval = e.structural_Force(U, None)
    Mi, Mv = e.get_mass_matrix()
    res.update(state=state.numpy(), R=R.numpy(), indptr=ip, indices=ix, values=vv,
               energy=float(c.assembly._total_Potential_Energy(GC=state)),
               elem_force_index=fi.numpy(), elem_R=Re.numpy(), elem_K_indices=Kidx.numpy(),
               elem_K_values=Kval.numpy(), elem_slot=e._index_matrix_coalesce.numpy(),
               elem_energy=float(e.potential_Energy(U)), mass_indices=Mi.numpy(), mass_values=Mv.numpy())
    # pressure load alone (force and stiffness values in the load's own order)
    Rf_i, Rf_v, Kf_i, Kf_v = ld.get_stiffness(c.assembly._GC2RGC(state))
    res.update(pressure_force_index=Rf_i.numpy(), pressure_force=Rf_v.numpy(),
               pressure_K_indices=Kf_i.numpy(), pressure_K=Kf_v.numpy(),
               pressure_energy=float(ld.get_potential_energy(c.assembly._GC2RGC(state))))
    # adjoint recipe (tests/gradient_test/test_grad.py:87-99): autograd of
    # (R . lam) with respect to the nodal coordinates and mu, at the converged GC
    lam = torch.randn(gc.shape, generator=torch.Generator().manual_seed(3))
    Xg = part.nodes.clone().requires_grad_(True)
    part.nodes = Xg
    mu_t = torch.tensor(mu, requires_grad=True)
    e.materials.mu = mu_t
    c.initialize()
    Rg = c.assembly.assemble_Stiffness_Matrix(GC=gc)[0]
    gX, gmu = torch.autograd.grad((Rg * lam).sum(), [Xg, mu_t])
    res.update(adj_lambda=lam.numpy(), adj_gX=gX.numpy(), adj_gmu=float(gmu))
    np.savez_compressed(os.path.join(out, "%s.npz" % name), **res)
    print(name, "E", el.shape[0], "n", gc0.shape[0], "nnz", vv.shape[0], "final max|R|", rm)


def case_rotated(FEA, O, out, n=3, mu=1.0, kappa=50.0, p=0.02, name="rot_hex3"):
    """Two instances of one jittered C3D8 block: 'a' in place, 'b' rotated
    (rotation vector ROT) and translated (TRANS); each clamped on its x = 0
    face and loaded by pressure on its x = 1 face (the part's frame).  The
    reduced R, K and energy at a state, the converged GC, instance b's
    element-level outputs (structural_Force with its rotation matrix), its
    energy and mass through the Instance API, and autograd of (R . lam)
    with respect to the part's nodes (both instances) and mu."""
    rot, trans = [0.3, -0.5, 0.7], [1.5, -2.0, 0.5]
    X, el = O.hex_block(n, jitter=0.1, seed=6)
    h = 1.0 / n
    clamp = torch.nonzero(X[:, 0] < 0.5 * h).flatten().numpy()
    xe = X[el][:, [1, 2, 6, 5], 0]
    endel = torch.nonzero(xe.min(dim=1).values > 1 - 0.5 * h).flatten().numpy()
    part = FEA.Part(X.clone())
    e = FEA.elements.C3D8(elems=el.clone(), elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(FEA.materials.NeoHookean(torch.tensor(mu), torch.tensor(kappa)))
    e.set_density(torch.tensor([1.0]))
    part.add_element(e)
    part.set_nodes["clamp"] = clamp
    part.add_surface_set("end", [(endel, 3)])
    asm = FEA.Assembly()
    asm.add_part(part, "p")
    ia, ib = FEA.Instance(part), FEA.Instance(part)
    ib._rotation = torch.tensor(rot)
    ib._translation = torch.tensor(trans)
    asm.add_instance(ia, "a")
    asm.add_instance(ib, "b")
    for nm in ("a", "b"):
        asm.add_load(FEA.loads.Pressure(instance_name=nm, surface_set="end", pressure=p), "p_" + nm)
        asm.add_boundary(FEA.boundarys.Boundary_Condition(instance_name=nm, set_nodes_name="clamp"), "bc_" + nm)
    c = FEA.FEAController()
    c.assembly = asm
    c.solver = FEA.solver.StaticImplicitSolver(tol_error=1e-10)
    c.initialize()
    gc0 = c.assembly.GC.clone()
    res = dict(X=X.numpy(), elems=el.numpy(), fixed=clamp, end_elems=endel, mu=mu, kappa=kappa, p=p,
               rotation=np.array(rot), translation=np.array(trans), gc0=gc0.numpy(),
               rotation_matrix=ib.rotation_matrix.numpy())
    gc, rm = converge(FEA, c, gc0)
    res.update(gc_converged=gc.numpy(), resid_converged=rm)
    state = gc + 2e-3 * torch.randn(gc.shape, generator=torch.Generator().manual_seed(8))
    R, Ki, Kv = c.assembly.assemble_Stiffness_Matrix(GC=state)
    ip, ix, vv = coalesced_csr(R, Ki, Kv)
    RGC = c.assembly._GC2RGC(state)
    Ub = RGC[ib._RGC_index]
    fi, Re, Kidx, Kval = e.structural_Force(Ub, ib.rotation_matrix)
    Mi, Mv = ib.get_mass_matrix()
    res.update(state=state.numpy(), R=R.numpy(), indptr=ip, indices=ix, values=vv,
               energy=float(c.assembly._total_Potential_Energy(GC=state)),
               force=c.assembly.assemble_force(GC=state).numpy(),
               Ub=Ub.numpy(), elem_force_index=fi.numpy(), elem_R=Re.numpy(), elem_K_indices=Kidx.numpy(),
               elem_K_values=Kval.numpy(), inst_energy=float(ib.potential_energy(RGC)),
               inst_mass_indices=Mi.numpy(), inst_mass_values=Mv.numpy())
    lam = torch.randn(gc.shape, generator=torch.Generator().manual_seed(9))
    Xg = part.nodes.clone().requires_grad_(True)
    part.nodes = Xg
    mu_t = torch.tensor(mu, requires_grad=True)
    e.materials.mu = mu_t
    c.initialize()
    Rg = c.assembly.assemble_Stiffness_Matrix(GC=gc)[0]
    gX, gmu = torch.autograd.grad((Rg * lam).sum(), [Xg, mu_t])
    res.update(adj_lambda=lam.numpy(), adj_gX=gX.numpy(), adj_gmu=float(gmu))
    np.savez_compressed(os.path.join(out, "%s.npz" % name), **res)
    print(name, "E", el.shape[0], "n", gc0.shape[0], "nnz", vv.shape[0], "final max|R|", rm)


def case_couple(FEA, O, out, n=3, mu=1.0, kappa=50.0, name="couple_hex3"):
    """A jittered C3D8 block, bottom (k = 0) clamped, its top nodes (k = n)
    tied by a Couple constraint to a reference point above the block
    (couple.py:34-198) that carries a concentrated force and a moment
    (concentrate_force.py, moment.py).  Reduced R, K, energy and residual
    at a seeded state with a finite RP rotation, and the converged GC."""
    X, el = O.hex_block(n, jitter=0.1, seed=11)
    k = torch.arange(X.shape[0]) % (n + 1)
    bottom = torch.nonzero(k == 0).flatten().numpy()
    top = torch.nonzero(k == n).flatten().numpy()
    part = FEA.Part(X.clone())
    e = FEA.elements.C3D8(elems=el.clone(), elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(FEA.materials.NeoHookean(torch.tensor(mu), torch.tensor(kappa)))
    e.set_density(torch.tensor([1.0]))
    part.add_element(e)
    part.set_nodes["bottom"] = bottom
    part.set_nodes["top"] = top
    asm = FEA.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(FEA.Instance(part), "p")
    rp_xyz = [0.5, 0.5, 1.5]
    force, moment = [0.01, 0.02, -0.05], [0.01, -0.02, 0.015]
    rp = asm.add_reference_point(FEA.ReferencePoint(rp_xyz))
    asm.add_constraint(FEA.constraints.Couple(instance_name="p", set_nodes_name="top", rp_name=rp))
    asm.add_load(FEA.loads.Concentrate_Force(rp_name=rp, force=force), "f")
    asm.add_load(FEA.loads.Moment(rp_name=rp, moment=moment), "m")
    asm.add_boundary(FEA.boundarys.Boundary_Condition(instance_name="p", set_nodes_name="bottom"), "bc")
    c = FEA.FEAController()
    c.assembly = asm
    c.solver = FEA.solver.StaticImplicitSolver(tol_error=1e-10)
    c.initialize()
    gc0 = c.assembly.GC.clone()
    res = dict(X=X.numpy(), elems=el.numpy(), fixed=bottom, top=top, mu=mu, kappa=kappa, rp=np.array(rp_xyz),
               force=np.array(force), moment=np.array(moment), gc0=gc0.numpy())
    gc, rm = converge(FEA, c, gc0)
    res.update(gc_converged=gc.numpy(), resid_converged=rm)
    state = gc + 2e-3 * torch.randn(gc.shape, generator=torch.Generator().manual_seed(12))
    state[-3:] += torch.tensor([0.05, -0.03, 0.04])            # a finite RP rotation
    R, Ki, Kv = c.assembly.assemble_Stiffness_Matrix(GC=state)
    ip, ix, vv = coalesced_csr(R, Ki, Kv)
    res.update(state=state.numpy(), R=R.numpy(), indptr=ip, indices=ix, values=vv,
               energy=float(c.assembly._total_Potential_Energy(GC=state)),
               force_R=c.assembly.assemble_force(GC=state).numpy(),
               rgc_state=torch.cat([r.reshape(-1) for r in c.assembly._GC2RGC(state)]).numpy())
    np.savez_compressed(os.path.join(out, "%s.npz" % name), **res)
    print(name, "E", el.shape[0], "n", gc0.shape[0], "nnz", vv.shape[0], "final max|R|", rm,
          "rp", gc[-6:].numpy())


def case_explicit_loaded(FEA, O, out, n=3, rho=1.0, p=0.05, steps=40, name="explicit_loaded"):
    """DynamicExplicitSolver with a pressure load and two element groups: a
    Kuhn-tet cube split into two C3D4 groups of different materials (even
    and odd cells), bottom clamped, pressure on the top face, from rest with
    a seeded initial velocity, a state stored every step."""
    X, el = O.tet_block(n)
    cell = torch.arange(el.shape[0]) // 6
    g0, g1 = el[cell % 2 == 0], el[cell % 2 == 1]
    bottom = torch.nonzero(X[:, 2].abs() < 1e-9).flatten().numpy()
    sets = O.boundary_faces("C3D4", el, X, 2, 1.0)
    part = FEA.Part(X.clone())
    mats = [(1.0, 10.0), (2.0, 30.0)]
    groups = []
    for k, (g, (mu, kappa)) in enumerate(zip((g0, g1), mats)):
        idx = torch.nonzero(cell % 2 == k).flatten()
        e = FEA.elements.C3D4(elems=g.clone(), elems_index=idx, part=part)
        e.set_materials(FEA.materials.NeoHookean(torch.tensor(mu), torch.tensor(kappa)))
        e.set_density(torch.tensor([rho]))
        part.add_element(e, "g%d" % k)
        groups.append(e)
    # the top faces as (element labels, face id) of the whole mesh
    surf = [(idx.numpy(), fid) for idx, fid, _ in sets]
    part.add_surface_set("top", surf)
    part.set_nodes["bottom"] = bottom
    asm = FEA.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(FEA.Instance(part), "p")
    ld = FEA.loads.Pressure(instance_name="p", surface_set="top", pressure=p)
    asm.add_load(ld, "pressure")
    asm.add_boundary(FEA.boundarys.Boundary_Condition(instance_name="p", set_nodes_name="bottom"), "bc")
    c = FEA.FEAController()
    c.assembly = asm
    x = X[el]
    vol = torch.einsum("ei,ei->e", torch.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], dim=1), x[:, 3] - x[:, 0]).abs() / 6
    fa = []
    for tri in ([0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]):
        a = x[:, tri]
        fa.append(0.5 * torch.cross(a[:, 1] - a[:, 0], a[:, 2] - a[:, 0], dim=1).norm(dim=1))
    hmin = (3 * vol / torch.stack(fa, 1).max(1).values).min()
    cwave = np.sqrt((30.0 + 4 * 2.0 / 3) / rho)
    dt = float(0.5 * hmin / cwave)
    T = dt * steps
    c.solver = FEA.solver.DynamicExplicitSolver(time_end=T * (1 - 1e-9), time_per_storage=0.5 * dt)
    c.initialize()
    c.solver._deltaT = dt
    gc0 = torch.zeros_like(c.assembly.GC)
    gv0 = 0.01 * torch.randn(gc0.shape, generator=torch.Generator().manual_seed(10))
    minv = c.solver.get_lumped_mass_inv(gc0)
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        c.solver.solve(GC0=gc0, GV0=gv0)
    res = dict(X=X.numpy(), elems0=g0.numpy(), elems1=g1.numpy(), cell=cell.numpy(),
               mats=np.array(mats), rho=rho, p=p, dt=dt, steps=steps, fixed=bottom,
               face_elem=np.concatenate([i for i, _ in surf]),
               face_id=np.concatenate([np.full(len(i), f) for i, f in surf]),
               pressure_faces=torch.cat([s._elems for s in ld.surface_element]).numpy(),
               gv0=gv0.numpy(), minv=minv.numpy(), u_final=c.solver._GC_list[-1].numpy(),
               v_final=c.solver._GV_list[-1].numpy(), a_final=c.solver._GA_list[-1].numpy(),
               n_stored=len(c.solver._GC_list), time_final=c.solver._time_list[-1])
    np.savez_compressed(os.path.join(out, "%s.npz" % name), **res)
    print(name, "dt", dt, "stored", len(c.solver._GC_list), "max|u|", float(res["u_final"].__abs__().max()))


def case_explicit(FEA, O, out, n=4, mu=1.0, kappa=10.0, rho=1.0, steps=40, name="explicit_tet4"):
    """Config-3 style explicit run on a small Kuhn-tet cube, no BCs."""
    X, el = O.tet_block(n)
    c, part, (e,), _ = build_reference(FEA, X, [("C3D4", el, mu, kappa, rho)], [], [])
    h = 1.0 / n
    # fixed dt = 0.5 * min altitude / wave speed (the reference has only a placeholder dt)
    x = X[el]
    vol = torch.einsum("ei,ei->e", torch.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], dim=1), x[:, 3] - x[:, 0]).abs() / 6
    fa = []
    for tri in ([0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]):
        a = x[:, tri]
        fa.append(0.5 * torch.cross(a[:, 1] - a[:, 0], a[:, 2] - a[:, 0], dim=1).norm(dim=1))
    hmin = (3 * vol / torch.stack(fa, 1).max(1).values).min()
    cwave = np.sqrt((kappa + 4 * mu / 3) / rho)
    dt = float(0.5 * hmin / cwave)
    T = dt * steps
    # The reference advances from the last *stored* displacement
    # (dynamic_explicit.py:100), so only storage at every step follows the
    # central-difference recurrence; store every step.
    c.solver = FEA.solver.DynamicExplicitSolver(time_end=T * (1 - 1e-9), time_per_storage=0.5 * dt)
    c.initialize()
    c.solver._deltaT = dt
    gc0 = torch.zeros_like(c.assembly.GC)
    gv0 = 0.01 * torch.randn(gc0.shape, generator=torch.Generator().manual_seed(4))
    minv = c.solver.get_lumped_mass_inv(gc0)
    c.solver.solve(GC0=gc0, GV0=gv0)
    res = dict(X=X.numpy(), elems=el.numpy(), mu=mu, kappa=kappa, rho=rho, dt=dt, steps=steps,
               gv0=gv0.numpy(), minv=minv.numpy(), u_final=c.solver._GC_list[-1].numpy(),
               v_final=c.solver._GV_list[-1].numpy(), a_final=c.solver._GA_list[-1].numpy(),
               n_stored=len(c.solver._GC_list), time_final=c.solver._time_list[-1])
    np.savez_compressed(os.path.join(out, "%s.npz" % name), **res)
    print(name, "dt", dt, "stored", len(c.solver._GC_list), "t", c.solver._time_list[-1])


def case_implicit_dynamic(FEA, O, out, n=2, mu=1.0, kappa=10.0, rho=1.0, p=0.05, dt=0.05, steps=4, tol=1e-8,
                          name="newmark_tet2", kind="C3D4"):
    """Implicit Newmark run (DynamicImplicitSolver) on a small block of Kuhn
    tets (or hexes): bottom clamped, top pressure, from rest; the stored
    GC/GV/GA histories and the reduced consistent mass."""
    X, el = O.tet_block(n) if kind == "C3D4" else O.hex_block(n)
    bottom = torch.nonzero(X[:, 2].abs() < 1e-9).flatten().numpy()
    sets = O.boundary_faces(kind, el, X, 2, 1.0)
    surf = [(idx.numpy(), fid) for idx, fid, _ in sets]
    c, part, (e,), (ld,) = build_reference(FEA, X, [(kind, el, mu, kappa, rho)], [(surf, p)], [(bottom, (0, 1, 2))])
    c.solver = FEA.solver.DynamicImplicitSolver(deltaT=dt, time_end=steps * dt * (1 - 1e-9), tol_error=tol)
    c.initialize()
    gc0 = torch.zeros_like(c.assembly.GC)
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        ok = c.solver.solve(GC0=gc0)
    if ok is not True or len(c.solver._GC_list) != steps + 1:
        raise RuntimeError("reference implicit dynamics did not finish")
    mi, mv = c.assembly.assemble_mass_matrix(GC_now=gc0)
    ip, ix, vv = coalesced_csr(gc0, mi, mv)
    res = dict(X=X.numpy(), elems=el.numpy(), kind=kind, mu=mu, kappa=kappa, rho=rho, p=p, dt=dt, steps=steps, tol=tol,
               fixed=bottom, pressure_faces=torch.cat([s_._elems for s_ in ld.surface_element]).numpy(),
               face_elem=np.concatenate([i for i, _ in surf]),
               face_id=np.concatenate([np.full(len(i), f) for i, f in surf]),
               GC=torch.stack(c.solver._GC_list).numpy(), GV=torch.stack(c.solver._GV_list).numpy(),
               GA=torch.stack(c.solver._GA_list).numpy(), time=np.array(c.solver._time_list),
               mass_indptr=ip, mass_indices=ix, mass_values=vv)
    np.savez_compressed(os.path.join(out, "%s.npz" % name), **res)
    print(name, "E", el.shape[0], "n", gc0.shape[0], "steps", steps, "max|GC|", float(res["GC"][-1].__abs__().max()))


def case_inp(FEA, out):
    """The reference's FEA_INP.read_inp and from_inp on the sample INP files
    of inp_samples.py: what it parses (nodes, element arrays, sets, surfaces,
    sections, the element material table, materials, instances) and the
    model it builds (per element group: type, labels, connectivity, mu,
    kappa, density; per part: node sets)."""
    import inp_samples
    for name, path in inp_samples.write_samples(out).items():
        inp = FEA.FEA_INP()
        inp.read_inp(path)
        d = {}
        for pn, p in inp.part.items():
            d["nodes:%s" % pn] = p.nodes.numpy()
            d["elemtypes:%s" % pn] = np.array(list(p.elems.keys()))
            for t, e in p.elems.items():
                d["elems:%s:%s" % (pn, t)] = np.asarray(e, dtype=np.int64)
            for sn, m in p.sets_nodes.items():
                d["nset:%s:%s" % (pn, sn)] = np.array(sorted(m), dtype=np.int64)
            for sn, m in p.sets_elems.items():
                d["elset:%s:%s" % (pn, sn)] = np.array(sorted(m), dtype=np.int64)
            d["surfaces:%s" % pn] = np.array(list(p.surfaces.keys()))
            for sn, entries in p.surfaces.items():
                d["surfn:%s:%s" % (pn, sn)] = np.array(len(entries))
                for k, (labels, face) in enumerate(entries):
                    d["surf:%s:%s:%d:labels" % (pn, sn, k)] = np.asarray(labels, dtype=np.int64)
                    d["surf:%s:%s:%d:face" % (pn, sn, k)] = np.array(face)
            d["sections:%s" % pn] = np.array(p.sections)
            d["elems_material:%s" % pn] = p.elems_material.numpy()
        for mn, m in inp.material.items():
            d["material:%s" % mn] = np.array([m.type, m.mat_para[0], m.mat_para[1], m.density], dtype=np.float64)
        for iname, (part_name, T) in getattr(inp.assemble, "instances", {}).items():
            d["instance:%s" % iname] = np.asarray(T, dtype=np.float64)
            d["instancepart:%s" % iname] = np.array(part_name)
        for sn, m in getattr(inp.assemble, "sets_nodes", {}).items():
            d["asm_nset:%s" % sn] = np.array(sorted(m), dtype=np.int64)
        for sn, m in getattr(inp.assemble, "sets_elems", {}).items():
            d["asm_elset:%s" % sn] = np.array(sorted(m), dtype=np.int64)
        fe = FEA.from_inp(inp)
        for pn, part in fe.assembly._parts.items():
            for sn, m in part.set_nodes.items():
                d["pset:%s:%s" % (pn, sn)] = np.asarray(m, dtype=np.int64)
            for k, (en, e) in enumerate(part.elems.items()):
                g = "group:%s:%d" % (pn, k)
                d[g + ":type"] = np.array(type(e).__name__)
                d[g + ":elems_index"] = e._elems_index.numpy().astype(np.int64)
                d[g + ":elems"] = e._elems.numpy().astype(np.int64)
                d[g + ":mu"] = np.array(float(e.materials.mu))
                d[g + ":kappa"] = np.array(float(e.materials.kappa))
                d[g + ":density"] = np.asarray(e.density, dtype=np.float64)
            d["ngroups:%s" % pn] = np.array(len(part.elems))
        np.savez_compressed(os.path.join(out, name + ".npz"), **d)
        print("wrote", name, len(d), "arrays")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the reference source tree (the directory holding FEA/)")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--case", default="all", help="all, or one of: cfg1 tet3 hex5 explicit newmark newmark_hex inp rotated explicit_loaded couple")
    a = ap.parse_args()
    FEA = import_reference(a.ref)
    from oracle import fea_oracle as O  # mesh generators only
    torch.set_num_threads(os.cpu_count())
    run = lambda name: a.case in ("all", name)
    if run("cfg1"):
        case_tet_cube(FEA, O, a.out, n=10, name="cfg1")
    if run("tet3"):
        case_tet_cube(FEA, O, a.out, n=3, full_element=True, name="tet3")
    if run("hex5"):
        case_hex_block(FEA, O, a.out)
    if run("explicit"):
        case_explicit(FEA, O, a.out)
    if run("newmark"):
        case_implicit_dynamic(FEA, O, a.out)
    if run("inp"):
        sys.path.insert(0, HERE)
        case_inp(FEA, a.out)
    if run("newmark_hex"):
        case_implicit_dynamic(FEA, O, a.out, n=2, kappa=20.0, p=0.05, dt=0.05, name="newmark_hex2", kind="C3D8")
    if run("rotated"):
        case_rotated(FEA, O, a.out)
    if run("explicit_loaded"):
        case_explicit_loaded(FEA, O, a.out)
    if run("couple"):
        case_couple(FEA, O, a.out)


if __name__ == "__main__":
    main()
