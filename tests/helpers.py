"""Model builders shared by the tests (fea_b200 API and the CPU oracle)."""
import numpy as np
import torch

from oracle import fea_oracle as O


def surface_list(g):
    """Surface set [(element labels, face id)] of a golden case."""
    if "face_id" in g:
        fid = g["face_id"]
        return [(g["face_elem"][fid == f], int(f)) for f in np.unique(fid)]
    return [(g["end_elems"], 3)]


def fea_model(g, kind, pressure=True, fixed=True, p=None, solver=None):
    import fea_b200 as F
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    part = F.Part(X)
    cls = F.elements.C3D4 if kind == "C3D4" else F.elements.C3D8
    e = cls(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(float(g["mu"]), float(g["kappa"])))
    e.set_density(float(g["rho"]) if "rho" in g else 1.0)
    part.add_element(e)
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    load = None
    if pressure:
        part.add_surface_set("surf", surface_list(g))
        load = F.loads.Pressure(instance_name="p", surface_set="surf", pressure=float(g["p"]) if p is None else p)
        asm.add_load(load, "pressure")
    if fixed:
        part.set_nodes["fix"] = g["fixed"]
        asm.add_boundary(F.boundarys.Boundary_Condition(instance_name="p", set_nodes_name="fix"), "bc")
    c = F.FEAController()
    c.assembly = asm
    c.solver = solver if solver is not None else F.solver.StaticImplicitSolver()
    return c, e, load


def oracle_model(g, kind, pressure=True, fixed=True):
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    rho = float(g["rho"]) if "rho" in g else 1.0
    loads = [O.PressureLoad(torch.from_numpy(g["pressure_faces"]), float(g["p"]))] if pressure else []
    fx = [(g["fixed"], (0, 1, 2))] if fixed else []
    return O.Model(X, [O.Group(kind, el, float(g["mu"]), float(g["kappa"]), rho)], loads, fx)


def rel(a, b):
    a = torch.as_tensor(a).detach().double().cpu().reshape(-1)
    b = torch.as_tensor(b).detach().double().cpu().reshape(-1)
    return float((a - b).norm() / max(float(b.norm()), 1e-300))


def csr_from_api(asm):
    P = asm.plan
    return P.indptr.cpu().numpy(), P.indices.cpu().numpy()


def top_faces(kind, X, el, n):
    """Surface set and face node lists of the z = max side, chosen by topology
    (the nodes of a jittered block do not lie on a plane)."""
    if kind == "C3D8":
        pos = np.nonzero(np.arange(el.shape[0]) % n == n - 1)[0]
        loc = [4, 5, 6, 7]                      # face 1 of C3D8
        return [(pos, 1)], torch.as_tensor(np.asarray(el)[pos][:, loc])
    sets = O.boundary_faces(kind, torch.as_tensor(el), torch.as_tensor(X), 2, float(np.asarray(X)[:, 2].max()))
    return [(i.numpy(), f) for i, f, _ in sets], torch.cat([f for _, _, f in sets])
