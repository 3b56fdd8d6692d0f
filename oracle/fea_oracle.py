"""CPU float64 oracle for the FEA hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``fea_b200``) may import or
call this module; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it, and only as the checker or the timed CPU
baseline.

It restates, in torch-on-CPU float64 code of its own, the algorithms of the
reference package sssnnn7119/FEA for the path that the CUDA library replaces.
Every function names the reference lines (``path:line`` inside that project)
whose behaviour it follows.  The arithmetic is kept in the reference's own
form (a materialised 81-entry material tangent, einsum contractions over
``[gauss, element, ...]`` tensors, a sort-based COO pattern) so that it is an
independent check of the factored formulas used by the kernels.

Parity of this oracle is pinned against golden fixtures produced by running
the reference package itself (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

DT = torch.float64

# ---------------------------------------------------------------------------
# Reference elements: Gauss points, weights, shape functions and derivatives
# ---------------------------------------------------------------------------


def tet4_rule():
    """C3D4: one Gauss point at (1/4, 1/4, 1/4), weight 1/6, linear N.

    Follows FEA/assemble/elements/C3/tetrahedral.py:28-42 (shape table
    N0 = 1-x-y-z, N1 = x, N2 = y, N3 = z; p0 and the 1/6 weight).
    Returns (N [G,nn], dN/dxi [G,3,nn], weight [G]).
    """
    p = torch.tensor([[0.25, 0.25, 0.25]], dtype=DT)
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    N = torch.stack([1 - x - y - z, x, y, z], dim=1)
    dN = torch.zeros(1, 3, 4, dtype=DT)
    dN[:, :, 0] = -1.0
    for m in range(3):
        dN[:, m, m + 1] = 1.0
    return N, dN, torch.tensor([1.0 / 6.0], dtype=DT)


HEX_CORNERS = torch.tensor([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                            [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=DT)


def hex8_rule():
    """C3D8: 2x2x2 Gauss points at +-1/sqrt(3) (weight 1), trilinear N.

    Follows FEA/assemble/elements/C3/brick.py:47-164: node ordering of the
    Abaqus brick (the 8 corners listed at brick.py:15-25), Gauss point order
    at brick.py:151-160, N_a = 1/8 (1+g g_a)(1+h h_a)(1+r r_a).
    """
    q = 1.0 / np.sqrt(3.0)
    p = HEX_CORNERS * q
    s = HEX_CORNERS
    G = p.shape[0]
    N = torch.zeros(G, 8, dtype=DT)
    dN = torch.zeros(G, 3, 8, dtype=DT)
    for g in range(G):
        f = 1.0 + s * p[g]                      # [8,3] factors (1 + xi*xi_a)
        N[g] = 0.125 * f.prod(dim=1)
        for m in range(3):
            others = [d for d in range(3) if d != m]
            dN[g, m] = 0.125 * s[:, m] * f[:, others[0]] * f[:, others[1]]
    return N, dN, torch.ones(G, dtype=DT)


def rule(kind: str):
    return {"C3D4": tet4_rule, "C3D8": hex8_rule}[kind]()


def tri3_rule():
    """T3 surface: 3-point rule (1/6,1/6),(2/3,1/6),(1/6,2/3), weights 1/6.

    Follows FEA/assemble/elements/C3/surfaces/triangle.py (shape table and the
    three-point rule of T3.initialize).  Returns (N [G,nn], dN [G,2,nn], w [G]).
    """
    p = torch.tensor([[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]], dtype=DT)
    N = torch.stack([1 - p[:, 0] - p[:, 1], p[:, 0], p[:, 1]], dim=1)
    dN = torch.tensor([[-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]], dtype=DT).expand(3, 2, 3).clone()
    return N, dN, torch.full((3,), 1.0 / 6.0, dtype=DT)


def quad4_rule():
    """Q4 surface: 2x2 Gauss at +-1/sqrt(3), weight 1, bilinear N.

    Follows FEA/assemble/elements/C3/surfaces/quadrilateral.py (Q4 shape table,
    Gauss points (-g,-g),(g,-g),(g,g),(-g,g)).
    """
    q = 1.0 / math.sqrt(3.0)
    p = torch.tensor([[-q, -q], [q, -q], [q, q], [-q, q]], dtype=DT)
    c = torch.tensor([[-1, -1], [1, -1], [1, 1], [-1, 1]], dtype=DT)
    N = torch.zeros(4, 4, dtype=DT)
    dN = torch.zeros(4, 2, 4, dtype=DT)
    for g in range(4):
        f = 1.0 + c * p[g]
        N[g] = 0.25 * f[:, 0] * f[:, 1]
        dN[g, 0] = 0.25 * c[:, 0] * f[:, 1]
        dN[g, 1] = 0.25 * c[:, 1] * f[:, 0]
    return N, dN, torch.ones(4, dtype=DT)


# Face node lists per volume element (face id -> local nodes), outward ordering.
# C3D4: tetrahedral.py:45-64.  C3D8: brick.py:166-201.
FACES = {
    "C3D4": {0: [0, 2, 1], 1: [0, 1, 3], 2: [1, 2, 3], 3: [0, 3, 2]},
    "C3D8": {0: [0, 3, 2, 1], 1: [4, 5, 6, 7], 2: [0, 1, 5, 4], 3: [1, 2, 6, 5],
             4: [2, 3, 7, 6], 5: [0, 4, 7, 3]},
}


# ---------------------------------------------------------------------------
# Element geometry (reference configuration)
# ---------------------------------------------------------------------------


def preload_gaussian(kind: str, X: torch.Tensor, elems: torch.Tensor):
    """dN/dX, N and w*detJ at every Gauss point of every element.

    Follows Element_3D._pre_load_gaussian, FEA/assemble/elements/C3/C3base.py:
    155-216: Jacobian J[g,e,i,m] = sum_a dN_a/dxi_m X_{a,i}; dN/dX =
    J^{-T} dN/dxi; weight = detJ * w_g (the sign of detJ is kept).
    Returns dNdX [G,E,3,nn], wdet [G,E], N [G,E,nn].
    """
    N, dN, w = rule(kind)
    Xe = X[elems]                                        # [E,nn,3]
    Jac = torch.einsum("gma,eai->geim", dN, Xe)          # [G,E,3(i),3(m)]
    det = torch.linalg.det(Jac)
    inv = torch.linalg.inv(Jac)                          # [G,E,m,i]
    dNdX = torch.einsum("gemi,gma->geia", inv, dN)
    G, E = Jac.shape[:2]
    return dNdX, det * w[:, None], N[:, None, :].expand(G, E, N.shape[1])


# ---------------------------------------------------------------------------
# Element pattern (unreduced, per element group)
# ---------------------------------------------------------------------------


def element_pattern(elems: torch.Tensor):
    """Unique sorted COO of the group's DOF pairs and the element-to-slot map.

    Follows Element_3D.initialize, C3base.py:109-153: entries are enumerated in
    (a, j, b, k, e) order with e fastest; the COO is the sorted set of distinct
    (row, col) = (3 n_a + j, 3 n_b + k) pairs; the slot map gives, for every
    enumerated entry, its position in that COO.  The force index is
    3 n_a + j in (a, j, e) order.
    Returns (indices_matrix int64 [2,nnz], slot_map int64 [(3nn)^2 E],
             indices_force int64 [3 nn E]).
    """
    E, nn = elems.shape
    el = elems.to(torch.int64).T                         # [nn,E]
    j3 = torch.arange(3, dtype=torch.int64)
    row = (3 * el[:, None, None, None, :] + j3[None, :, None, None, None]).expand(nn, 3, nn, 3, E)
    col = (3 * el[None, None, :, None, :] + j3[None, None, None, :, None]).expand(nn, 3, nn, 3, E)
    S = int(3 * int(elems.max()) + 3)
    key = (row * S + col).reshape(-1)
    uniq, inverse = torch.unique(key, sorted=True, return_inverse=True)
    idx = torch.stack([uniq // S, uniq % S])
    return idx, inverse, element_force_index(elems)


def element_force_index(elems: torch.Tensor):
    """The residual index 3 n_a + j in (a, j, e) order alone: what
    structural_Force(if_onlyforce=True) scatters with (C3base.py:413-426),
    precomputed by Element_3D.initialize (C3base.py:109-153)."""
    el = elems.to(torch.int64).T                         # [nn,E]
    j3 = torch.arange(3, dtype=torch.int64)
    return (3 * el[:, None, :] + j3[None, :, None]).reshape(-1)


# ---------------------------------------------------------------------------
# Kinematics and Neo-Hookean material
# ---------------------------------------------------------------------------


def deformation_gradient(U: torch.Tensor, elems: torch.Tensor, dNdX: torch.Tensor):
    """F[g,e,I,i] = delta_Ii + sum_a U_{a,I} dN_a/dX_i.

    Follows Element_3D.components_Solid, C3base.py:454-469 (and the same sum in
    potential_Energy, C3base.py:387-400).
    """
    Ue = U[elems]                                        # [E,nn,3]
    F = torch.einsum("geia,eaI->geIi", dNdX, Ue)
    F = F + torch.eye(3, dtype=DT)
    return F


def neohookean_energy(F, mu, kappa):
    """W = mu/2 (J^{-2/3} tr(F^T F) - 3) + kappa/2 (J-1)^2.

    Follows NeoHookean.strain_energy_density_C3, hyperelastic.py:25-33.
    """
    J = torch.linalg.det(F)
    I1 = (F ** 2).sum((-1, -2)) * J ** (-2.0 / 3.0)
    return mu / 2 * (I1 - 3) + kappa / 2 * (J - 1) ** 2


def neohookean_stress_tangent(F, mu, kappa):
    """s = P^T and the full C_ijkl = ds_ij/dF_kl (materialised).

    Follows NeoHookean.material_Constitutive_C3, hyperelastic.py:35-84 with
    J, J^{-2/3}, I1 and F^{-1} as in C3base.py:466-469.
    """
    invF = torch.linalg.inv(F)
    J = torch.linalg.det(F)[..., None, None]
    Jm = J ** (-2.0 / 3.0)
    I1 = (F ** 2).sum((-1, -2))[..., None, None] * Jm
    muJ = mu * Jm
    FtJ = F.transpose(-1, -2) * muJ
    muI1inv = mu * I1 * invF
    kJinv = kappa * J * invF
    s = FtJ - muI1inv / 3.0 + kJinv * (J - 1)
    T1 = -2.0 / 3.0 * FtJ + kJinv * (2 * J - 1) + 2.0 / 9.0 * muI1inv
    T2 = -2.0 / 3.0 * muJ * invF
    T3 = muI1inv / 3.0 - kJinv * (J - 1)
    C = torch.einsum("geij,gelk->geijkl", T1, invF)
    C = C + torch.einsum("geij,gekl->geijkl", T2, F)
    C = C + torch.einsum("geik,gelj->geijkl", T3, invF)
    d = torch.eye(3, dtype=DT)
    C = C + muJ[..., None, None] * torch.einsum("il,jk->ijkl", d, d)
    return s, C


def element_residual_tangent(kind, X, elems, U, mu, kappa, want_K=True):
    """Per-element residual R_e[a,j,e] and tangent K_e[a,j,b,k,e].

    Follows Element_3D.structural_Force, C3base.py:413-452:
    R_e = sum_g s_ij dN_ai w ('geij,geia,ge->aje'),
    K_e = sum_g C_ijkl dN_ai dN_bl w ('geijkl,gelb,geia,ge->ajbke').
    """
    dNdX, w, _ = preload_gaussian(kind, X, elems)
    F = deformation_gradient(U, elems, dNdX)
    s, C = neohookean_stress_tangent(F, mu, kappa)
    R = torch.einsum("geij,geia,ge->aje", s, dNdX, w)
    if not want_K:
        return R, None
    K = torch.einsum("geijkl,gelb,geia,ge->ajbke", C, dNdX, dNdX, w)
    return R, K


def element_energy(kind, X, elems, U, mu, kappa):
    """sum_{g,e} W(F) w.  Follows Element_3D.potential_Energy, C3base.py:387-411."""
    dNdX, w, _ = preload_gaussian(kind, X, elems)
    F = deformation_gradient(U, elems, dNdX)
    return (neohookean_energy(F, mu, kappa) * w).sum()


def element_mass(kind, X, elems, rho):
    """Consistent element mass M_ab = sum_g rho N_a N_b w  [nn,nn,E].

    Follows Element_3D.get_mass_matrix, C3base.py:348-384 (before the 3-DOF
    expansion and the slot scatter).
    """
    _, w, N = preload_gaussian(kind, X, elems)
    return torch.einsum("gea,geb,ge->abe", N, N, w * rho)


# ---------------------------------------------------------------------------
# Follower pressure (enclosed-volume potential) on T3 / Q4 faces
# ---------------------------------------------------------------------------


def _surface_rule(nn):
    return tri3_rule() if nn == 3 else quad4_rule()


def _surface_frames(x, faces):
    N, dN, w = _surface_rule(faces.shape[1])
    sfa = torch.cat([N[:, None, :], dN], dim=1)          # [G,3(m),nn]
    xf = x[faces]                                        # [E,nn,3]
    r = torch.einsum("gma,eai->geim", sfa, xf)           # columns: x, x_xi, x_eta
    return sfa, r, w


def pressure_force_tangent(x, faces, p, want_K=True):
    """Follower pressure from the enclosed-volume potential.

    Follows Pressure.get_stiffness, FEA/assemble/loads/pressure.py:80-132:
    V = 1/3 sum_g w det[x, x_xi, x_eta]; the load's force values are
    -p dV/dx in (e, i, a) order and its stiffness values -p d2V/dx2 in
    (e, i, a, j, b) order.  Returns (f [E,3,nn], k [E,3,nn,3,nn] or None).
    """
    sfa, r, w = _surface_frames(x, faces)
    det = torch.linalg.det(r)
    inv = torch.linalg.inv(r)
    cof = det[..., None, None] * inv.transpose(-1, -2)   # d det / d r[i,m]
    Vdr = w[:, None, None, None] * cof / 3.0
    f = torch.einsum("gma,geim->eia", sfa, Vdr)
    if not want_K:
        return -p * f, None
    part1 = torch.einsum("geim,genj->geimjn", cof, inv)
    part2 = part1.permute(0, 1, 2, 5, 4, 3)
    V2 = (part1 - part2) * w[:, None, None, None, None, None] / 3.0
    k = torch.einsum("gma,gnb,geimjn->eiajb", sfa, sfa, V2)
    return -p * f, -p * k


def pressure_volume(x, faces):
    """Enclosed-volume functional; follows Pressure.get_potential_energy, pressure.py:134-159."""
    _, r, w = _surface_frames(x, faces)
    return (w[:, None] * torch.linalg.det(r)).sum() / 3.0


# ---------------------------------------------------------------------------
# A model in the reference's terms: one instance, element groups, pressure
# loads on faces and Dirichlet node sets.
# ---------------------------------------------------------------------------


def reduced_pattern_csr(elem_groups, free, n_nodes):
    """Reduced coalesced CSR pattern (indptr int64 [n+1], indices int64 [nnz])
    from the node-level restatement of the element pattern, for meshes too
    large for the DOF-level sort of ``element_pattern``.

    The reference's pattern (C3base.py:109-153) is the sorted set of DOF
    pairs (3 n_a + j, 3 n_b + k) of every element; after the Dirichlet mask
    and the relabelling (assembly.py:357-387) a free row (n, j) holds, in
    ascending order, the free DOFs of every node sharing an element with n.
    Here the distinct node pairs are found with one sort of E nn^2 keys and
    expanded to DOFs with numpy.  ``free`` is the [3 N] free-DOF mask.
    """
    free = np.asarray(free, dtype=bool).reshape(n_nodes, 3)
    keys = []
    for el in elem_groups:
        el = np.asarray(el, dtype=np.int64)
        keys.append((el[:, :, None] * n_nodes + el[:, None, :]).reshape(-1))
    pairs = np.unique(np.concatenate(keys))
    pn, pc = pairs // n_nodes, pairs % n_nodes               # sorted by (n, c)
    fc = free.sum(1)                                          # free DOFs per node
    rdof = np.concatenate([[0], np.cumsum(fc)[:-1]])          # first reduced DOF of each node
    # node column list: for every pair (n, c), the free DOFs of c in order
    cnt = fc[pc]
    start = np.repeat(rdof[pc] - np.concatenate([[0], np.cumsum(cnt)[:-1]]), cnt)
    cols = start + np.arange(int(cnt.sum()))
    L = np.bincount(pn, weights=cnt, minlength=n_nodes).astype(np.int64)   # columns per row of node n
    seg = np.concatenate([[0], np.cumsum(L)[:-1]])
    # every free row (n, j) repeats its node's column list
    rown = np.repeat(np.arange(n_nodes), fc)
    rl = L[rown]
    indptr = np.concatenate([[0], np.cumsum(rl)]).astype(np.int64)
    first = np.repeat(seg[rown] - indptr[:-1], rl)
    indices = cols[first + np.arange(int(indptr[-1]))]
    return indptr, indices


@dataclass
class Group:
    kind: str
    elems: torch.Tensor          # [E,nn] int64 (part node ids)
    mu: float
    kappa: float
    rho: float = 1.0


@dataclass
class PressureLoad:
    faces: torch.Tensor          # [F,nf] int64 node ids (T3 or Q4)
    p: float


@dataclass
class Model:
    X: torch.Tensor                                      # [N,3]
    groups: list = field(default_factory=list)
    pressures: list = field(default_factory=list)
    fixed: list = field(default_factory=list)            # list of (node ids, dofs)

    def __post_init__(self):
        self.X = self.X.to(DT)
        self._free = None

    # DOF bookkeeping: assembly.py:157-183 and boundary_condition.py:35-41
    def free_mask(self):
        """Free DOFs in RGC order; computed once, like the reference's
        reduction mask (the model is not changed after construction)."""
        if self._free is None:
            N = self.X.shape[0]
            m = torch.zeros(N, 3, dtype=torch.bool)
            for g in self.groups:
                m[torch.unique(g.elems)] = True
            for pl in self.pressures:
                m[torch.unique(pl.faces)] = True
            for nodes, dofs in self.fixed:
                for d in dofs:
                    m[torch.as_tensor(nodes, dtype=torch.int64), d] = False
            self._free = m.reshape(-1)
        return self._free.clone()

    def initial_gc(self):
        """GC0 with the 1e-5 seed on the last node (assembly.py:113)."""
        N = self.X.shape[0]
        rgc = torch.zeros(N, 3, dtype=DT)
        rgc[-1] = 1e-5
        for nodes, dofs in self.fixed:
            for d in dofs:
                rgc[torch.as_tensor(nodes, dtype=torch.int64), d] = 0.0
        return rgc.reshape(-1)[self.free_mask()]

    def gc_to_u(self, gc):
        """_GC2RGC, assembly.py:470-492 (Dirichlet values are zero)."""
        u = torch.zeros(self.X.shape[0] * 3, dtype=DT)
        u[self.free_mask()] = gc
        return u.reshape(-1, 3)

    # assembly.py:311-387
    def assemble(self, gc, want_K=True):
        """Reduced (R, coalesced CSR (indptr, indices, values)).

        Follows Assembly._assemble_generalized_Matrix and
        _assemble_reduced_Matrix (assembly.py:311-387): element R and K plus
        the loads' -f and -k, scattered over all DOFs, then rows/cols of
        Dirichlet DOFs dropped and the rest relabelled in GC order.
        """
        u = self.gc_to_u(gc)
        ndof = self.X.shape[0] * 3
        R0 = torch.zeros(ndof, dtype=DT)
        rows, cols, vals = [], [], []
        for g in self.groups:
            Re, Ke = element_residual_tangent(g.kind, self.X, g.elems, u, g.mu, g.kappa, want_K)
            if want_K:
                idx, slot, force = element_pattern(g.elems)
            else:
                force = element_force_index(g.elems)
            R0.scatter_add_(0, force, Re.reshape(-1))
            if want_K:
                v = torch.zeros(idx.shape[1], dtype=DT).scatter_add_(0, slot, Ke.reshape(-1))
                rows.append(idx[0]); cols.append(idx[1]); vals.append(v)
        x = self.X + u
        for pl in self.pressures:
            f, k = pressure_force_tangent(x, pl.faces, pl.p, want_K)
            fi = torch.stack([3 * pl.faces, 3 * pl.faces + 1, 3 * pl.faces + 2], dim=1)
            R0.scatter_add_(0, fi.reshape(-1), -f.reshape(-1))
            if want_K:
                E, nf = pl.faces.shape
                ra = (3 * pl.faces[:, None, :, None, None] + torch.arange(3)[None, :, None, None, None])
                cb = (3 * pl.faces[:, None, None, None, :] + torch.arange(3)[None, None, None, :, None])
                rows.append(ra.expand(E, 3, nf, 3, nf).reshape(-1))
                cols.append(cb.expand(E, 3, nf, 3, nf).reshape(-1))
                vals.append(-k.reshape(-1))
        free = self.free_mask()
        R = R0[free]
        if not want_K:
            return R, None
        rows = torch.cat(rows); cols = torch.cat(cols); vals = torch.cat(vals)
        keep = free[rows] & free[cols]
        rid = torch.cumsum(free.to(torch.int64), 0) - 1    # rank among free DOFs
        n = int(free.sum())
        A = torch.sparse_coo_tensor(torch.stack([rid[rows[keep]], rid[cols[keep]]]), vals[keep], (n, n)).coalesce()
        Ac = A.to_sparse_csr()
        return R, (Ac.crow_indices(), Ac.col_indices(), Ac.values())

    def stiffness_coo(self, gc, patterns, chunk=16384):
        """One Assembly.assemble_Stiffness_Matrix call in the reference's own
        output form: (R [n], K_indices [2, M], K_values [M]), an UNCOALESCED
        reduced COO.

        Follows assembly.py:283-387 step by step: per element group
        structural_Force (C3base.py:413-452: element R and K, R scattered by
        the force index, K scattered by the element-to-slot map into the
        group's coalesced values), the loads' -f and -k as COO
        (pressure.py:80-132), concatenation, the Dirichlet mask on rows and
        columns (assembly.py:373-376) and the relabelling of each index row
        by ``unique(return_inverse=True)`` (assembly.py:379-380).
        ``patterns`` holds one ``element_pattern`` per group: the
        reference's ``initialize`` builds them once per mesh.  The element
        arithmetic runs over ``chunk`` elements at a time (the same values
        as one pass; bounded host memory).
        """
        u = self.gc_to_u(gc)
        ndof = self.X.shape[0] * 3
        R0 = torch.zeros(ndof, dtype=DT)
        rows, cols, vals = [], [], []
        for g, (idx, slot, force) in zip(self.groups, patterns):
            E, nn = g.elems.shape
            v = torch.zeros(idx.shape[1], dtype=DT)
            slot2 = slot.view(-1, E)                         # (a, j, b, k) x e, e fastest
            force2 = force.view(-1, E)                       # (a, j) x e
            for e0 in range(0, E, chunk):
                e1 = min(E, e0 + chunk)
                Re, Ke = element_residual_tangent(g.kind, self.X, g.elems[e0:e1], u, g.mu, g.kappa)
                R0.scatter_add_(0, force2[:, e0:e1].reshape(-1), Re.reshape(-1))
                v.scatter_add_(0, slot2[:, e0:e1].reshape(-1), Ke.reshape(-1))
            rows.append(idx[0]); cols.append(idx[1]); vals.append(v)
        x = self.X + u
        for pl in self.pressures:
            f, k = pressure_force_tangent(x, pl.faces, pl.p)
            fi = torch.stack([3 * pl.faces, 3 * pl.faces + 1, 3 * pl.faces + 2], dim=1)
            R0.scatter_add_(0, fi.reshape(-1), -f.reshape(-1))
            E, nf = pl.faces.shape
            ra = (3 * pl.faces[:, None, :, None, None] + torch.arange(3)[None, :, None, None, None])
            cb = (3 * pl.faces[:, None, None, None, :] + torch.arange(3)[None, None, None, :, None])
            rows.append(ra.expand(E, 3, nf, 3, nf).reshape(-1))
            cols.append(cb.expand(E, 3, nf, 3, nf).reshape(-1))
            vals.append(-k.reshape(-1))
        free = self.free_mask()
        rows = torch.cat(rows); cols = torch.cat(cols); vals = torch.cat(vals)
        keep = free[rows] & free[cols]
        rows, cols, vals = rows[keep], cols[keep], vals[keep]
        rows = rows.unique(return_inverse=True)[1]
        cols = cols.unique(return_inverse=True)[1]
        return R0[free], torch.stack([rows, cols]), vals

    def energy(self, gc):
        """Assembly._total_Potential_Energy, assembly.py:389-415 (pressure.py:134-159)."""
        u = self.gc_to_u(gc)
        e = torch.zeros((), dtype=DT)
        for g in self.groups:
            e = e + element_energy(g.kind, self.X, g.elems, u, g.mu, g.kappa)
        x = self.X + u
        for pl in self.pressures:
            e = e + pl.p * pressure_volume(x, pl.faces)
        return e

    def lumped_mass_inv(self):
        """Row-sum lumped inverse mass over free DOFs.

        Follows Element_3D.get_mass_matrix (C3base.py:348-384), the reduction
        in Assembly.assemble_mass_matrix (assembly.py:421-443) and
        DynamicExplicitSolver.get_lumped_mass_inv (dynamic_explicit.py:147-167).
        """
        free = self.free_mask()
        ndof = self.X.shape[0] * 3
        m = torch.zeros(ndof, dtype=DT)
        for g in self.groups:
            Me = element_mass(g.kind, self.X, g.elems, g.rho)      # [nn,nn,E]
            for d in range(3):
                ra = 3 * g.elems.T + d                             # [nn,E]
                contrib = Me * free[(3 * g.elems.T + d)][None, :, :]   # drop fixed columns
                m.scatter_add_(0, ra.reshape(-1), contrib.sum(1).reshape(-1))
        m = m[free]
        m[m.abs() < 1e-12] = 1.0
        return 1.0 / m

    def mass_coo(self):
        """Reduced consistent mass as duplicate COO (rows, cols, values).

        Follows Element_3D.get_mass_matrix (C3base.py:348-384: M_ab times the
        3x3 identity of every element, stored as full 3x3 blocks on the
        stiffness pattern, zeros included) and Assembly.assemble_mass_matrix
        (assembly.py:421-443: entries of fixed DOFs dropped, rows and columns
        relabelled in GC order).
        """
        free = self.free_mask()
        rid = torch.cumsum(free.to(torch.int64), 0) - 1
        rows, cols, vals = [], [], []
        for g in self.groups:
            Me = element_mass(g.kind, self.X, g.elems, g.rho)         # [nn,nn,E]
            nn = g.elems.shape[1]
            for j in range(3):
                for k in range(3):
                    ra = (3 * g.elems.T[:, None, :] + j).expand(nn, nn, -1)
                    cb = (3 * g.elems.T[None, :, :] + k).expand(nn, nn, -1)
                    rows.append(ra.reshape(-1)); cols.append(cb.reshape(-1))
                    vals.append(Me.reshape(-1) if j == k else torch.zeros(Me.numel(), dtype=DT))
        rows = torch.cat(rows); cols = torch.cat(cols); vals = torch.cat(vals)
        keep = free[rows] & free[cols]
        return rid[rows[keep]], rid[cols[keep]], vals[keep]

    def mass_matrix(self):
        """The reduced consistent mass as a scipy CSR matrix (duplicates summed)."""
        import scipy.sparse as sp
        r, c, v = self.mass_coo()
        n = int(self.free_mask().sum())
        return sp.coo_matrix((v.numpy(), (r.numpy(), c.numpy())), shape=(n, n)).tocsr()


# ---------------------------------------------------------------------------
# Couple constraint: nodes tied to a reference point's rigid motion
# ---------------------------------------------------------------------------


def _eps3():
    e = torch.zeros(3, 3, 3, dtype=DT)
    e[0, 1, 2] = e[1, 2, 0] = e[2, 0, 1] = 1.0
    e[0, 2, 1] = e[2, 1, 0] = e[1, 0, 2] = -1.0
    return e


def couple_motion(z, y):
    """Displacement of tied nodes by the rotation vector z of a reference
    point, R(z) y - y for rows of y (offsets from the point), and its first
    and second derivatives with respect to z: (Y [n,3], Ydot [n,3,3],
    Ydot2 [n,3,3,3]).

    Follows Couple._rotation3d and Couple._calculate_Ydotz
    (FEA/assemble/constraints/couple.py:169-282): Rodrigues' formula in the
    angle theta = |z| + 1e-20 and the axis w = z / theta, differentiated by
    the chain rule through (theta, w) with dtheta/dz = w,
    dw/dz = I/theta - z z^T/theta^3 and its derivative.
    """
    z = z.to(DT)
    y = y.to(DT)
    th = z.norm() + 1e-20
    w = z / th
    c, s = torch.cos(th), torch.sin(th)
    E = _eps3()
    wy = y @ w                                            # [n]
    wxy = torch.einsum("ijk,j,nk->ni", E, w, y)           # w x y
    Y = y * c + wxy * s + w[None, :] * wy[:, None] * (1 - c) - y
    I3 = torch.eye(3, dtype=DT)
    f_t = -y * s + wxy * c + w[None, :] * wy[:, None] * s                 # d/dtheta
    f_tt = -y * c - wxy * s + w[None, :] * wy[:, None] * c
    Ey = torch.einsum("ilk,nk->nil", E, y)                               # d(w x y)_i / dw_l
    wxI = I3[None] * wy[:, None, None] + w[None, :, None] * y[:, None, :]  # d(w (w.y))_i / dw_l
    f_w = s * Ey + (1 - c) * wxI
    f_wt = c * Ey + s * wxI
    f_ww = (1 - c) * (torch.einsum("il,nm->nilm", I3, y) + torch.einsum("im,nl->nilm", I3, y))
    dw = I3 / th - torch.outer(z, z) / th ** 3                           # dw/dz = d2theta/dz2
    d2w = 3 * torch.einsum("i,p,q->ipq", z, z, z) / th ** 5 - (
        torch.einsum("ip,q->ipq", I3, z) + torch.einsum("iq,p->ipq", I3, z) + torch.einsum("pq,i->ipq", I3, z)) / th ** 3
    Ydot = torch.einsum("nil,lp->nip", f_w, dw) + torch.einsum("ni,p->nip", f_t, w)
    Ydot2 = (torch.einsum("ni,pq->nipq", f_t, dw) + torch.einsum("ni,p,q->nipq", f_tt, w, w)
             + torch.einsum("nil,lq,p->nipq", f_wt, dw, w) + torch.einsum("nil,lp,q->nipq", f_wt, dw, w)
             + torch.einsum("nilm,lp,mq->nipq", f_ww, dw, dw) + torch.einsum("nil,lpq->nipq", f_w, d2w))
    return Y, Ydot, Ydot2


@dataclass
class CoupledModel:
    """A Model whose ``coupled`` nodes follow a reference point at ``rp``
    (Couple, couple.py), with a concentrated force and a moment on the point
    (concentrate_force.py, moment.py).  Reduced DOFs: the base model's free
    node DOFs minus the tied nodes, then the point's 6 DOFs (v, z), in the
    reference's order (instances first, reference points after,
    assembly.py:90-105)."""
    base: Model
    coupled: np.ndarray
    rp: torch.Tensor
    force: torch.Tensor
    moment: torch.Tensor

    def node_free(self):
        m = self.base.free_mask().view(-1, 3).clone()
        m[torch.as_tensor(np.asarray(self.coupled), dtype=torch.int64)] = False
        return m.reshape(-1)

    def split(self, gc):
        nf = int(self.node_free().sum())
        return gc[:nf], gc[nf:nf + 3], gc[nf + 3:nf + 6]

    def offsets(self):
        return self.base.X[torch.as_tensor(np.asarray(self.coupled), dtype=torch.int64)] - self.rp.to(DT)[None, :]

    def node_u(self, gc):
        """Couple.modify_RGC (couple.py:34-40): tied nodes at v + R(z) y - y."""
        g, v, z = self.split(gc)
        u = torch.zeros(self.base.X.shape[0] * 3, dtype=DT)
        u[self.node_free()] = g
        Y = couple_motion(z, self.offsets())[0]
        u = u.view(-1, 3)
        u[torch.as_tensor(np.asarray(self.coupled), dtype=torch.int64)] = v[None, :] + Y
        return u.reshape(-1)

    def assemble(self, gc):
        """Reduced R and coalesced CSR: element and pressure R, K over every
        node DOF at the tied displacement, condensed onto the point's DOFs
        (couple.py:68-166) with P = d u / d gc, plus the point's loads."""
        b = self.base
        N = b.X.shape[0]
        uall = self.node_u(gc)
        full = Model(b.X, b.groups, b.pressures, [])
        full._free = torch.ones(3 * N, dtype=torch.bool)
        R0, (ip, ix, vv) = full.assemble(uall)
        rows = torch.repeat_interleave(torch.arange(3 * N), ip[1:] - ip[:-1])
        K = torch.sparse_coo_tensor(torch.stack([rows, ix]), vv, (3 * N, 3 * N))
        g, v, z = self.split(gc)
        _, Yd, Yd2 = couple_motion(z, self.offsets())
        nf = self.node_free()
        nfree = int(nf.sum())
        n = nfree + 6
        cols = torch.full((3 * N,), -1, dtype=torch.int64)
        cols[nf] = torch.arange(nfree)
        pr, pc, pv = [torch.nonzero(nf).flatten()], [cols[nf]], [torch.ones(nfree, dtype=DT)]
        cn = torch.as_tensor(np.asarray(self.coupled), dtype=torch.int64)
        for q in range(3):
            pr.append(3 * cn + q); pc.append(torch.full_like(cn, nfree + q)); pv.append(torch.ones(cn.shape[0], dtype=DT))
            for p_ in range(3):
                pr.append(3 * cn + q); pc.append(torch.full_like(cn, nfree + 3 + p_)); pv.append(Yd[:, q, p_])
        Pm = torch.sparse_coo_tensor(torch.stack([torch.cat(pr), torch.cat(pc)]), torch.cat(pv), (3 * N, n)).coalesce()
        Pd = Pm.to_dense()
        Kr = Pd.T @ (K.to_dense() @ Pd)
        Rc = R0.view(-1, 3)[cn]
        Kr[nfree + 3:, nfree + 3:] += torch.einsum("ai,aipq->pq", Rc, Yd2)
        R = Pd.T @ R0
        R[nfree:nfree + 3] -= self.force.to(DT)
        R[nfree + 3:] -= self.moment.to(DT)
        # structural pattern: the element pattern's entries (stored zeros
        # included) with every tied DOF spread over all six point DOFs
        Kp = torch.sparse_coo_tensor(torch.stack([rows, ix]), torch.ones_like(vv), (3 * N, 3 * N)).to_dense()
        Ps = (Pd != 0).to(DT)
        Ps[3 * cn[:, None] + torch.arange(3)[None, :], nfree:] = 1.0
        pattern = (Ps.T @ (Kp @ Ps)) != 0
        pattern[nfree:, nfree:] = True
        idx = torch.nonzero(pattern).T
        A = torch.sparse_coo_tensor(idx, Kr[idx[0], idx[1]], (n, n)).coalesce().to_sparse_csr()
        return R, (A.crow_indices(), A.col_indices(), A.values())

    def energy(self, gc):
        """Element and pressure energy at the tied displacement minus the
        point loads' work (assembly.py:389-415)."""
        b = self.base
        uall = self.node_u(gc)
        full = Model(b.X, b.groups, b.pressures, [])
        full._free = torch.ones(3 * b.X.shape[0], dtype=torch.bool)
        g, v, z = self.split(gc)
        return full.energy(uall) - (self.force.to(DT) * v).sum() - (self.moment.to(DT) * z).sum()


# ---------------------------------------------------------------------------
# Solvers
# ---------------------------------------------------------------------------


def csr_matvec(indptr, indices, values, x):
    A = torch.sparse_csr_tensor(indptr, indices, values, (x.shape[0], x.shape[0]))
    return A @ x


def conjugate_gradient(indptr, indices, values, b, x0=None, tol=1e-3, max_iter=1500):
    """Plain CG with the squared-ratio stop test ||r||^2/||b||^2 < tol.

    Follows _linear_solver.conjugate_gradient, FEA/solver/_linear_solver.py:6-42.
    Returns (x, iterations).
    """
    x = torch.zeros_like(b) if x0 is None else x0.clone()
    r_r0 = torch.dot(b, b)
    r = b - csr_matvec(indptr, indices, values, x)
    p = r.clone()
    rs = torch.dot(r, r)
    it = 0
    for it in range(1, max_iter + 1):
        Ap = csr_matvec(indptr, indices, values, p)
        a = rs / torch.dot(p, Ap)
        x = x + a * p
        r = r - a * Ap
        rsn = torch.dot(r, r)
        if rsn / r_r0 < tol:
            break
        p = r + rsn / rs * p
        rs = rsn
    return x, it


def jacobi_scaled_cg(indptr, indices, values, R, x0, tol=1e-5, max_iter=1500):
    """Symmetric Jacobi scaling d = sqrt|diag K| then CG on D^-1 K D^-1.

    Follows StaticImplicitSolver._solve_linear_equation, static_implicit.py:
    352-405 (diag from the COO diagonal, zero diag -> 1, x0 = dGC0 * d, result
    divided by d).
    """
    n = R.shape[0]
    rows = torch.repeat_interleave(torch.arange(n), indptr[1:] - indptr[:-1])
    diag = torch.zeros(n, dtype=DT).scatter_add_(0, rows[rows == indices], values[rows == indices]).abs().sqrt()
    diag[diag == 0] = 1.0
    vs = values / diag[rows] / diag[indices]
    y, it = conjugate_gradient(indptr, indices, vs, R / diag, x0 * diag, tol, max_iter)
    return y / diag, it


def direct_solve(indptr, indices, values, b):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    n = b.shape[0]
    A = sp.csr_matrix((values.numpy(), indices.numpy(), indptr.numpy()), shape=(n, n))
    return torch.from_numpy(spla.spsolve(A.tocsc(), b.numpy()))


def newton_solve(model: Model, gc0, tol_error=1e-5, max_iter=100, rtol=None, linear="direct",
                 cg_tol=1e-5, cg_max=6000):
    """Newton with Armijo backtracking on the total potential.

    Follows StaticImplicitSolver._solve_iteration and _line_search,
    static_implicit.py:153-350 (c1 = 0.3, halving, alpha < 1e-12 -> 0; stop
    when (max|dGC| < tol and max|R| < tol) or max|R| < 1e-6).  With ``rtol``
    set, the stop test is instead ||R||/||R(gc0)|| <= rtol.
    Returns (gc, iterations).
    """
    gc = gc0.clone()
    energy = model.energy(gc)
    dgc = torch.zeros_like(gc)
    r_ref = None
    it = 0
    while it < max_iter:
        R, (ip, ix, vv) = model.assemble(gc)
        if r_ref is None:
            r_ref = R.norm()
        it += 1
        if rtol is not None and R.norm() <= rtol * r_ref:
            break
        if linear == "direct":
            dgc = direct_solve(ip, ix, vv, -R)
        else:
            dgc, _ = jacobi_scaled_cg(ip, ix, vv, -R, dgc, cg_tol, cg_max)
        # line search (static_implicit.py:153-232)
        alpha, c1 = 1.0, 0.3
        dE = (dgc * R).sum()
        if dE > 0:
            dgc, dE = -dgc, -dE
        while True:
            trial = gc + alpha * dgc
            e_new = model.energy(trial)
            if torch.isnan(e_new) or torch.isinf(e_new) or e_new > energy + c1 * dE * alpha:
                alpha *= 0.5
                if alpha < 1e-12:
                    alpha, trial, e_new = 0.0, gc.clone(), energy
                    break
            else:
                break
        if alpha == 0.0:
            break
        gc, energy = trial, e_new
        if rtol is None and ((dgc.abs().max() < tol_error and R.abs().max() < tol_error)
                             or R.abs().max() < 1e-6):
            break
    return gc, it


def explicit_run(model: Model, gc0, gv0, dt, steps):
    """Central difference with half-step velocity and lumped mass.

    Follows DynamicExplicitSolver.solve, dynamic_explicit.py:66-145.
    Returns (u, v, a) after ``steps`` steps (v is the averaged velocity).
    """
    minv = model.lumped_mass_inv()
    a = minv * -model.assemble(gc0, want_K=False)[0]
    vh_prev = gv0 - 0.5 * dt * a
    u = gc0.clone()
    v = gv0.clone()
    for _ in range(steps):
        vh = vh_prev + dt * a
        u = u + dt * vh
        a = minv * -model.assemble(u, want_K=False)[0]
        v = 0.5 * (vh + vh_prev)
        vh_prev = vh
    return u, v, a


def newmark_run(model: Model, gc0, gv0, dt, steps, tol_error=1e-5, max_iter=10000, beta=0.25, gamma=0.5):
    """Implicit Newmark dynamics with Newton per step and direct solves.

    Follows DynamicImplicitSolver (dynamic_implicit.py): the initial
    acceleration solves M a0 = R(gc0) with R the assembled residual, as
    written there (:300-302); each step predicts gc_pre = gc + dt v +
    dt^2 a / 4 (:180) and minimises the incremental energy
    Pi(x) + (x - gc_pre) M (x - gc_pre) / (2 beta dt^2) (:103-114) by Newton
    on R + M (x - gc_pre) / (beta dt^2) with tangent K + M / (beta dt^2)
    (:116-146) and Armijo backtracking (c1 = 0.3, halving, alpha < 1e-12 ->
    0, :304-351); the Newton loop (:353-460) stops when max|dx| < tol and
    max|R| < tol.  The CPU direct solve stands for its solver on the CPU
    (:487-493).  Velocity and acceleration follow :269-289.
    Returns the lists (GC, GV, GA), one entry per stored time.
    """
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    Mm = model.mass_matrix()
    c = 1.0 / (beta * dt * dt)

    def inc_energy(x, pre):
        d = (x - pre).numpy()
        return float(model.energy(x)) + float(d @ (Mm @ d)) * c / 2

    def next_va(x, x0, v0, a0):
        v = gamma / (beta * dt) * (x - x0) + (1 - gamma / beta) * v0 + dt * (1 - gamma / (2 * beta)) * a0
        a = c * (x - x0) - v0 / (beta * dt) - (1 / (2 * beta) - 1) * a0
        return v, a

    R0 = model.assemble(gc0, want_K=False)[0]
    a0 = torch.from_numpy(spla.spsolve(Mm.tocsc(), R0.numpy()))
    GC, GV, GA = [gc0.clone()], [gv0.clone()], [a0]
    for _ in range(steps):
        pre = GC[-1] + dt * GV[-1] + 0.25 * dt * dt * GA[-1]
        x = GC[-1].clone()
        energy = inc_energy(x, pre)
        low_alpha, it = 0, 0
        while True:
            if it > max_iter:
                raise RuntimeError("Newton did not converge")
            Rv, (ip, ix, vv) = model.assemble(x)
            d = (x - pre).numpy()
            R = Rv + torch.from_numpy(Mm @ d) * c
            n = R.shape[0]
            K = sp.csr_matrix((vv.numpy(), ix.numpy(), ip.numpy()), shape=(n, n)) + Mm * c
            it += 1
            dx = torch.from_numpy(spla.spsolve(K.tocsc(), -R.numpy()))
            alpha, c1 = 1.0, 0.3
            dE = float((dx * R).sum())
            if dE > 0:
                dx, dE = -dx, -dE
            while True:
                trial = x + alpha * dx
                e_new = inc_energy(trial, pre)
                if not math.isfinite(e_new) or e_new > energy + c1 * dE * alpha:
                    alpha *= 0.5
                    if alpha < 1e-12:
                        alpha, trial, e_new = 0.0, x.clone(), energy
                        break
                else:
                    break
            rmax = float(R.abs().max())
            if alpha == 0.0 and rmax > tol_error:
                raise RuntimeError("line search failed")
            if alpha == 0.0:
                break
            low_alpha = low_alpha + 1 if alpha < 0.01 else max(0, low_alpha - 5)
            if low_alpha > 10:
                if rmax < 1e-3:
                    break
                raise RuntimeError("Newton stalled")
            x, energy = trial, inc_energy(trial, pre)
            if float(dx.abs().max()) < tol_error and rmax < tol_error:
                break
        v, a = next_va(x, GC[-1], GV[-1], GA[-1])
        GC.append(x); GV.append(v); GA.append(a)
    return GC, GV, GA


# ---------------------------------------------------------------------------
# Synthetic meshes of the benchmark configurations (seeded)
# ---------------------------------------------------------------------------


def grid_nodes(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0):
    gx = np.linspace(0, lx, nx + 1)
    gy = np.linspace(0, ly, ny + 1)
    gz = np.linspace(0, lz, nz + 1)
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)


def _nid(i, j, k, ny, nz):
    return (i * (ny + 1) + j) * (nz + 1) + k


def hex_block(n, jitter=0.0, seed=0, dims=None, lengths=(1.0, 1.0, 1.0)):
    """Structured C3D8 block with optional seeded nodal jitter U(-j h, j h)."""
    nx, ny, nz = dims if dims is not None else (n, n, n)
    nodes = grid_nodes(nx, ny, nz, *lengths)
    if jitter:
        h = np.array([lengths[0] / nx, lengths[1] / ny, lengths[2] / nz])
        nodes = nodes + np.random.default_rng(seed).uniform(-1, 1, nodes.shape) * jitter * h
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    f = lambda a, b, c: _nid(a, b, c, ny, nz)
    el = np.stack([f(i, j, k), f(i + 1, j, k), f(i + 1, j + 1, k), f(i, j + 1, k),
                   f(i, j, k + 1), f(i + 1, j, k + 1), f(i + 1, j + 1, k + 1), f(i, j + 1, k + 1)], 1)
    return torch.tensor(nodes, dtype=DT), torch.tensor(el, dtype=torch.int64)


def tet_block(n, dims=None, lengths=(1.0, 1.0, 1.0)):
    """Hex grid with every cell Kuhn-split into 6 positively oriented C3D4.

    The 6 tets follow the paths 0 -> x -> y -> z permutations along the cell's
    0-6 diagonal; tets with negative volume get two nodes swapped.
    """
    nx, ny, nz = dims if dims is not None else (n, n, n)
    nodes = grid_nodes(nx, ny, nz, *lengths)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    off = {1: (1, 0, 0), 2: (0, 1, 0), 4: (0, 0, 1)}
    paths = [(1, 2, 4), (1, 4, 2), (2, 1, 4), (2, 4, 1), (4, 1, 2), (4, 2, 1)]
    tets = []
    for pth in paths:
        c = np.zeros(3, dtype=np.int64)
        t = [_nid(i, j, k, ny, nz)]
        for s in pth:
            c = c + np.array(off[s])
            t.append(_nid(i + c[0], j + c[1], k + c[2], ny, nz))
        tets.append(np.stack(t, 1))
    el = np.stack(tets, 1).reshape(-1, 4)               # cell-major, 6 tets per cell
    x = nodes[el]
    v = np.einsum("ei,ei->e", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]), x[:, 3] - x[:, 0])
    neg = v < 0
    el[neg] = el[neg][:, [0, 2, 1, 3]]
    return torch.tensor(nodes, dtype=DT), torch.tensor(el, dtype=torch.int64)


def boundary_faces(kind, elems, X, axis, value, tol=1e-9):
    """Faces (node lists in the element's outward face order) lying on a plane."""
    res = []
    on = (X[:, axis] - value).abs() < tol
    for fid, loc in FACES[kind].items():
        f = elems[:, loc]
        m = on[f].all(dim=1)
        if m.any():
            res.append((torch.nonzero(m).flatten(), fid, f[m]))
    return res
