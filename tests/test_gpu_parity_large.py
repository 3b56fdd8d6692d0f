"""Parity on the benchmarked configurations themselves, through the CUDA path.

- The 64^3 jittered C3D8 block of the assembly benchmark (262,144 elements,
  63,695,790 nonzeros): reduced CSR bit-exact against the oracle's
  node-level pattern; the full residual and, on three node planes (next to
  the clamp, the middle, the loaded face), every K entry of those rows
  within 1e-12 of the oracle's element arithmetic.
- The 2.06M-tet explicit cube: three central-difference steps against the
  oracle's loop, within 1e-12.
- The 40^3 compliance block: the residual VJP (lam . dR/dX, lam . dR/dmu)
  against torch autograd of the oracle's residual, within 1e-12.
- C3D8 fans whose middle axis node has 50 and 162 active neighbours: rows
  longer than one pass of the node-row gather, and (162) staged regions too
  large for two nodes per warp, against the oracle.
"""
import math

import numpy as np
import pytest
import torch

from oracle import fea_oracle as O
from tests.helpers import rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rows_oracle_K(X, el, u, mu, kappa, free, rid, row_nodes, faces=None, p=0.0):
    """Coalesced reduced COO of the K rows of ``row_nodes`` from the oracle's
    element arithmetic over the elements (and pressure faces) touching them:
    (rows, cols, values) sorted by (row, col)."""
    want = torch.zeros(X.shape[0], dtype=torch.bool)
    want[row_nodes] = True
    sel = want[el].any(1)
    els = el[sel]
    rows, cols, vals = [], [], []
    _, Ke = O.element_residual_tangent("C3D8", X, els, u, mu, kappa)        # [a,j,b,k,e]
    nn = els.shape[1]
    j3 = torch.arange(3)
    ra = (3 * els.T[:, None, None, None, :] + j3[None, :, None, None, None]).expand(nn, 3, nn, 3, -1)
    cb = (3 * els.T[None, None, :, None, :] + j3[None, None, None, :, None]).expand(nn, 3, nn, 3, -1)
    rows.append(ra.reshape(-1)); cols.append(cb.reshape(-1)); vals.append(Ke.reshape(-1))
    fs = faces[want[faces].any(1)] if faces is not None else None
    if fs is not None and fs.shape[0] > 0:
        _, k = O.pressure_force_tangent(X + u, fs, p)                       # [f,i,a,j,b]
        nf = fs.shape[1]
        ra = (3 * fs[:, None, :, None, None] + j3[None, :, None, None, None]).expand(-1, 3, nf, 3, nf)
        cb = (3 * fs[:, None, None, None, :] + j3[None, None, None, :, None]).expand(-1, 3, nf, 3, nf)
        rows.append(ra.reshape(-1)); cols.append(cb.reshape(-1)); vals.append(-k.reshape(-1))
    rows, cols, vals = torch.cat(rows), torch.cat(cols), torch.cat(vals)
    keep = want[rows // 3] & free[rows] & free[cols]
    n = int(free.sum())
    A = torch.sparse_coo_tensor(torch.stack([rid[rows[keep]], rid[cols[keep]]]), vals[keep], (n, n)).coalesce()
    return A.indices()[0], A.indices()[1], A.values()


@pytest.fixture(scope="module")
def block64():
    import bench
    asm, el, X, load = bench.build_block_model(64)
    return asm, torch.from_numpy(el), torch.from_numpy(X)


def test_config2_csr_bit_exact(block64):
    asm, el, X = block64
    n = 64
    N = X.shape[0]
    free = np.ones((N, 3), dtype=bool)
    free[:(n + 1) * (n + 1)] = False                       # node plane i = 0 clamped
    ip, ix = O.reduced_pattern_csr([el.numpy()], free, N)
    P = asm.plan
    assert P.nnz == 63695790 and ip[-1] == P.nnz
    assert np.array_equal(P.indptr.cpu().numpy(), ip)
    assert np.array_equal(P.indices.cpu().numpy().astype(np.int64), ix)


def test_config2_residual_and_tangent_rows(block64):
    asm, el, X = block64
    n, mu, kappa, p = 64, 1.0, 50.0, 0.02
    N = X.shape[0]
    P = asm.plan
    gc = 1e-3 * torch.randn(P.ndof, generator=torch.Generator().manual_seed(0), dtype=torch.float64)
    R, Kidx, Kv = asm.assemble_Stiffness_Matrix(GC=gc.cuda())
    R, Kv = R.cpu(), Kv.cpu()
    ip, ix = P.indptr.cpu(), P.indices.cpu().to(torch.int64)
    free = torch.ones(N * 3, dtype=torch.bool)
    free[:3 * (n + 1) * (n + 1)] = False
    rid = torch.cumsum(free.to(torch.int64), 0) - 1
    u = torch.zeros(N * 3, dtype=torch.float64)
    u[free] = gc
    u = u.view(N, 3)
    E = el.shape[0]
    end = torch.nonzero(torch.arange(E) // (n * n) == n - 1).flatten()
    faces = el[end][:, [1, 2, 6, 5]]
    # the whole residual
    R0 = torch.zeros(N * 3, dtype=torch.float64)
    force = O.element_force_index(el).view(-1, E)
    for e0 in range(0, E, 32768):
        Re, _ = O.element_residual_tangent("C3D8", X, el[e0:e0 + 32768], u, mu, kappa, want_K=False)
        R0.scatter_add_(0, force[:, e0:e0 + 32768].reshape(-1), Re.reshape(-1))
    f, _ = O.pressure_force_tangent(X + u, faces, p, want_K=False)
    fi = torch.stack([3 * faces, 3 * faces + 1, 3 * faces + 2], dim=1)
    R0.scatter_add_(0, fi.reshape(-1), -f.reshape(-1))
    assert rel(R, R0[free]) < TOL
    # K rows of three node planes, entry by entry
    for i in (1, 32, 64):
        nodes = torch.arange(i * (n + 1) ** 2, (i + 1) * (n + 1) ** 2)
        r, c, v = _rows_oracle_K(X, el, u, mu, kappa, free, rid, nodes, faces, p)
        rows = torch.unique(r)
        lo, hi = int(ip[rows[0]]), int(ip[rows[-1] + 1])
        assert torch.equal(rows, torch.arange(int(rows[0]), int(rows[-1]) + 1))   # contiguous free rows
        gr = torch.repeat_interleave(torch.arange(int(rows[0]), int(rows[-1]) + 1), ip[rows[0] + 1:rows[-1] + 2] -
                                     ip[rows[0]:rows[-1] + 1])
        assert torch.equal(gr, r) and torch.equal(ix[lo:hi], c)
        assert rel(Kv[lo:hi], v) < TOL, i


def test_config3_explicit_steps_2M_tets():
    import fea_b200 as F
    from fea_b200 import meshes
    X, el = meshes.tet_block(70)
    assert el.shape[0] == 2058000
    part = F.Part(X)
    e = F.elements.C3D4(elems=el, elems_index=np.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 10.0))
    e.set_density(1.0)
    part.add_element(e)
    asm = F.Assembly()
    asm.add_part(part, "cube")
    asm.add_instance(F.Instance(part), "cube")
    asm.initialize()
    P = asm.plan
    sol = F.solver.DynamicExplicitSolver()
    sol.assembly = asm
    dt = sol.cfl_timestep(0.5)
    v0 = 0.01 * torch.randn(P.ndof, generator=torch.Generator().manual_seed(0), dtype=torch.float64)
    minv = asm.lumped_mass_inv()
    u = torch.zeros(P.ndof, dtype=torch.float64, device="cuda")
    v = v0.cuda()
    vh, acc = torch.empty_like(u), torch.empty_like(u)
    P.explicit_run(0, 1.0, 10.0, minv, dt, 0, u, vh, acc, v, init=True)
    steps = 3
    P.explicit_run(0, 1.0, 10.0, minv, dt, steps, u, vh, acc, v, init=False)
    m = O.Model(torch.from_numpy(X), [O.Group("C3D4", torch.from_numpy(el), 1.0, 10.0, 1.0)], [], [])
    assert rel(minv, m.lumped_mass_inv()) < 1e-14
    uo, vo, ao = O.explicit_run(m, torch.zeros(P.ndof, dtype=torch.float64), v0, dt, steps)
    assert rel(u, uo) < TOL and rel(v, vo) < TOL and rel(acc, ao) < TOL


def test_config5_residual_vjp_40cube():
    import fea_b200 as F
    from fea_b200 import adjoint
    n, mu, kappa, p = 40, 1.0, 50.0, 0.03
    X, el = O.hex_block(n, jitter=0.1, seed=0)
    E = el.shape[0]
    top = torch.nonzero(torch.arange(E) % n == n - 1).flatten()            # k = n - 1 layer, face 1
    faces = el[top][:, [4, 5, 6, 7]]
    bottom = torch.nonzero(torch.arange(X.shape[0]) % (n + 1) == 0).flatten()
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=torch.arange(E), part=part)
    e.set_materials(F.materials.NeoHookean(mu, kappa))
    part.add_element(e)
    part.add_surface_set("top", [(top.numpy(), 1)])
    part.set_nodes["bottom"] = bottom.numpy()
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    asm.add_load(F.loads.Pressure("p", "top", p))
    asm.add_boundary(F.boundarys.Boundary_Condition("p", "bottom"))
    asm.initialize()
    g = torch.Generator().manual_seed(5)
    gc = 1e-3 * torch.randn(asm.GC.shape, generator=g, dtype=torch.float64)
    lam = torch.randn(asm.GC.shape, generator=g, dtype=torch.float64)
    dX, dmu = adjoint.residual_vjp(asm, gc.cuda(), lam.cuda())
    Xg = X.clone().requires_grad_(True)
    mug = torch.tensor(mu, dtype=torch.float64, requires_grad=True)
    m = O.Model(Xg, [O.Group("C3D8", el, mug, kappa)], [O.PressureLoad(faces, p)], [(bottom, (0, 1, 2))])
    Ro, _ = m.assemble(gc, want_K=False)
    (Ro * lam).sum().backward()
    assert rel(dX, Xg.grad) < TOL
    assert abs(float(dmu[0]) - float(mug.grad)) <= TOL * abs(float(mug.grad))


def fan_mesh(M=12, layers=2):
    """C3D8 fan around the z axis: M kite-shaped sectors (axis node, ring
    node, outer node, next ring node) extruded over ``layers`` layers; the
    inner axis node is shared by 2M hexes and has 3 + 6M neighbours, 2 + 4M
    of them active when the bottom plane is clamped."""
    th = 2 * math.pi * np.arange(M) / M
    ring = np.stack([np.cos(th), np.sin(th)], 1)
    outer = 1.6 * np.stack([np.cos(th + math.pi / M), np.sin(th + math.pi / M)], 1)
    plane = np.concatenate([[[0.0, 0.0]], ring, outer])               # 0: axis, 1..M ring, M+1..2M outer
    P2 = plane.shape[0]
    X = np.concatenate([np.concatenate([plane, np.full((P2, 1), 0.4 * z)], 1) for z in range(layers + 1)])
    X = X + np.random.default_rng(3).uniform(-0.02, 0.02, X.shape)
    quads = np.array([[0, 1 + i, 1 + M + i, 1 + (i + 1) % M] for i in range(M)])
    el = np.concatenate([np.concatenate([quads + z * P2, quads + (z + 1) * P2], 1) for z in range(layers)])
    return torch.from_numpy(X), torch.from_numpy(el.astype(np.int64))


@pytest.mark.parametrize("M", [12, 40])
def test_high_valence_c3d8_node_rows(M):
    """M = 12: rows of 50 blocks, more than one pass of a 16- or 32-lane
    node group.  M = 40: the middle axis node stages 12 M = 480 blocks, two
    such regions per warp exceed the 227 KB of shared memory of a CTA and the
    gather falls back to one node per warp."""
    import fea_b200 as F
    X, el = fan_mesh(M)
    dNdX, w, _ = O.preload_gaussian("C3D8", X, el)
    assert bool((w > 0).all())                               # valid hexes at every Gauss point
    P2 = 1 + 2 * M
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=torch.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 50.0))
    part.add_element(e)
    fixed = np.arange(P2)                                     # bottom plane clamped
    part.set_nodes["fix"] = fixed
    asm = F.Assembly()
    asm.add_part(part, "p")
    asm.add_instance(F.Instance(part), "p")
    asm.add_boundary(F.boundarys.Boundary_Condition("p", "fix"))
    asm.initialize()
    P = asm.plan
    adj = P.adjptr.cpu().numpy() if hasattr(P, "adjptr") else None
    if adj is not None:
        assert int(np.diff(adj).max()) == 2 + 4 * M              # the middle axis node's row
    maxblk = int(P.groups[0].desc.maxblk)
    assert maxblk == 12 * M
    assert (8 * maxblk * 72 > 227 * 1024) == (M == 40)        # two regions per warp do not fit
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 50.0)], [], [(fixed, (0, 1, 2))])
    gc = 1e-2 * torch.randn(int(m.free_mask().sum()), generator=torch.Generator().manual_seed(7),
                            dtype=torch.float64)
    Ro, (ip, ix, vv) = m.assemble(gc)
    assert torch.equal(P.indptr.cpu(), ip) and torch.equal(P.indices.cpu().to(torch.int64), ix)
    for _ in range(2):
        R, Kidx, Kv = asm.assemble_Stiffness_Matrix(GC=gc.cuda())
        assert rel(R, Ro) < TOL and rel(Kv, vv) < TOL
    assert rel(asm.assemble_force(GC=gc.cuda()), Ro) < TOL
