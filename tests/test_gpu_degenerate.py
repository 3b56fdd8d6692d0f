"""Degenerate inputs through the CUDA path.

- An element group without elements beside a populated one (C3D8 and
  C3D4): the same reduced pattern as the populated group alone; the empty
  group's assembly, residual-only pass and energy add nothing, so both
  groups accumulated into zeroed buffers give the populated group's values
  bit for bit; a pressure load on an empty face group adds nothing either.
- A mesh whose every DOF is fixed: an empty reduced system; the entry points
  take NULL for the (empty) solution, residual and matrix and the energy of
  the undeformed mesh is zero.
"""
import numpy as np
import pytest
import torch

from oracle import fea_oracle as O

pytestmark = pytest.mark.gpu

MU, KAPPA = 1.0, 10.0


def _mesh(kind, n):
    X, el = (O.hex_block(n, jitter=0.1, seed=3) if kind == "C3D8" else O.tet_block(n))
    return X.numpy(), el.numpy().astype(np.int32)


@pytest.mark.parametrize("kind,n", [("C3D8", 3), ("C3D4", 2)])
def test_empty_group_beside_a_populated_one(kind, n):
    from fea_b200.plan import DevicePlan
    X, el = _mesh(kind, n)
    N = X.shape[0]
    free = np.full(N, 7, np.uint8)
    free[:(n + 1) ** 2] = 0                                   # the plane x = 0 clamped
    empty = np.zeros((0, el.shape[1]), np.int32)
    P1 = DevicePlan(X, free, [(kind, el)])
    no_faces = ("Q4", np.zeros((0, 4), np.int32)) if kind == "C3D8" else ("T3", np.zeros((0, 3), np.int32))
    P2 = DevicePlan(X, free, [(kind, empty), (kind, el)], faces=[no_faces])
    assert P2.groups[0].ne == 0 and not P2.groups[0].covers_active
    assert P1.nnz == P2.nnz and P1.ndof == P2.ndof
    assert torch.equal(P1.indptr, P2.indptr) and torch.equal(P1.indices, P2.indices)
    gc = (1e-3 * torch.randn(P1.ndof, generator=torch.Generator().manual_seed(5), dtype=torch.float64)).cuda()
    K1, R1 = P1.zeros(P1.nnz), P1.zeros(P1.ndof)
    P1.assemble_volume(0, MU, KAPPA, gc, K=K1, R=R1)
    K2, R2 = P2.zeros(P2.nnz), P2.zeros(P2.ndof)
    P2.assemble_volume(0, MU, KAPPA, gc, K=K2, R=R2, accumulate=True)
    torch.cuda.synchronize()
    assert not K2.any() and not R2.any()                      # the empty group adds nothing
    P2.assemble_volume(1, MU, KAPPA, gc, K=K2, R=R2, accumulate=True)
    assert torch.equal(K1, K2) and torch.equal(R1, R2)
    # a pressure load on no face adds nothing and encloses no volume
    P2.assemble_pressure(0, 0.1, P2.X, gc, K=K2, R=R2)
    vol = P2.zeros(1)
    vol.fill_(7.0)
    P2.pressure_volume(0, P2.X, gc, vol)
    assert torch.equal(K1, K2) and torch.equal(R1, R2) and float(vol) == 0.0
    # the residual-only pass (its own kernel: the same bits as the populated
    # group's R-only pass alone, the K pass's residual to rounding)
    Rr1, Rr = P1.zeros(P1.ndof), P2.zeros(P2.ndof)
    P1.assemble_volume(0, MU, KAPPA, gc, R=Rr1)
    P2.assemble_volume(0, MU, KAPPA, gc, R=Rr, accumulate=True)
    torch.cuda.synchronize()
    assert not Rr.any()
    P2.assemble_volume(1, MU, KAPPA, gc, R=Rr, accumulate=True)
    assert torch.equal(Rr, Rr1)
    assert float((Rr - R1).norm() / R1.norm()) < 1e-13
    # energies: zero for the empty group, the populated group's unchanged
    e1, e2 = P1.zeros(1), P2.zeros(2)
    P1.energy_volume(0, MU, KAPPA, gc, e1)
    P2.energy_volume(0, MU, KAPPA, gc, e2[0:1])
    P2.energy_volume(1, MU, KAPPA, gc, e2[1:2])
    assert float(e2[0]) == 0.0 and float(e2[1]) == float(e1[0])
    # against the oracle
    u = torch.zeros(N * 3, dtype=torch.float64)
    fr = torch.from_numpy(np.repeat(free == 7, 3))
    u[fr] = gc.cpu()
    Re, _ = O.element_residual_tangent(kind, torch.from_numpy(X), torch.from_numpy(el).long(), u.view(N, 3), MU, KAPPA,
                                       want_K=False)
    R0 = torch.zeros(N * 3, dtype=torch.float64)
    R0.scatter_add_(0, O.element_force_index(torch.from_numpy(el).long()).view(-1), Re.reshape(-1))
    assert float((R1.cpu() - R0[fr]).norm() / R0[fr].norm()) < 1e-12


def test_fully_fixed_mesh_has_an_empty_system():
    from fea_b200.plan import DevicePlan
    X, el = _mesh("C3D8", 2)
    N = X.shape[0]
    P = DevicePlan(X, np.zeros(N, np.uint8), [("C3D8", el)])
    assert P.ndof == 0 and P.nnz == 0
    gc, K, R = P.zeros(0), P.zeros(0), P.zeros(0)
    P.assemble_volume(0, MU, KAPPA, gc, K=K, R=R)             # NULL solution, matrix and residual: no work
    out = P.zeros(1)
    out.fill_(7.0)
    P.energy_volume(0, MU, KAPPA, gc, out)                    # the undeformed mesh
    assert abs(float(out)) < 1e-14


def test_bad_buffers_are_refused_before_any_launch():
    """A caller's K / R / gc that is on the host, of another dtype, too short
    or strided raises ValueError and launches nothing."""
    from fea_b200 import _lib as L
    from fea_b200.plan import DevicePlan
    X, el = _mesh("C3D8", 2)
    N = X.shape[0]
    P = DevicePlan(X, np.full(N, 7, np.uint8), [("C3D8", el)])
    gc = P.zeros(P.ndof)
    K, R = P.zeros(P.nnz), P.zeros(P.ndof)
    P.assemble_volume(0, MU, KAPPA, gc, K=K, R=R)
    torch.cuda.synchronize()
    n0 = L.fea_launch_count()
    bad = [dict(K=K.cpu()), dict(K=K.float()), dict(K=K[:-1]), dict(R=P.zeros(2 * P.ndof)[::2]),
           dict(gc=gc[:-1])]
    for b in bad:
        args = dict(gc=gc, K=K, R=R)
        args.update(b)
        with pytest.raises(ValueError):
            P.assemble_volume(0, MU, KAPPA, args.pop("gc"), **args)
    assert L.fea_launch_count() == n0
