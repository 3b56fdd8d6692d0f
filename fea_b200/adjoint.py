"""Sensitivities of the static equilibrium by a hand-written adjoint.

The reference obtains shape and material sensitivities by differentiating
its torch graph: it forms work = (R(X) . lam) with a precomputed adjoint
field lam and calls autograd on it (tests/gradient_test/test_grad.py:
87-99).  Here the same vector-Jacobian products come from dedicated kernels
(``fea_adjoint_vjp_volume``, ``fea_adjoint_hvp_pressure``), and the
compliance gradient is assembled from them:

    C(X, mu) = f_ext . u,      R(u; X, mu) = 0,     f_ext = -p dV/dx,
    K lam = dC/du = f_ext - p (d2V/dx2) u        (K symmetric)
    dC/dX = -p (d2V/dx2) u - [lam . dR_int/dX + p (d2V/dx2) lam]
    dC/dmu = -lam . dR_int/dmu

(R = R_int + p dV/dx is the reduced residual of Assembly.assemble_force.)
"""
from __future__ import annotations

import torch


def _full(asm, reduced):
    """Reduced DOF vector -> all-DOF vector [N_total, 3] with zeros on
    Dirichlet and unused DOFs."""
    full = torch.zeros(asm.RGC_list_indexStart[-1], dtype=torch.float64, device=asm.device)
    full[asm._remain_dev] = reduced
    return full.view(-1, 3)


def residual_vjp(asm, GC, lam):
    """lam . dR/dX for every node ([N_total, 3]) and lam . dR/dmu per element
    group, R = reduced residual at GC, lam a reduced vector.  This is the
    quantity the reference obtains with autograd of (R . lam)."""
    P = asm.plan
    gc = asm._gc(GC=GC)
    lam_full = _full(asm, torch.as_tensor(lam, dtype=torch.float64, device=asm.device)).contiguous()
    dX = torch.zeros(P.n_nodes, 3, dtype=torch.float64, device=asm.device)
    dmu = []
    for gi, e in enumerate(asm._mat_elems):
        mu, kappa = e.materials.parameters()
        out = torch.zeros(1, dtype=torch.float64, device=asm.device)
        P.adjoint_vjp_volume(gi, mu, kappa, gc, lam_full, dX, out)
        dmu.append(out[0])
    for fi, ld in enumerate(asm._face_loads):
        P.adjoint_hvp_pressure(fi, float(ld.pressure), asm._Xinst, gc, lam_full, dX)
    return _to_part_frames(asm, dX), dmu


def _to_part_frames(asm, dX):
    """Coordinate gradients with respect to each part's own nodes: a rotated
    instance evaluates its elements at X R^T (and its loads at X R^T + t), so
    the gradient with respect to X is the assembly-frame one times R."""
    for name, ins in asm._instances.items():
        R = ins.rotation_matrix.to(torch.float64)
        if torch.equal(R, torch.eye(3, dtype=torch.float64)):
            continue
        o = asm._node_offset[name]
        n = ins.part.nodes.shape[0]
        dX[o:o + n] = dX[o:o + n] @ R.to(dX.device)
    return dX


def pressure_hvp(asm, GC, v_full):
    """sum over pressure loads of p (d2V/dx2) v for every node ([N_total, 3])."""
    P = asm.plan
    gc = asm._gc(GC=GC)
    out = torch.zeros(P.n_nodes, 3, dtype=torch.float64, device=asm.device)
    for fi, ld in enumerate(asm._face_loads):
        P.adjoint_hvp_pressure(fi, float(ld.pressure), asm._Xinst, gc, v_full.contiguous(), out)
    return out


def external_force(asm, GC):
    """f_ext = -p dV/dx over the reduced DOFs (the load part of the residual)."""
    P = asm.plan
    gc = asm._gc(GC=GC)
    Rp = P.zeros(P.ndof)
    for fi, ld in enumerate(asm._face_loads):
        P.assemble_pressure(fi, float(ld.pressure), asm._Xinst, gc, K=None, R=Rp)
    return -Rp


def compliance_gradient(asm, GC, pcg_tol=1e-26, pcg_max_iter=200000, return_lambda=False):
    """(C, dC/dX [N_total, 3], [dC/dmu per group], adjoint iterations) at an
    equilibrium GC; with return_lambda, the adjoint field is appended."""
    P = asm.plan
    gc = asm._gc(GC=GC)
    R, K = asm.assemble_csr(gc)
    f = external_force(asm, gc)
    C = torch.dot(f, gc)
    u_full = _full(asm, gc)
    Hu = pressure_hvp(asm, gc, u_full)
    rhs = (f - Hu.reshape(-1)[asm._remain_dev]).contiguous()
    lam = torch.zeros_like(rhs)
    it, rr, st = P.pcg(K, rhs, lam, pcg_tol, pcg_max_iter, check_every=50)
    dX, dmu = residual_vjp(asm, gc, lam)
    dCdX = -(dX + _to_part_frames(asm, Hu))
    if return_lambda:
        return C, dCdX, [-d for d in dmu], it, lam
    return C, dCdX, [-d for d in dmu], it


class ComplianceFunction(torch.autograd.Function):
    """C(X, mu) of an assembly with one instance and one element group.

    forward(X [N,3], mu 0-d, assembly, solver) solves the equilibrium for the
    given nodal coordinates and shear modulus and returns the compliance;
    backward returns dC/dX and dC/dmu from the adjoint.
    """

    @staticmethod
    def forward(ctx, X, mu, asm, solver):
        set_coordinates(asm, X)
        e = asm._mat_elems[0]
        e.materials.mu = torch.as_tensor(float(mu), dtype=torch.float64)
        gc = solver.solve(GC0=torch.zeros_like(asm.GC))
        if isinstance(gc, bool):
            raise RuntimeError("equilibrium solve failed")
        C, dX, dmu, _ = compliance_gradient(asm, gc)
        # gradients are returned on the devices of the inputs they belong to
        ctx.save_for_backward(dX.to(X.device), dmu[0].reshape(()).to(torch.as_tensor(mu).device))
        return C.detach().reshape(()).to(X.device)

    @staticmethod
    def backward(ctx, g):
        dX, dmu = ctx.saved_tensors
        return g.to(dX.device) * dX, g.to(dmu.device) * dmu, None, None


def set_coordinates(asm, X):
    """Replace the reference coordinates of a one-instance assembly in place."""
    if len(asm._instances) != 1:
        raise NotImplementedError("set_coordinates covers one instance")
    ins = next(iter(asm._instances.values()))
    X = torch.as_tensor(X, dtype=torch.float64)
    ins.part.nodes = X.detach().cpu().clone()
    P = asm.plan
    P.X.copy_(asm._element_frame_nodes(ins).to(P.device))
    asm._Xinst.copy_(ins.nodes.to(P.device))
