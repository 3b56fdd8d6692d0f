"""Constraints (mirrors FEA/assemble/constraints of sssnnn7119/FEA).

``Couple`` ties the nodes of a node set to the rigid motion of a reference
point (couple.py:7-282): node b moves by v + R(z) y_b - y_b, where y_b is its
offset from the point in the assembly frame, v the point's translation and
R(z) the rotation by the rotation vector z (Rodrigues' formula in the angle
|z| + 1e-20 and the axis z / angle, as the reference writes it).  The tied
nodes' DOFs leave the reduced system; the point's six DOFs enter it.  The
condensation of R and K onto the point is done by ``coupled.CoupledSystem``
from the plan's element R and K.
"""
from __future__ import annotations

import numpy as np
import torch


class BaseConstraint:
    def __init__(self) -> None:
        self._RGC_requirements = [0]
        self._RGC_index = None

    def set_RGC_index(self, index):
        self._RGC_index = index

    def initialize(self, assembly):
        self._assembly = assembly

    def set_required_DoFs(self, RGC_remain_index):
        return RGC_remain_index

    def modify_RGC(self, RGC):
        return RGC


def _levi_civita(device):
    e = torch.zeros(3, 3, 3, dtype=torch.float64, device=device)
    e[0, 1, 2] = e[1, 2, 0] = e[2, 0, 1] = 1.0
    e[0, 2, 1] = e[2, 1, 0] = e[1, 0, 2] = -1.0
    return e


def rigid_motion(z, y, order=2):
    """Displacement Y = R(z) y - y of offsets y [n, 3] and its derivatives
    with respect to the rotation vector z: (Y, dY/dz [n,3,3], d2Y/dz2
    [n,3,3,3]) (couple.py:169-282).  Written in the angle t = |z| + 1e-20
    and the axis w = z / t: with c = cos t, s = sin t,
      R(z) y = c y + s (w x y) + (1 - c) w (w . y),
    its partial derivatives in t and w, and dt/dz = w,
    dw/dz = I / t - z z^T / t^3 (the reference's forms, which take |z| = t)."""
    z = z.to(torch.float64)
    y = y.to(torch.float64)
    dev = y.device
    t = torch.linalg.vector_norm(z) + 1e-20
    w = z / t
    c, s = torch.cos(t), torch.sin(t)
    eps = _levi_civita(dev)
    wy = y @ w
    wxy = torch.einsum("ijk,j,nk->ni", eps, w, y)
    Y = c * y + s * wxy + (1 - c) * w[None, :] * wy[:, None] - y
    if order == 0:
        return Y, None, None
    eye = torch.eye(3, dtype=torch.float64, device=dev)
    d_t = -s * y + c * wxy + s * w[None, :] * wy[:, None]
    cross = torch.einsum("ilk,nk->nil", eps, y)                          # d (w x y)_i / d w_l
    outer = eye[None] * wy[:, None, None] + w[None, :, None] * y[:, None, :]   # d (w (w . y))_i / d w_l
    d_w = s * cross + (1 - c) * outer
    w_z = eye / t - torch.outer(z, z) / t ** 3
    dY = torch.einsum("nil,lp->nip", d_w, w_z) + d_t[:, :, None] * w[None, None, :]
    if order == 1:
        return Y, dY, None
    d_tt = -c * y - s * wxy + c * w[None, :] * wy[:, None]
    d_wt = c * cross + s * outer
    d_ww = (1 - c) * (eye[None, :, :, None] * y[:, None, None, :] + eye[None, :, None, :] * y[:, None, :, None])
    w_zz = 3 * torch.einsum("i,p,q->ipq", z, z, z) / t ** 5 - (
        eye[:, :, None] * z[None, None, :] + eye[:, None, :] * z[None, :, None]
        + eye[None, :, :] * z[:, None, None]) / t ** 3
    dw_t = torch.einsum("nil,lp->nip", d_wt, w_z)
    d2Y = (d_t[:, :, None, None] * w_z[None] + d_tt[:, :, None, None] * (w[:, None] * w[None, :])[None]
           + dw_t[:, :, None, :] * w[None, None, :, None]
           + dw_t[:, :, :, None] * w[None, None, None, :]
           + torch.einsum("nilm,lp,mq->nipq", d_ww, w_z, w_z) + torch.einsum("nil,lpq->nipq", d_w, w_zz))
    return Y, dY, d2Y


class Couple(BaseConstraint):
    """Nodes of ``set_nodes_name`` of an instance follow reference point
    ``rp_name`` rigidly (couple.py:7-282)."""

    def __init__(self, instance_name: str, set_nodes_name: str, rp_name: str) -> None:
        super().__init__()
        self.instance_name = instance_name
        self.set_nodes_name = set_nodes_name
        self.rp_name = rp_name

    def initialize(self, assembly):
        super().initialize(assembly)
        inst = assembly.get_instance(self.instance_name)
        self._indexNodes = np.asarray(inst.set_nodes[self.set_nodes_name], dtype=np.int64)
        rp = assembly.get_reference_point(self.rp_name)
        self._rp_index = rp._RGC_index
        self._couple_index = inst._RGC_index
        self._ref_location = (inst.nodes[torch.from_numpy(self._indexNodes)] - rp.node.view(1, 3)).to(torch.float64)

    def set_required_DoFs(self, RGC_remain_index):
        RGC_remain_index[self._couple_index][self._indexNodes] = False
        RGC_remain_index[self._rp_index][:] = True
        return RGC_remain_index

    def modify_RGC(self, RGC):
        """Tied nodes at v + R(z) y - y (couple.py:34-40)."""
        rp = RGC[self._rp_index]
        y = self._ref_location.to(rp.device)
        Y = rigid_motion(rp[3:], y, order=0)[0]
        RGC[self._couple_index][torch.from_numpy(self._indexNodes).to(rp.device)] = rp[:3][None, :] + Y
        return RGC
