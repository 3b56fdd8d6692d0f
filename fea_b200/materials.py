"""Materials of the element path.

Mirrors FEA/assemble/elements/materials (sssnnn7119/FEA): NeoHookean with
W = mu/2 (J^-2/3 tr(F^T F) - 3) + kappa/2 (J-1)^2 (hyperelastic.py:6-84) and
the type-id factory initialize_materials (materials/__init__.py:8-21).  The
constitutive update itself runs inside the element kernels.
"""
from __future__ import annotations

import torch


class Materials_Base:
    type: int = 0

    def parameters(self):
        raise NotImplementedError


def _scalar(v):
    if isinstance(v, torch.Tensor):
        if v.numel() != 1:
            raise ValueError("fea_b200 supports one material value per element group (got %d values)" % v.numel())
        return v
    return torch.tensor(float(v), dtype=torch.float64)


class NeoHookean(Materials_Base):
    """Compressible Neo-Hookean material (type id 1).

    ``mu`` and ``kappa`` may be Python floats or one-element tensors.  The
    reference turns Python floats into float32 tensors of shape [1]
    (hyperelastic.py:15-20); here they are kept as float64 scalars.
    """

    def __init__(self, mu, kappa) -> None:
        self.type = 1
        self.mu = _scalar(mu)
        self.kappa = _scalar(kappa)

    def parameters(self):
        return float(self.mu), float(self.kappa)

    def strain_energy_density_C3(self, F: torch.Tensor):
        """W(F) per Gauss point (hyperelastic.py:25-33), for host-side checks."""
        J = torch.linalg.det(F)
        I1 = (F ** 2).sum((-1, -2)) * J ** (-2.0 / 3.0)
        return self.mu / 2 * (I1 - 3) + self.kappa / 2 * (J - 1) ** 2


def initialize_materials(materials_type: int, materials_params: torch.Tensor):
    """Factory by type id (materials/__init__.py:8-21); only Neo-Hookean runs on the B200 path."""
    if materials_type == 1:
        return NeoHookean(materials_params[0, 0], materials_params[0, 1])
    raise NotImplementedError("material type %r is outside the B200 element path" % (materials_type,))
