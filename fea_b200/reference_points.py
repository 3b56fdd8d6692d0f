"""Reference points (mirrors FEA/assemble/reference_points.py of sssnnn7119/FEA)."""
from __future__ import annotations

import torch


class ReferencePoint:
    """A point with six generalized coordinates (UX, UY, UZ, RX, RY, RZ):
    a translation v and a rotation vector z (reference_points.py:5-23)."""

    def __init__(self, node=None) -> None:
        self.node = torch.as_tensor(node, dtype=torch.float64).reshape(3).clone()
        self._RGC_requirements = 6
        self._RGC_index = None
        self._index_start = None

    def set_RGC_index(self, index):
        self._RGC_index = index

    def initialize(self, assembly):
        self._assembly = assembly
        self._index_start = assembly.RGC_list_indexStart[self._RGC_index]
