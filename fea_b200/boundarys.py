"""Dirichlet conditions (FEA/assemble/boundarys/boundary_condition.py)."""
from __future__ import annotations


class BaseBoundary:
    def __init__(self) -> None:
        self._RGC_requirements = [0]
        self._RGC_index = None

    def set_RGC_index(self, index):
        self._RGC_index = index

    def initialize(self, assembly):
        self._assembly = assembly


class Boundary_Condition(BaseBoundary):
    """Fix DOFs `indexDoF` of the nodes of a node set to zero (boundary_condition.py:5-41)."""

    def __init__(self, instance_name: str, set_nodes_name: str, indexDoF=(0, 1, 2)) -> None:
        super().__init__()
        self.instance_name = instance_name
        self.set_nodes_name = set_nodes_name
        self.indexDoF = list(indexDoF)

    def initialize(self, assembly):
        super().initialize(assembly)
        inst = assembly.get_instance(self.instance_name)
        self.index_nodes = inst.set_nodes[self.set_nodes_name]
        self._constraint_index = inst._RGC_index


class Boundary_Condition_RP(BaseBoundary):
    """Fix DOFs `indexDoF` (0-2 translation, 3-5 rotation) of a reference
    point to zero (boundary_condition_rp.py:5-32)."""

    def __init__(self, rp_name: str, indexDoF=(0, 1, 2, 3, 4, 5)) -> None:
        super().__init__()
        self.rp_name = rp_name
        self.indexDoF = list(indexDoF)

    def initialize(self, assembly):
        super().initialize(assembly)
        self._constraint_index = assembly.get_reference_point(self.rp_name)._RGC_index
