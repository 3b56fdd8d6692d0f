"""Loads on the B200 path: the follower pressure (FEA/assemble/loads/pressure.py)."""
from __future__ import annotations


class BaseLoad:
    def __init__(self) -> None:
        self._RGC_requirements = [0]
        self._RGC_index = None
        self._assembly = None

    def set_RGC_index(self, index):
        self._RGC_index = index

    def initialize(self, assembly):
        self._assembly = assembly


class Pressure(BaseLoad):
    """Follower pressure p on a surface set, derived from the enclosed-volume
    potential -p V with V = 1/3 sum_faces int x . n dA (pressure.py:5-169).

    Its force and stiffness are evaluated by the library's face kernels and
    added into the assembled R and K; ``pressure`` may be changed between
    solves (load increments).
    """

    def __init__(self, instance_name: str, surface_set: str, pressure: float) -> None:
        super().__init__()
        self.instance_name = instance_name
        self.surface_name = surface_set
        self.pressure = pressure
        self.surface_element = []

    def initialize(self, assembly):
        super().initialize(assembly)
        inst = assembly.get_instance(self.instance_name)
        self.surface_element = inst.extract_surfaces(self.surface_name)
        self._load_index = inst._RGC_index
