"""Loads on the B200 path: the follower pressure (FEA/assemble/loads/pressure.py)
and the concentrated force and moment on a reference point
(concentrate_force.py, moment.py)."""
from __future__ import annotations

import torch


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


class _PointLoad(BaseLoad):
    """A constant generalized force on three DOFs of a reference point."""

    _offset = 0

    def __init__(self, rp_name: str, value) -> None:
        super().__init__()
        self.rp_name = rp_name
        self._value = torch.as_tensor(value, dtype=torch.float64).reshape(3)

    def initialize(self, assembly):
        super().initialize(assembly)
        self.rp_index = assembly.get_reference_point(self.rp_name)._RGC_index

    def set_required_DoFs(self, RGC_remain_index):
        RGC_remain_index[self.rp_index][self._offset:self._offset + 3] = True
        return RGC_remain_index


class Concentrate_Force(_PointLoad):
    """Force on a reference point's translation DOFs (concentrate_force.py:5-55):
    it adds -force to their residual and -force . v to the total potential."""

    def __init__(self, rp_name: str, force) -> None:
        super().__init__(rp_name, force)

    @property
    def force(self):
        return self._value

    @force.setter
    def force(self, value):
        self._value = torch.as_tensor(value, dtype=torch.float64).reshape(3)


class Moment(_PointLoad):
    """Moment on a reference point's rotation DOFs (moment.py:5-55): it adds
    -moment to their residual and -moment . z to the total potential."""

    _offset = 3

    def __init__(self, rp_name: str, moment) -> None:
        super().__init__(rp_name, moment)

    @property
    def moment(self):
        return self._value

    @moment.setter
    def moment(self, value):
        self._value = torch.as_tensor(value, dtype=torch.float64).reshape(3)
