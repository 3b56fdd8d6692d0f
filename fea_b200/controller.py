"""FEAController (mirrors FEA/controller.py of sssnnn7119/FEA)."""
from __future__ import annotations


class FEAController:
    def __init__(self, maximum_iteration: int = 10000) -> None:
        self.assembly = None
        self.solver = None

    def initialize(self, *args, **kwargs):
        self.assembly.initialize(*args, **kwargs)
        self.solver.initialize(assembly=self.assembly, *args, **kwargs)

    def solve(self, GC0=None, if_initialize: bool = True, *args, **kwargs):
        if if_initialize:
            self.initialize()
        return self.solver.solve(GC0=GC0, *args, **kwargs)
