"""Part and Instance (mirrors FEA/assemble/part.py of sssnnn7119/FEA)."""
from __future__ import annotations

import torch

from .elements import merge_surfaces


class _Surfaces:
    """Named surface sets: name -> list of (element labels, face id) (part.py:14-93)."""

    def __init__(self):
        self._surface_dict = {}

    def __getitem__(self, key):
        return self._surface_dict[key]

    def __setitem__(self, key, value):
        self._surface_dict[key] = value

    def __delitem__(self, key):
        del self._surface_dict[key]

    def __contains__(self, key):
        return key in self._surface_dict

    def keys(self):
        return list(self._surface_dict.keys())


class Part:
    def __init__(self, nodes) -> None:
        self.nodes = torch.as_tensor(nodes, dtype=torch.float64)
        self.elems = {}
        self.set_nodes = {}
        self.surfaces = _Surfaces()

    def initialize(self, *args, **kwargs):
        for e in self.elems.values():
            e.initialize()

    def add_element(self, element, name: str = None):
        if name is None:
            number = len(self.elems)
            while ("element-%d" % number) in self.elems:
                number += 1
            name = "element-%d" % number
        self.elems[name] = element
        return name

    def delete_element(self, name: str):
        if name not in self.elems:
            raise ValueError("Element '%s' not found in the model." % name)
        del self.elems[name]

    def add_surface_set(self, name: str, elements):
        self.surfaces[name] = elements
        return name

    def delete_surface_set(self, name: str):
        if name not in self.surfaces:
            raise KeyError("Surface set '%s' not found in the model." % name)
        del self.surfaces[name]

    def extract_surfaces(self, name: str):
        """Faces of a surface set, merged by kind (part.py:291-313)."""
        out = []
        for elem_ind, surf_ind in self.surfaces[name]:
            for e in self.elems.values():
                out += e.extract_surface(surf_ind, elem_ind)
        if not out:
            raise ValueError("Surface %s not found in the model." % name)
        return merge_surfaces(out)


class Instance:
    """A part placed in the assembly (part.py:334-431)."""

    def __init__(self, part: Part) -> None:
        self.part = part
        self._RGC_requirements = tuple(part.nodes.shape)
        self._translation = torch.zeros(3, dtype=torch.float64)
        self._rotation = torch.zeros(3, dtype=torch.float64)
        self._RGC_index = None
        self._index_start = None

    @property
    def rotation_matrix(self):
        theta = torch.norm(self._rotation)
        if theta == 0:
            return torch.eye(3, dtype=torch.float64)
        r = (self._rotation / theta).view(3, 1)
        K = torch.tensor([[0, -r[2, 0], r[1, 0]], [r[2, 0], 0, -r[0, 0]], [-r[1, 0], r[0, 0], 0]], dtype=torch.float64)
        return torch.cos(theta) * torch.eye(3, dtype=torch.float64) + (1 - torch.cos(theta)) * (r @ r.t()) + torch.sin(theta) * K

    @property
    def elems(self):
        return self.part.elems

    @property
    def nodes(self):
        """Instance coordinates: rotated part nodes plus the translation (part.py:364-398)."""
        v = self.part.nodes.view(-1, 3)
        theta = torch.norm(self._rotation)
        if theta != 0:
            r = (self._rotation / theta).view(1, 3)
            v = v * torch.cos(theta) + torch.cross(r.expand_as(v), v, dim=1) * torch.sin(theta) + \
                r * (r * v).sum(1, keepdim=True) * (1 - torch.cos(theta))
        return v + self._translation.view(1, 3)

    @property
    def surfaces(self):
        return self.part.surfaces

    @property
    def set_nodes(self):
        return self.part.set_nodes

    def set_RGC_index(self, index):
        self._RGC_index = index

    def initialize(self, assembly):
        self._assembly = assembly
        self._index_start = assembly.RGC_list_indexStart[self._RGC_index]

    def extract_surfaces(self, name):
        return self.part.extract_surfaces(name)
