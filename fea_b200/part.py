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

    # -- element pass-through (part.py:250-289, 317-330) --------------------------
    def potential_energy(self, RGC):
        """Sum of the element groups' potential energies; RGC [N, 3] in the
        part's frame."""
        return self._sum(e.potential_Energy(RGC) for e in self.elems.values())

    @staticmethod
    def _sum(vals):
        total = None
        for v in vals:
            total = v if total is None else total + v
        return total if total is not None else torch.zeros((), dtype=torch.float64)

    def structural_stiffness(self, RGC, rotation_matrix=None):
        """(R_indices, R_values, K_indices, K_values): the element groups'
        structural_Force outputs concatenated (duplicate COO, part DOFs)."""
        out = [e.structural_Force(RGC=RGC, rotation_matrix=rotation_matrix) for e in self.elems.values()]
        return (torch.cat([o[0] for o in out]), torch.cat([o[1] for o in out]),
                torch.cat([o[2] for o in out], dim=1), torch.cat([o[3] for o in out]))

    def structural_force(self, RGC, rotation_matrix=None):
        """(R_indices, R_values) of every element group, concatenated."""
        out = [e.structural_Force(RGC=RGC, rotation_matrix=rotation_matrix, if_onlyforce=True)
               for e in self.elems.values()]
        return torch.cat([o[0] for o in out]), torch.cat([o[1] for o in out])

    def get_mass_matrix(self, rotation_matrix=None):
        """(M_indices, M_values): every group's consistent mass, concatenated."""
        out = [e.get_mass_matrix(rotation_matrix=rotation_matrix) for e in self.elems.values()]
        return torch.cat([o[0] for o in out], dim=1), torch.cat([o[1] for o in out])

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
        return self._transform(self.part.nodes, self._rotation) + self._translation.view(1, 3)

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

    @staticmethod
    def _transform(vector0, rotation_vector=None):
        """Rodrigues rotation of rows of vector0 [n, 3] by a rotation vector."""
        v = torch.as_tensor(vector0, dtype=torch.float64).reshape(-1, 3)
        if rotation_vector is None:
            return v
        rv = torch.as_tensor(rotation_vector, dtype=torch.float64).to(v.device)
        theta = torch.norm(rv)
        if theta == 0:
            return v
        r = (rv / theta).view(1, 3)
        return v * torch.cos(theta) + torch.cross(r.expand_as(v), v, dim=1) * torch.sin(theta) + \
            r * (r * v).sum(1, keepdim=True) * (1 - torch.cos(theta))

    # -- element pass-through in the instance frame (part.py:409-431) -------------
    def structural_stiffness(self, RGC, if_onlyforce: bool = False, *args, **kwargs):
        """The part's element outputs for this instance's displacement block
        RGC[self._RGC_index] (instance frame), shifted by the instance's
        first DOF."""
        U = RGC[self._RGC_index]
        if if_onlyforce:
            ri, rv = self.part.structural_force(U, self.rotation_matrix)
            return ri + self._index_start, rv
        ri, rv, ki, kv = self.part.structural_stiffness(U, self.rotation_matrix)
        return ri + self._index_start, rv, ki + self._index_start, kv

    def potential_energy(self, RGC):
        """The part's energy at the displacement rotated back into the part
        frame."""
        return self.part.potential_energy(self._transform(RGC[self._RGC_index], -self._rotation))

    def get_mass_matrix(self):
        mi, mv = self.part.get_mass_matrix(self.rotation_matrix)
        return mi + self._index_start, mv
