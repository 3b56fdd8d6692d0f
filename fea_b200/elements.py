"""C3D4 / C3D8 solid elements on the B200 kernels.

Mirrors the element API of sssnnn7119/FEA (FEA/assemble/elements/base.py,
C3/C3base.py, C3/tetrahedral.py, C3/brick.py): the class-name registry used
by the element factory (base.py:11-15, elements/__init__.py:12-35),
``initialize``, ``structural_Force``, ``potential_Energy``,
``extract_surface``.  Element math runs in the library's gather kernels; a
per-group plan over all DOFs of the group's nodes reproduces the unreduced
element-level outputs of the reference (``_indices_force``,
``_indices_matrix`` and their values, C3base.py:109-153 and 413-452).
"""
from __future__ import annotations

import numpy as np
import torch

from . import materials as _materials

FACES = {
    # face id -> local nodes, outward ordering (tetrahedral.py:45-64, brick.py:166-201)
    "C3D4": {0: [0, 2, 1], 1: [0, 1, 3], 2: [1, 2, 3], 3: [0, 3, 2]},
    "C3D8": {0: [0, 3, 2, 1], 1: [4, 5, 6, 7], 2: [0, 1, 5, 4], 3: [1, 2, 6, 5], 4: [2, 3, 7, 6], 5: [0, 4, 7, 3]},
}


class Surface:
    """A group of T3 or Q4 faces (node lists in outward order)."""

    def __init__(self, elems: torch.Tensor):
        self._elems = elems.to(torch.int64)
        self.num_nodes_per_elem = int(elems.shape[1])
        self.kind = {3: "T3", 4: "Q4"}.get(self.num_nodes_per_elem)
        if self.kind is None:
            raise NotImplementedError("surface with %d nodes is outside the B200 path" % self.num_nodes_per_elem)


def merge_surfaces(surfaces):
    """Concatenate faces of the same kind (surfaces/__init__.py merge_surfaces)."""
    by = {}
    for s in surfaces:
        by.setdefault(s.kind, []).append(s._elems)
    return [Surface(torch.cat(v, 0)) for k, v in sorted(by.items()) if sum(x.shape[0] for x in v) > 0]


class BaseElement:
    _subclasses: dict = {}

    def __init_subclass__(cls, **kw):
        super().__init_subclass__(**kw)
        BaseElement._subclasses[cls.__name__] = cls

    def __init__(self, elems_index=None, elems=None, part=None) -> None:
        self._elems_index = torch.as_tensor(elems_index).to(torch.int64).cpu()
        self._elems = torch.as_tensor(elems).to(torch.int64).cpu()
        self.part = part
        self.materials = None
        self.density = torch.tensor(1.0, dtype=torch.float64)

    def set_materials(self, materials):
        self.materials = materials

    def set_density(self, density):
        self.density = torch.as_tensor(density, dtype=torch.float64).reshape(-1)[:1].reshape(())

    def initialize(self, *args, **kwargs):
        pass

    def extract_surface(self, surface_ind, elems_ind):
        return []


def initialize_element(element_type, elems_index, elems, part, *args, **kwargs):
    """Factory by class name (elements/__init__.py:12-35)."""
    cls = BaseElement._subclasses.get(element_type)
    if cls is None:
        raise ValueError("Element type '%s' is not recognized." % element_type)
    return cls(elems_index=elems_index, elems=elems, part=part)


class Element_3D(BaseElement):
    kind: str = ""
    num_nodes_per_elem: int = 0
    _num_gaussian: int = 0

    def __init__(self, elems=None, elems_index=None, part=None) -> None:
        super().__init__(elems_index=elems_index, elems=elems, part=part)
        self._plan = None
        self._frame = None

    def initialize(self, *args, **kwargs):
        if self._elems.shape[1] != self.num_nodes_per_elem:
            raise ValueError("%s needs %d nodes per element" % (self.kind, self.num_nodes_per_elem))
        # force index 3 n_a + j in (a, j, e) order (C3base.py:147-153)
        el = self._elems.T
        self._indices_force_cpu = (3 * el[:, None, :] + torch.arange(3)[None, :, None]).reshape(-1)
        self._plan = None
        self._frame = None

    # -- per-group plan (all DOFs of the group's nodes active) ---------------
    def _group_plan(self):
        if self._plan is None:
            from .plan import DevicePlan
            N = self.part.nodes.shape[0]
            mask = np.zeros(N, np.uint8)
            mask[np.unique(self._elems.numpy())] = 7
            self._plan = DevicePlan(self.part.nodes, mask, [(self.kind, self._elems.numpy())])
            self._frame = None
            free = torch.from_numpy(np.repeat(mask != 0, 3))
            self._free = free.to(self._plan.device)
            self._dof_map = torch.nonzero(free).flatten().to(self._plan.device)
            self._indices_force = self._indices_force_cpu.to(self._plan.device)
            self._indices_matrix = self._dof_map[self._plan.coo_indices()]
        return self._plan

    def _gc(self, U):
        P = self._group_plan()
        U = torch.as_tensor(U, dtype=torch.float64).to(P.device)
        return U.reshape(-1)[self._free].contiguous()

    @staticmethod
    def _frame_key(rotation_matrix):
        """None for the part's own frame (no rotation or the identity), else
        the rotation as a float64 CPU tensor."""
        if rotation_matrix is None:
            return None
        R = torch.as_tensor(rotation_matrix, dtype=torch.float64).detach().cpu()
        if tuple(R.shape) != (3, 3):
            raise ValueError("rotation_matrix must be 3 x 3")
        return None if torch.equal(R, torch.eye(3, dtype=torch.float64)) else R

    def _framed_plan(self, rotation_matrix=None):
        """The group plan with its coordinates in the frame of
        ``rotation_matrix``: the part's nodes X rotated to R X.  An isotropic
        element evaluated on R X with the instance's (global) displacement
        gives R R_e and R K_e R^T of the part frame, which is what the
        reference computes by rotating U in and R_e, K_e out
        (C3base.py:417-418, 441-443)."""
        P = self._group_plan()
        key = self._frame_key(rotation_matrix)
        cur = self._frame
        if (cur is None) != (key is None) or (key is not None and not torch.equal(cur, key)):
            X = self.part.nodes.to(torch.float64).cpu()
            if key is not None:
                X = X @ key.T
            P.X.copy_(X.to(P.device))
            self._frame = key
        return P

    def structural_Force(self, RGC, rotation_matrix=None, if_onlyforce: bool = False, *args, **kwargs):
        """Element residual (and tangent) of the group (C3base.py:413-452).

        Returns (indices_force, R_e[(a,j,e)]) or, with the tangent,
        (indices_force, R_e, indices_matrix [2,nnz_e], values [nnz_e]) where
        indices_matrix is the sorted unique DOF-pair COO of the group.  With
        a rotation matrix R (the instance's), RGC is the displacement in the
        instance frame and the outputs are R R_e and R K_e R^T.
        """
        P = self._framed_plan(rotation_matrix)
        mu, kappa = self.materials.parameters()
        gc = self._gc(RGC)
        elemR = P.zeros(self.num_nodes_per_elem * 3 * self._elems.shape[0])
        if if_onlyforce:
            P.assemble_volume(0, mu, kappa, gc, R=P.zeros(P.ndof), elemR=elemR)
            return self._indices_force, elemR
        K = torch.empty(P.nnz, dtype=torch.float64, device=P.device)
        P.assemble_volume(0, mu, kappa, gc, K=K, elemR=elemR)
        return self._indices_force, elemR, self._indices_matrix, K

    def potential_Energy(self, RGC):
        """sum_{g,e} W(F) w  (C3base.py:387-411) as a 0-d device tensor;
        RGC is the displacement in the part's own frame."""
        P = self._framed_plan(None)
        mu, kappa = self.materials.parameters()
        out = P.zeros(1)
        P.energy_volume(0, mu, kappa, self._gc(RGC), out)
        return out[0]

    def get_mass_matrix(self, rotation_matrix=None):
        """(indices_matrix [2, nnz_e], values [nnz_e]): the consistent mass
        rho N_a N_b w times the 3 x 3 identity of every element on the
        group's pattern (C3base.py:348-384).  R M R^T = M for this isotropic
        mass, so a rotation leaves the values unchanged."""
        self._frame_key(rotation_matrix)
        P = self._framed_plan(None)
        return self._indices_matrix, P.mass_csr([float(self.density)])

    def get_volumn(self, U=None):
        raise NotImplementedError("element volume queries are outside the B200 path")

    def extract_surface(self, surface_ind: int, elems_ind):
        """Faces `surface_ind` of the elements whose labels are in elems_ind."""
        pos = np.nonzero(np.isin(self._elems_index.numpy(), np.asarray(elems_ind)))[0]
        loc = FACES[self.kind].get(int(surface_ind))
        if loc is None:
            raise ValueError("Invalid surface index: %s" % surface_ind)
        f = self._elems[torch.from_numpy(pos)][:, loc] if pos.size else torch.empty((0, len(loc)), dtype=torch.int64)
        return [Surface(f)]

    def set_required_DoFs(self, RGC_remain_index):
        RGC_remain_index[np.unique(self._elems.numpy())] = True
        return RGC_remain_index


class C3D4(Element_3D):
    """4-node linear tetrahedron, 1 Gauss point (tetrahedral.py:6-64)."""
    kind = "C3D4"
    num_nodes_per_elem = 4
    _num_gaussian = 1
    num_surfaces = 4


class C3D8(Element_3D):
    """8-node trilinear brick, 2x2x2 Gauss points (brick.py:6-201)."""
    kind = "C3D8"
    num_nodes_per_elem = 8
    _num_gaussian = 8
    num_surfaces = 6


materials = _materials
