"""Assembly on the B200 kernels (mirrors FEA/assemble/assembly.py of sssnnn7119/FEA).

``Assembly.initialize`` reproduces the reference's DOF bookkeeping —
redundant generalized coordinates (RGC) per object in name order, the 1e-5
seed on the last node of the last instance (assembly.py:113), required DOFs
from elements and pressure faces, Dirichlet DOFs removed last
(assembly.py:76-185) — and then builds ONE device plan for the whole reduced
system.  Every later call (``assemble_Stiffness_Matrix``, ``assemble_force``,
``_total_Potential_Energy``) only launches kernels: the reference's
per-iteration host copy of the K indices and the two ``unique`` relabels
(assembly.py:373-380) have no counterpart here.

K is returned coalesced, in CSR order (the reference returns the same matrix
as an uncoalesced COO with duplicate entries).
"""
from __future__ import annotations

import numpy as np
import torch

from ._trace import nvtx
from .boundarys import Boundary_Condition
from .loads import Pressure
from .part import Instance, Part
from .plan import DevicePlan


class Assembly:
    def __init__(self, device=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self._parts = {}
        self._instances = {}
        self._reference_points = {}
        self._loads = {}
        self._constraints = {}
        self._boundarys = {}
        self.RGC = []
        self.RGC_remain_index = []
        self.RGC_list_indexStart = [0]
        self._RGC_size = []
        self.GC = None
        self._plan = None

    # -- model building (assembly.py:511-766) --------------------------------
    @staticmethod
    def _name(d, obj, prefix):
        number = len(d)
        while ("%s-%d" % (prefix, number)) in d:
            number += 1
        return "%s-%d" % (prefix, number)

    def add_part(self, part: Part, name: str = None):
        name = name or self._name(self._parts, part, "Part")
        if name in self._parts:
            raise ValueError("Part with name %s already exists in the assembly." % name)
        self._parts[name] = part

    def get_part(self, name):
        if name not in self._parts:
            raise ValueError("Part with name %s does not exist in the assembly." % name)
        return self._parts[name]

    def delete_part(self, name):
        self.get_part(name)
        del self._parts[name]

    def add_instance(self, instance: Instance, name: str = None):
        name = name or self._name(self._instances, instance, "Instance")
        if name in self._instances:
            raise ValueError("Instance with name %s already exists in the assembly." % name)
        self._instances[name] = instance

    def get_instance(self, name):
        if name not in self._instances:
            raise ValueError("Instance with name %s does not exist in the assembly." % name)
        return self._instances[name]

    def delete_instance(self, name):
        self.get_instance(name)
        del self._instances[name]

    def add_load(self, load, name: str = None):
        name = name or self._name(self._loads, load, load.__class__.__name__)
        self._loads[name] = load
        return name

    def add_loads(self, loads_dict):
        for name, load in loads_dict.items():
            self.add_load(load, name)

    def get_load(self, name):
        if name not in self._loads:
            raise ValueError("Load '%s' not found in the model." % name)
        return self._loads[name]

    def delete_load(self, name):
        self.get_load(name)
        del self._loads[name]

    def delete_all_loads(self):
        self._loads.clear()

    def add_boundary(self, boundary, name: str = None):
        name = name or self._name(self._boundarys, boundary, boundary.__class__.__name__)
        self._boundarys[name] = boundary
        return name

    def get_boundary(self, name):
        if name not in self._boundarys:
            raise ValueError("Boundary '%s' not found in the model." % name)
        return self._boundarys[name]

    def delete_boundary(self, name):
        self.get_boundary(name)
        del self._boundarys[name]

    def add_reference_point(self, rp, name: str = None):
        raise NotImplementedError("reference points (and their couplings) are outside the B200 element path")

    def add_constraint(self, constraint, name: str = None):
        raise NotImplementedError("constraints are outside the B200 element path")

    # -- initialization (assembly.py:76-185) -----------------------------------
    def _allocate_RGC(self, size):
        idx = len(self.RGC)
        self.RGC.append(torch.zeros(size, dtype=torch.float64, device=self.device))
        self.RGC_remain_index.append(np.zeros(size, dtype=bool))
        self._RGC_size.append(tuple(size))
        self.RGC_list_indexStart.append(self.RGC_list_indexStart[-1] + int(np.prod(size)))
        return idx

    def initialize(self, *args, **kwargs):
        self._parts = dict(sorted(self._parts.items()))
        self._instances = dict(sorted(self._instances.items()))
        self._loads = dict(sorted(self._loads.items()))
        self._boundarys = dict(sorted(self._boundarys.items()))
        for name, ld in self._loads.items():
            if not isinstance(ld, Pressure):
                raise NotImplementedError("load %r (%s) is outside the B200 path" % (name, type(ld).__name__))
        for name, b in self._boundarys.items():
            if not isinstance(b, Boundary_Condition):
                raise NotImplementedError("boundary %r (%s) is outside the B200 path" % (name, type(b).__name__))
        if not self._instances:
            raise ValueError("the assembly has no instance")
        self.RGC, self.RGC_remain_index, self.RGC_list_indexStart, self._RGC_size = [], [], [0], []
        idx = None
        for ins in self._instances.values():
            idx = self._allocate_RGC(ins._RGC_requirements)
            ins.set_RGC_index(idx)
        self.RGC[idx][-1] = 1e-5                  # the reference's seed (assembly.py:113)
        for ld in self._loads.values():
            ld.set_RGC_index(self._allocate_RGC(ld._RGC_requirements))
        for b in self._boundarys.values():
            b.set_RGC_index(self._allocate_RGC(b._RGC_requirements))
        for part in self._parts.values():
            part.initialize(self)
        for ins in self._instances.values():
            ins.initialize(self)
        for ld in self._loads.values():
            ld.initialize(self)
        for b in self._boundarys.values():
            b.initialize(self)
        # required DOFs: element nodes, pressure face nodes; Dirichlet last
        for ins in self._instances.values():
            rem = self.RGC_remain_index[ins._RGC_index]
            for e in ins.part.elems.values():
                rem = e.set_required_DoFs(rem)
        for ld in self._loads.values():
            rem = self.RGC_remain_index[ld._load_index]
            for s in ld.surface_element:
                rem[np.unique(s._elems.numpy())] = True
        for b in self._boundarys.values():
            rem = self.RGC_remain_index[b._constraint_index]
            for d in b.indexDoF:
                rem[np.asarray(b.index_nodes, dtype=np.int64), d] = False
                self.RGC[b._constraint_index][torch.as_tensor(np.asarray(b.index_nodes, dtype=np.int64)), d] = 0.0
        self.RGC_remain_index_flatten = torch.from_numpy(
            np.concatenate([r.reshape(-1) for r in self.RGC_remain_index]))
        self._remain_dev = self.RGC_remain_index_flatten.to(self.device)
        self.GC = self._RGC2GC(self.RGC)
        self._GC_list_indexStart = np.cumsum([0] + [int(r.sum()) for r in self.RGC_remain_index]).tolist()
        self._build_plan()

    def _build_plan(self):
        X, Xi, masks, groups, mats, faces, self._face_loads = [], [], [], [], [], [], []
        self._node_offset = {}
        off = 0
        for name, ins in self._instances.items():
            self._node_offset[name] = off
            R = ins.rotation_matrix
            if not torch.equal(R, torch.eye(3, dtype=torch.float64)):
                raise NotImplementedError("rotated instances are outside the B200 element path")
            X.append(ins.part.nodes.to(torch.float64).cpu())
            Xi.append(ins.nodes.to(torch.float64).cpu())
            rem = self.RGC_remain_index[ins._RGC_index]
            masks.append((rem[:, 0] * 1 + rem[:, 1] * 2 + rem[:, 2] * 4).astype(np.uint8))
            for e in ins.part.elems.values():
                if e.materials is None:
                    raise ValueError("element group without materials")
                groups.append((e.kind, e._elems.numpy() + off))
                mats.append(e)
            off += ins.part.nodes.shape[0]
        for ld in self._loads.values():
            o = self._node_offset[ld.instance_name]
            for s in ld.surface_element:
                faces.append((s.kind, s._elems.numpy() + o))
                self._face_loads.append(ld)
        self._mat_elems = mats
        self._plan = DevicePlan(torch.cat(X), np.concatenate(masks), groups, faces, device=self.device)
        self._Xinst = torch.cat(Xi).to(self.device).contiguous()
        self._energy_buf = torch.zeros(1, dtype=torch.float64, device=self.device)

    @property
    def plan(self) -> DevicePlan:
        if self._plan is None:
            raise RuntimeError("Assembly.initialize() has not been called")
        return self._plan

    # -- GC <-> RGC (assembly.py:470-499) ---------------------------------------
    def _GC2RGC(self, GC):
        full = torch.zeros(self.RGC_list_indexStart[-1], dtype=torch.float64, device=self.device)
        full[self._remain_dev] = GC.to(self.device, torch.float64)
        return [full[self.RGC_list_indexStart[i]:self.RGC_list_indexStart[i + 1]].view(self._RGC_size[i])
                for i in range(len(self._RGC_size))]

    def _RGC2GC(self, RGC):
        return torch.cat([RGC[i].reshape(-1)[torch.from_numpy(self.RGC_remain_index[i].reshape(-1)).to(RGC[i].device)]
                          for i in range(len(RGC))])

    def _gc(self, RGC=None, GC=None):
        if GC is None:
            if RGC is None:
                raise ValueError("Either RGC or GC must be provided.")
            GC = self._RGC2GC(RGC)
        return torch.as_tensor(GC, dtype=torch.float64).to(self.device).contiguous()

    # -- assembly ------------------------------------------------------------------
    def assemble_csr(self, GC, want_K=True, K=None, R=None):
        """Reduced residual R [n] and K values [nnz] in the plan's CSR order."""
        with nvtx("fea.assemble_csr" if want_K else "fea.assemble_force"):
            return self._assemble_csr(GC, want_K, K, R)

    def _assemble_csr(self, GC, want_K, K, R):
        P = self.plan
        gc = self._gc(GC=GC)
        R = P.zeros(P.ndof) if R is None else R
        if want_K and K is None:
            K = torch.empty(P.nnz, dtype=torch.float64, device=P.device)
        # the first group stores whole rows when it touches every active node;
        # otherwise all groups accumulate into zeroed buffers
        store_first = len(P.groups) > 0 and P.groups[0].covers_active
        if not store_first:
            R.zero_()
            if want_K:
                K.zero_()
        for gi, e in enumerate(self._mat_elems):
            mu, kappa = e.materials.parameters()
            P.assemble_volume(gi, mu, kappa, gc, K=K if want_K else None, R=R,
                              accumulate=(gi > 0 or not store_first))
        for fi, ld in enumerate(self._face_loads):
            P.assemble_pressure(fi, float(ld.pressure), self._Xinst, gc, K=K if want_K else None, R=R)
        return R, (K if want_K else None)

    def assemble_Stiffness_Matrix(self, RGC=None, GC=None):
        """(R [n], K_indices int64 [2,nnz], K_values [nnz]) in reduced numbering
        (assembly.py:283-309)."""
        R, K = self.assemble_csr(self._gc(RGC, GC))
        return R, self.plan.coo_indices(), K

    def assemble_force(self, RGC=None, GC=None):
        """Reduced residual R [n] (assembly.py:230-281)."""
        return self.assemble_csr(self._gc(RGC, GC), want_K=False)[0]

    def _total_Potential_Energy(self, RGC=None, GC=None):
        """sum of element energies + p V of every pressure load (assembly.py:389-415)."""
        P = self.plan
        gc = self._gc(RGC, GC)
        total = torch.zeros((), dtype=torch.float64, device=self.device)
        for gi, e in enumerate(self._mat_elems):
            mu, kappa = e.materials.parameters()
            P.energy_volume(gi, mu, kappa, gc, self._energy_buf)
            total = total + self._energy_buf[0]
        for fi, ld in enumerate(self._face_loads):
            P.pressure_volume(fi, self._Xinst, gc, self._energy_buf)
            total = total + float(ld.pressure) * self._energy_buf[0]
        return total

    # -- dynamics (assembly.py:187-206, 421-443) -----------------------------------
    def initialize_dynamic(self):
        rhos = [float(e.density) for e in self._mat_elems]
        self._minv = self.plan.lumped_mass_inv(rhos)
        self._mass_values = self.plan.mass_csr(rhos)

    def mass_csr(self):
        """Consistent mass as values of the reduced CSR pattern [nnz] (constant)."""
        if getattr(self, "_mass_values", None) is None:
            self.initialize_dynamic()
        return self._mass_values

    def assemble_mass_matrix(self, GC_now=None):
        """(indices int64 [2, nnz], values [nnz]) of the reduced consistent mass
        (assembly.py:421-443): the same sparse matrix as the reference's
        duplicate COO, given on the stiffness pattern (entries that couple
        unlike directions are zero).  The mass does not depend on GC_now."""
        return self.plan.coo_indices(), self.mass_csr()

    def lumped_mass_inv(self):
        if getattr(self, "_minv", None) is None:
            self.initialize_dynamic()
        return self._minv

    def refine_RGC(self, RGC):
        return [r.clone().detach() for r in RGC]
