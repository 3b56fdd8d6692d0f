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
from .boundarys import Boundary_Condition, Boundary_Condition_RP
from .constraints import Couple
from .coupled import CoupledSystem
from .loads import Concentrate_Force, Moment, Pressure
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
        if name is None:
            number = len(self._reference_points)
            while ("rp-%d" % number) in self._reference_points:
                number += 1
            name = "rp-%d" % number
        self._reference_points[name] = rp
        return name

    def get_reference_point(self, name):
        if name not in self._reference_points:
            raise ValueError("Reference point '%s' not found in the model." % name)
        return self._reference_points[name]

    def delete_reference_point(self, name):
        self.get_reference_point(name)
        del self._reference_points[name]

    def add_constraint(self, constraint, name: str = None):
        name = name or self._name(self._constraints, constraint, constraint.__class__.__name__)
        self._constraints[name] = constraint
        return name

    def get_constraint(self, name):
        if name not in self._constraints:
            raise ValueError("Constraint '%s' not found in the model." % name)
        return self._constraints[name]

    def delete_constraint(self, name):
        self.get_constraint(name)
        del self._constraints[name]

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
        self._reference_points = dict(sorted(self._reference_points.items()))
        self._loads = dict(sorted(self._loads.items()))
        self._constraints = dict(sorted(self._constraints.items()))
        self._boundarys = dict(sorted(self._boundarys.items()))
        for name, ld in self._loads.items():
            if not isinstance(ld, (Pressure, Concentrate_Force, Moment)):
                raise NotImplementedError("load %r (%s) is outside the B200 path" % (name, type(ld).__name__))
        for name, b in self._boundarys.items():
            if not isinstance(b, (Boundary_Condition, Boundary_Condition_RP)):
                raise NotImplementedError("boundary %r (%s) is outside the B200 path" % (name, type(b).__name__))
        for name, c in self._constraints.items():
            if not isinstance(c, Couple):
                raise NotImplementedError("constraint %r (%s) is outside the B200 path" % (name, type(c).__name__))
        if not self._instances:
            raise ValueError("the assembly has no instance")
        self.RGC, self.RGC_remain_index, self.RGC_list_indexStart, self._RGC_size = [], [], [0], []
        idx = None
        for ins in self._instances.values():
            idx = self._allocate_RGC(ins._RGC_requirements)
            ins.set_RGC_index(idx)
        for rp in self._reference_points.values():
            idx = self._allocate_RGC((rp._RGC_requirements,))
            rp.set_RGC_index(idx)
        self.RGC[idx][-1] = 1e-5                  # the reference's seed (assembly.py:113)
        for ld in self._loads.values():
            ld.set_RGC_index(self._allocate_RGC(ld._RGC_requirements))
        for c in self._constraints.values():
            c.set_RGC_index(self._allocate_RGC(c._RGC_requirements))
        for b in self._boundarys.values():
            b.set_RGC_index(self._allocate_RGC(b._RGC_requirements))
        for part in self._parts.values():
            part.initialize(self)
        for ins in self._instances.values():
            ins.initialize(self)
        for rp in self._reference_points.values():
            rp.initialize(self)
        for ld in self._loads.values():
            ld.initialize(self)
        for c in self._constraints.values():
            c.initialize(self)
        for b in self._boundarys.values():
            b.initialize(self)
        # required DOFs: element nodes, pressure face nodes, reference points
        # carrying loads or ties; tied nodes and Dirichlet DOFs removed
        # (assembly.py:150-170)
        for ins in self._instances.values():
            rem = self.RGC_remain_index[ins._RGC_index]
            for e in ins.part.elems.values():
                rem = e.set_required_DoFs(rem)
        for ld in self._loads.values():
            if isinstance(ld, Pressure):
                rem = self.RGC_remain_index[ld._load_index]
                for s in ld.surface_element:
                    rem[np.unique(s._elems.numpy())] = True
            else:
                ld.set_required_DoFs(self.RGC_remain_index)
        for c in self._constraints.values():
            c.set_required_DoFs(self.RGC_remain_index)
        for b in self._boundarys.values():
            rem = self.RGC_remain_index[b._constraint_index]
            if isinstance(b, Boundary_Condition_RP):
                for d in b.indexDoF:
                    rem[d] = False
                    self.RGC[b._constraint_index][d] = 0.0
                continue
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
            X.append(self._element_frame_nodes(ins))
            Xi.append(ins.nodes.to(torch.float64).cpu())
            rem = self.RGC_remain_index[ins._RGC_index].copy()
            for c in self._constraints.values():      # tied nodes stay rows of the plan
                if c._couple_index == ins._RGC_index:
                    rem[c._indexNodes] = True
            masks.append((rem[:, 0] * 1 + rem[:, 1] * 2 + rem[:, 2] * 4).astype(np.uint8))
            for e in ins.part.elems.values():
                if e.materials is None:
                    raise ValueError("element group without materials")
                groups.append((e.kind, e._elems.numpy() + off))
                mats.append(e)
            off += ins.part.nodes.shape[0]
        for ld in self._loads.values():
            if not isinstance(ld, Pressure):              # point loads act on reference points only
                continue
            o = self._node_offset[ld.instance_name]
            for s in ld.surface_element:
                faces.append((s.kind, s._elems.numpy() + o))
                self._face_loads.append(ld)
        self._mat_elems = mats
        plan_mask = np.concatenate(masks)
        self._plan = DevicePlan(torch.cat(X), plan_mask, groups, faces, device=self.device)
        self._Xinst = torch.cat(Xi).to(self.device).contiguous()
        self._energy_buf = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._system = None
        if self._constraints:
            tied = []
            for c in self._constraints.values():
                name = next(k for k, v in self._instances.items() if v._RGC_index == c._couple_index)
                tied.append((c, c._indexNodes + self._node_offset[name], c.rp_name))
            self._system = CoupledSystem(self, plan_mask, tied)
        elif self._reference_points:
            raise NotImplementedError("reference points without a Couple constraint are outside the B200 path")

    @property
    def system(self):
        """The reduced linear system the solvers see (CSR, PCG): the plan
        itself, or the system condensed onto reference points when nodes are
        tied to them."""
        return self._system if self._system is not None else self.plan

    @staticmethod
    def _element_frame_nodes(ins):
        """Coordinates the element kernels of an instance use: the part's
        nodes, rotated by the instance's rotation when it has one.  With the
        instance's displacement (assembly frame) this gives the reference's
        rotated element outputs R R_e, R K_e R^T (C3base.py:417-418,
        441-443) for the isotropic material; translation does not enter the
        element arithmetic."""
        X = ins.part.nodes.to(torch.float64).cpu()
        R = ins.rotation_matrix.to(torch.float64).cpu()
        return X if torch.equal(R, torch.eye(3, dtype=torch.float64)) else X @ R.T

    @property
    def plan(self) -> DevicePlan:
        if self._plan is None:
            raise RuntimeError("Assembly.initialize() has not been called")
        return self._plan

    # -- GC <-> RGC (assembly.py:470-499) ---------------------------------------
    def _GC2RGC(self, GC):
        full = torch.zeros(self.RGC_list_indexStart[-1], dtype=torch.float64, device=self.device)
        full[self._remain_dev] = GC.to(self.device, torch.float64)
        RGC = [full[self.RGC_list_indexStart[i]:self.RGC_list_indexStart[i + 1]].view(self._RGC_size[i])
               for i in range(len(self._RGC_size))]
        for c in self._constraints.values():      # tied nodes follow their points (couple.py:34-40)
            RGC = c.modify_RGC(RGC)
        return RGC

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
        if self._system is not None:
            S = self._system
            gc = self._gc(GC=GC)
            mot = S.motions(gc)
            Rp, Kp = self._assemble_plan(S.plan_gc(gc, mot), want_K, None, None)
            Rr, Kr = S.condense(gc, Rp, Kp, mot)
            if R is not None:
                R.copy_(Rr)
                Rr = R
            if K is not None and Kr is not None:
                K.copy_(Kr)
                Kr = K
            return Rr, Kr
        return self._assemble_plan(self._gc(GC=GC), want_K, K, R)

    def _assemble_plan(self, gc, want_K, K, R):
        """R and K of the plan's rows at the plan displacement gc."""
        P = self.plan
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
        return R, self.system.coo_indices(), K

    def assemble_force(self, RGC=None, GC=None):
        """Reduced residual R [n] (assembly.py:230-281)."""
        return self.assemble_csr(self._gc(RGC, GC), want_K=False)[0]

    def _total_Potential_Energy(self, RGC=None, GC=None):
        """sum of element energies + p V of every pressure load (assembly.py:389-415)."""
        P = self.plan
        gc = self._gc(RGC, GC)
        total = torch.zeros((), dtype=torch.float64, device=self.device)
        if self._system is not None:
            S = self._system
            gcr = gc
            gc = S.plan_gc(gcr)
            f = S.point_loads()
            for name, rp, keep, b0 in S.points:
                if name in f:
                    q = torch.zeros(6, dtype=torch.float64, device=self.device)
                    q[torch.as_tensor(keep, device=self.device)] = gcr[b0:b0 + keep.shape[0]]
                    total = total - (f[name] * q).sum()
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
        if self._system is not None:
            raise NotImplementedError("dynamics with reference points are outside the B200 path")
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
