"""Solvers on the B200 kernels (mirrors FEA/solver of sssnnn7119/FEA).

StaticImplicitSolver keeps the reference's Newton control flow — Armijo
backtracking on the total potential, low-alpha bookkeeping, the absolute
stop test (static_implicit.py:153-350) — and replaces the linear solve by
the device Jacobi-PCG (static_implicit.py:352-405: symmetric Jacobi scaling
+ CG is Jacobi-PCG).  Where the reference switches to its CPU direct solver
(scaled residual below 1e-3, or repeated small steps, static_implicit.py:
384-388) this solver runs the PCG to a tight tolerance instead.  ``rtol``
adds a relative stop test ||R|| / ||R_first|| <= rtol; in that mode a
residual that has stopped falling below ``floor_rtol`` (1e-9) of the first
one is the round-off floor and also ends the iteration.

DynamicImplicitSolver keeps the reference's Newmark time loop and per-step
Newton (dynamic_implicit.py) on the same device kernels, with the consistent
mass in the stiffness pattern.

DynamicExplicitSolver keeps the reference's time and storage bookkeeping
(dynamic_explicit.py:66-145) and advances the state with the fused
explicit kernel between storage points.
"""
from __future__ import annotations

import math
import time

import torch

from . import _lib as L
from ._trace import nvtx


class LinearSolve:
    """One tangent solve K x = b asked for by the Newton iteration: K in the
    plan's CSR order, b, the warm start x (updated in place), the squared
    scaled-residual tolerance and the iteration cap; the solver of the
    request fills in iterations, relres and the status code."""

    __slots__ = ("K", "b", "x", "x0", "tol", "cap", "tight", "it", "rr", "status")

    def __init__(self, K, b, x, tol, cap, tight):
        self.K, self.b, self.x, self.x0 = K, b, x, x.clone()
        self.tol, self.cap, self.tight = tol, cap, tight
        self.it, self.rr, self.status = 0, 0.0, L.FEA_OK


class BaseSolver:
    def __init__(self) -> None:
        self.assembly = None
        self.GC = None

    def initialize(self, assembly, *args, **kwargs):
        self.assembly = assembly

    def solve(self, GC0=None, *args, **kwargs):
        raise NotImplementedError


class StaticImplicitSolver(BaseSolver):
    def __init__(self, maximum_iteration: int = 10000, tol_error: float = 1e-5, rtol: float = None,
                 pcg_tol: float = 1e-5, pcg_max_iter: int = 1500, tight_pcg_tol: float = 1e-22,
                 tight_pcg_max_iter: int = 20000, precision: str = "fp64", verbose: bool = False,
                 device_line_search: bool = True) -> None:
        super().__init__()
        self.device_line_search = device_line_search
        # FP32 inner solves: a residual replacement after every batch of
        # iterations (0) or once the FP32 residual fell by this factor
        self.inner_tol = 0.0
        self.maximum_iteration = maximum_iteration
        self.tol_error = tol_error
        self.rtol = rtol
        self.pcg_tol = pcg_tol
        self.pcg_max_iter = pcg_max_iter
        self.tight_pcg_tol = tight_pcg_tol
        self.tight_pcg_max_iter = tight_pcg_max_iter
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self.verbose = verbose
        self.floor_rtol = 1e-9
        self._iter_now = 0
        self._maximum_step_length = 1e10
        self._low_alpha_count = 0
        self.history = []

    def solve(self, GC0=None, *args, **kwargs):
        t0 = time.time()
        if GC0 is None:
            GC0 = self.assembly.GC
        result = self._solve_iteration(GC=self.assembly._gc(GC=GC0), tol_error=self.tol_error)
        if isinstance(result, bool):
            return result
        self.GC = result
        self.assembly.GC = result
        self.assembly.RGC = self.assembly._GC2RGC(result)
        if self.verbose:
            print("total_iter:%d, total_time:%.2f" % (self._iter_now, time.time() - t0))
        return self.GC

    def get_total_energy(self, GC_now):
        return self.assembly._total_Potential_Energy(GC=GC_now)

    def get_stiffness_matrix(self, GC_now):
        return self.assembly.assemble_Stiffness_Matrix(GC=GC_now)

    def _line_search(self, GC0, dGC, R, energy0):
        """Armijo backtracking, c1 = 0.3, halving, alpha < 1e-12 -> 0
        (static_implicit.py:97-169): on the device (a ladder of trial steps
        per launch, one host read per ladder) unless the assembly has
        reference points or the predicted decrease is at round-off level."""
        self._last_smax = None
        if self.device_line_search and getattr(self.assembly, "_system", None) is None:
            res = self._line_search_device(GC0, dGC, R, energy0)
            if res is not None:
                return res
        return self._line_search_host(GC0, dGC, R, energy0)

    def _line_search_device(self, GC0, dGC, R, energy0):
        A = self.assembly
        P = A.plan
        dev = GC0.device
        e0 = torch.as_tensor(energy0, dtype=torch.float64, device=dev).reshape(1).contiguous()
        st = torch.empty(L.FEA_LS_NSTATE, dtype=torch.float64, device=dev)
        dGC = dGC.contiguous()
        P.ls_prepare(dGC, R.contiguous(), e0, st)
        gc = GC0.clone().contiguous()
        E = torch.empty(L.FEA_LS_M, dtype=torch.float64, device=dev)
        for k0 in range(0, 40, L.FEA_LS_M):
            acc = False
            for gi, e in enumerate(A._mat_elems):
                mu, kappa = e.materials.parameters()
                P.ls_energy_volume(gi, mu, kappa, GC0, dGC, st, k0, E, acc)
                acc = True
            for fi, ld in enumerate(A._face_loads):
                P.ls_energy_pressure(fi, float(ld.pressure), A._Xinst, GC0, dGC, st, k0, E, acc)
                acc = True
            P.ls_select(E, k0, 0.3, self._maximum_step_length, st, dGC, gc)
            h = st.tolist()
            if not (math.isfinite(h[L.FEA_LS_DE]) and math.isfinite(h[L.FEA_LS_SMAX])):
                raise ValueError("dGC has nan or inf")
            if h[L.FEA_LS_ROUND] != 0.0:
                return None
            self._last_smax = h[L.FEA_LS_SMAX]
            if h[L.FEA_LS_FOUND] == 1.0:
                return abs(h[L.FEA_LS_ALPHA]), gc, st[L.FEA_LS_ENEW].clone()
            if h[L.FEA_LS_FOUND] != 0.0:
                break
        return 0.0, GC0.clone(), energy0

    def _line_search_host(self, GC0, dGC, R, energy0):
        """The line search on the host: one energy (or, at round-off level,
        one residual norm) per trial step.

        When the predicted energy decrease is below the round-off of the
        energy itself (|dGC . R| <= 1e-10 |E|), the energy comparison carries
        no information; there a trial step is accepted when it reduces the
        residual norm instead.
        """
        alpha, c1 = 1.0, 0.3
        deltaE = float((dGC * R).sum())
        if deltaE > 0:
            dGC, deltaE = -dGC, -deltaE
        if not bool(torch.isfinite(dGC).all()):
            raise ValueError("dGC has nan or inf")
        e0 = float(energy0)
        step_max = float(dGC.abs().max())
        roundoff = abs(deltaE) <= 1e-10 * abs(e0)
        r0 = float(R.norm())
        while True:
            GCnew = GC0 + alpha * dGC
            if roundoff:
                rn = float(self.assembly.assemble_force(GC=GCnew).norm())
                ok = math.isfinite(rn) and rn < r0
            else:
                e_new = float(self.get_total_energy(GCnew))
                ok = math.isfinite(e_new) and e_new <= e0 + c1 * deltaE * alpha
            if ok and alpha * step_max <= self._maximum_step_length:
                e_new = float(self.get_total_energy(GCnew)) if roundoff else e_new
                return alpha, GCnew, torch.tensor(e_new, dtype=torch.float64)
            alpha *= 0.5
            if alpha < 1e-12:
                return 0.0, GC0.clone(), energy0

    def _solve_iteration(self, GC, tol_error):
        """Newton loop (static_implicit.py:234-350); returns GC or False.
        The linear solves asked for by the loop run on this device's PCG."""
        gen = self._newton(GC, tol_error)
        try:
            req = next(gen)
            while True:
                self._run_linear(req)
                req = gen.send(None)
        except StopIteration as stop:
            return stop.value

    def _newton(self, GC, tol_error):
        """The Newton loop as a generator: it yields a ``LinearSolve`` for each
        tangent solve and resumes once the caller has filled in its result
        (``_run_linear`` here; the batched engine of ``fea_b200.serving``
        when many solves share the device).  Returns GC or False."""
        self._iter_now = 0
        self._last_smax = None
        energy = self.get_total_energy(GC)
        dGC = torch.zeros_like(GC)
        low_alpha, alpha = 0, 0.0
        r_first = None
        self.history = []
        while True:
            if self._iter_now > self.maximum_iteration:
                return False
            R, Kv = self.assembly.assemble_csr(GC)
            self._iter_now += 1
            if R.numel():
                # one host read for the residual statistics of this iteration
                rmax, rnorm, srmax = torch.stack([R.abs().max(), R.norm(), self._scaled_rmax_dev(Kv, R)]).tolist()
            else:
                rmax, rnorm, srmax = 0.0, 0.0, 0.0
            if r_first is None:
                r_first = rnorm
            self.history.append(dict(iter=self._iter_now, rmax=rmax, rnorm=rnorm))
            if self.rtol is not None and rnorm <= self.rtol * max(r_first, 1e-300):
                break
            if self._at_floor(r_first):
                break
            req = self._linear_request(Kv, -R, self._iter_now, alpha, dGC, srmax=srmax)
            yield req
            dGC = self._linear_finish(req, Kv, -R)
            alpha, GCnew, energynew = self._line_search(GC, dGC, R, energy)
            self.history[-1].update(alpha=alpha)
            if alpha == 0 and rmax > tol_error and self.rtol is None:
                return False
            if alpha == 0:
                break
            if alpha < 0.01:
                low_alpha += 1
            else:
                low_alpha = max(0, low_alpha - 5)
            if low_alpha > 10:
                if self.rtol is not None and rnorm <= self.floor_rtol * r_first:
                    break
                return False
            GC = GCnew
            energy = self.get_total_energy(GC)
            if self.verbose:
                print("iter %3d  alpha %.2f  energy %.10e  max|R| %.4e" % (self._iter_now, alpha, float(energy), rmax))
            if self.rtol is None:
                dmax = self._last_smax if self._last_smax is not None else float(dGC.abs().max())
                if (dmax < tol_error and rmax < tol_error) or rmax < 1e-6:
                    break
        return GC

    def _at_floor(self, r_first):
        """Relative-residual mode only: the residual has stopped falling
        (no halving over the last three iterations) below ``floor_rtol`` of
        the first residual, i.e. Newton has reached the round-off floor of
        the residual evaluation and further iterations cannot reach ``rtol``."""
        h = self.history
        if self.rtol is None or len(h) < 4 or r_first == 0.0:
            return False
        last = h[-1]["rnorm"]
        return last <= self.floor_rtol * r_first and last > 0.5 * min(x["rnorm"] for x in h[-4:-1])

    def _solve_linear_equation(self, K_values, R, iter_now=0, alpha0=None, dGC0=None, tol_error=None):
        """K dGC = R by device PCG, warm-started from the previous step (static_implicit.py:352-405)."""
        req = self._linear_request(K_values, R, iter_now, alpha0, dGC0)
        self._run_linear(req)
        return self._linear_finish(req, K_values, R)

    def _linear_request(self, K_values, R, iter_now=0, alpha0=None, dGC0=None, srmax=None):
        """The PCG tolerance and cap for this Newton iteration: loose solves
        far from equilibrium, a tight solve where the reference switches to
        its exact solver (scaled residual below 1e-3, or repeated small
        steps, static_implicit.py:384-388)."""
        x = (torch.zeros_like(R) if dGC0 is None else dGC0.clone()).contiguous()
        alpha0 = 1e-10 if alpha0 is None else alpha0
        self._low_alpha_count = self._low_alpha_count + 1 if alpha0 < 1e-1 else 0
        if srmax is None:
            srmax = self._scaled_rmax(K_values, R)
        tight = self._low_alpha_count > 3 or srmax < 1e-3
        if tight:
            tol, cap = self.tight_pcg_tol, self.tight_pcg_max_iter
            self._low_alpha_count = 0
        else:
            tol = self.pcg_tol
            cap = 6000 if (iter_now % 20 == 0 or self._low_alpha_count > 0) else self.pcg_max_iter
        return LinearSolve(K_values, R.contiguous(), x, tol, cap, tight)

    def _run_linear(self, req):
        with nvtx("fea.pcg"):
            self._run_linear_inner(req)

    def _run_linear_inner(self, req):
        P = self.assembly.system
        if self.precision == "mixed":
            req.it, outer, req.rr, req.status = P.pcg_mixed(req.K, None, req.b, req.x, req.tol, self.inner_tol,
                                                            req.cap, raise_on_breakdown=False)
        else:
            req.it, req.rr, req.status = P.pcg(req.K, req.b, req.x, req.tol, req.cap, raise_on_breakdown=False)

    def _linear_finish(self, req, K_values, R):
        self.history[-1].update(pcg_iters=req.it, pcg_relres=req.rr, pcg_tight=req.tight, pcg_status=req.status)
        x = req.x
        if req.status == L.FEA_EBREAKDOWN:
            # K is not positive definite along the search space: keep the
            # iterate reached before the negative curvature (truncated CG);
            # with no progress, take the Jacobi-scaled residual direction
            if not bool(torch.isfinite(x).all()) or bool(torch.equal(x, req.x0)):
                x = R / self._diag(K_values).abs()
        return x

    def _scaled_rmax(self, K_values, R):
        return float(self._scaled_rmax_dev(K_values, R)) if R.numel() else 0.0

    def _scaled_rmax_dev(self, K_values, R):
        """max |R_i| / sqrt|K_ii| as a device scalar (static_implicit.py:384-388 test)."""
        diag = self._diag(K_values)
        return (R / diag.abs().sqrt().clamp_min(1e-300)).abs().max()

    def _diag(self, K_values):
        P = self.assembly.system
        if not hasattr(self, "_diag_pos") or self._diag_pos.numel() != P.ndof:
            rows = P.coo_indices()
            self._diag_pos = torch.nonzero(rows[0] == rows[1]).flatten()
        d = K_values[self._diag_pos]
        return torch.where(d == 0, torch.ones_like(d), d)


class DynamicImplicitSolver(StaticImplicitSolver):
    """Implicit Newmark dynamics (dynamic_implicit.py:15-501).

    Average acceleration (beta = 1/4, gamma = 1/2).  Each step predicts
    GC_pre = GC + dt GV + dt^2 GA / 4 and minimises the incremental energy
    Pi(x) + (x - GC_pre) M (x - GC_pre) / (2 beta dt^2) by Newton with the
    reference's Armijo line search and stop test; the tangent K + M /
    (beta dt^2) and the consistent mass M share the plan's CSR pattern, so
    the effective tangent is one axpy on the values and M x one node-row
    SpMV.  The linear solves are the device Jacobi-PCG of
    StaticImplicitSolver (tight where the reference takes its direct
    solver).  The initial acceleration solves M a0 = R(GC0) with the
    assembled residual R, as the reference does (dynamic_implicit.py:290-302).
    """

    def __init__(self, maximum_iteration: int = 10000, deltaT: float = 1e-2, time_end: float = 1.0,
                 tol_error: float = 1e-5, pcg_tol: float = 1e-5, pcg_max_iter: int = 1500,
                 tight_pcg_tol: float = 1e-22, tight_pcg_max_iter: int = 20000, verbose: bool = False) -> None:
        super().__init__(maximum_iteration=maximum_iteration, tol_error=tol_error, pcg_tol=pcg_tol,
                         pcg_max_iter=pcg_max_iter, tight_pcg_tol=tight_pcg_tol,
                         tight_pcg_max_iter=tight_pcg_max_iter, verbose=verbose)
        # the step's incremental potential includes the inertia term, which
        # the device ladder does not evaluate: the host line search serves
        self.device_line_search = False
        self._deltaT = deltaT
        self._time_end = time_end
        self._gamma = 0.5
        self._beta = 0.25
        self._GC_list = None
        self._GV_list = None
        self._GA_list = None
        self._time_list = []
        self._deltaT_list = []

    def initialize(self, assembly, *args, **kwargs):
        super().initialize(assembly)
        self.assembly.initialize_dynamic()
        self._GC_list, self._GV_list, self._GA_list = [], [], []
        self._time_list, self._deltaT_list = [], []

    def set_deltaT(self, deltaT: float):
        self._deltaT = deltaT

    # -- energies and the incremental system (dynamic_implicit.py:88-146) --------
    def _mass_dot(self, x):
        return self.assembly.plan.spmv(self.assembly.mass_csr(), x.contiguous())

    def get_total_energy(self, GC_now, GC0=None, GV0=None, GA0=None, deltaT=None):
        """Pi(GC_now) + v M v / 2 with v the Newmark velocity at GC_now."""
        if GC0 is None:
            return self.assembly._total_Potential_Energy(GC=GC_now)
        deltaT = self._deltaT if deltaT is None else deltaT
        v = self.get_next_velocity(GC_now, GC0, GV0, GA0, deltaT)[0]
        return self.assembly._total_Potential_Energy(GC=GC_now) + 0.5 * torch.dot(v, self._mass_dot(v))

    def get_incremental_energy(self, GC_now, GC_pre, deltaT=None):
        deltaT = self._deltaT if deltaT is None else deltaT
        d = GC_now - GC_pre
        return (self.assembly._total_Potential_Energy(GC=GC_now)
                + torch.dot(d, self._mass_dot(d)) / (2 * self._beta * deltaT ** 2))

    def _incremental_csr(self, GC_now, GC_pre):
        """(R + M (x - x_pre) / (beta dt^2), CSR values of K + M / (beta dt^2))."""
        c = 1.0 / (self._beta * self._deltaT ** 2)
        R, Kv = self.assembly.assemble_csr(GC_now)
        P = self.assembly.plan
        P.axpy(c, self._mass_dot(GC_now - GC_pre), R)
        P.axpy(c, self.assembly.mass_csr(), Kv)
        return R, Kv

    def get_incremental_stiffness_matrix(self, GC_now, GC_pre):
        """(R, K_indices int64 [2, nnz], K_values) of the step's Newton system."""
        R, Kv = self._incremental_csr(GC_now, GC_pre)
        return R, self.assembly.plan.coo_indices(), Kv

    def get_next_velocity(self, GC_now, GC0, GV0, GA0, deltaT):
        """Newmark velocity and acceleration at GC_now (dynamic_implicit.py:269-289)."""
        g, b = self._gamma, self._beta
        GV_now = g / (b * deltaT) * (GC_now - GC0) + (1 - g / b) * GV0 + deltaT * (1 - g / (2 * b)) * GA0
        GA_now = 1 / (b * deltaT ** 2) * (GC_now - GC0) - 1 / (b * deltaT) * GV0 - (1 / (2 * b) - 1) * GA0
        return GV_now, GA_now

    def get_current_acceleration(self, GC0, GV0=None):
        """M a = R(GC0), the assembled residual, as in the reference
        (dynamic_implicit.py:290-302); M by device PCG to round-off."""
        P = self.assembly.plan
        R = self.assembly.assemble_force(GC=GC0).contiguous()
        a = torch.zeros_like(R)
        P.pcg(self.assembly.mass_csr(), R, a, 1e-26, 10000, raise_on_breakdown=True)
        return a

    # -- time loop (dynamic_implicit.py:148-226) ---------------------------------
    def solve(self, GC0=None, GV0=None, *args, **kwargs):
        t0 = time.time()
        if GC0 is None:
            GC0 = self.assembly.GC.clone()
        GC0 = self.assembly._gc(GC=GC0)
        GV0 = torch.zeros_like(GC0) if GV0 is None else GV0.to(GC0.device, torch.float64)
        self._GC_list = [GC0]
        self._GV_list = [GV0]
        self._GA_list = [self.get_current_acceleration(GC0=GC0, GV0=GV0)]
        self._time_list = [0.0]
        self._deltaT_list = []
        self.E_history = [float(self.get_total_energy(GC0, GC0, GV0, self._GA_list[-1]))]
        step = 0
        while True:
            dt = self._deltaT
            GC_pre = self._GC_list[-1] + dt * self._GV_list[-1] + 0.25 * dt ** 2 * self._GA_list[-1]
            with nvtx("fea.newmark_step"):
                GC_now = self._solve_iteration(GC0=self._GC_list[-1], GC_pre=GC_pre, deltaT=dt,
                                               tol_error=self.tol_error)
            if isinstance(GC_now, bool):
                raise RuntimeError("Newton iteration of time step %d did not converge" % (step + 1))
            GV, GA = self.get_next_velocity(GC_now, self._GC_list[-1], self._GV_list[-1], self._GA_list[-1], dt)
            self.E_history.append(float(self.get_total_energy(GC_now, self._GC_list[-1], self._GV_list[-1],
                                                              self._GA_list[-1], dt)))
            self._GC_list.append(GC_now)
            self._GV_list.append(GV)
            self._GA_list.append(GA)
            self._deltaT_list.append(dt)
            self._time_list.append(self._time_list[-1] + dt)
            step += 1
            if self.verbose:
                print("step %d  time %.6g  newton %d" % (step, self._time_list[-1], self._iter_now))
            if self._time_list[-1] >= self._time_end:
                break
        self.GC = self._GC_list[-1]
        self.assembly.RGC = self.assembly.refine_RGC(self.assembly._GC2RGC(self.assembly.GC))
        if self.verbose:
            print("total_time:%.2f" % (time.time() - t0))
        return True

    # -- Newton per step (dynamic_implicit.py:304-460) ---------------------------
    def _dyn_line_search(self, GC_now, GC_pre, dGC, R, energy0, deltaT):
        """Armijo backtracking on the incremental energy (c1 = 0.3, halving,
        alpha < 1e-12 -> 0).  As in StaticImplicitSolver, where the predicted
        decrease is below the energy's round-off the trial step is accepted
        when it reduces the residual norm instead."""
        alpha, c1 = 1.0, 0.3
        deltaE = float((dGC * R).sum())
        if deltaE > 0:
            dGC, deltaE = -dGC, -deltaE
        if not bool(torch.isfinite(dGC).all()):
            raise ValueError("dGC has nan or inf")
        e0 = float(energy0)
        step_max = float(dGC.abs().max())
        roundoff = abs(deltaE) <= 1e-10 * abs(e0)
        r0 = float(R.norm())
        while True:
            GCnew = GC_now + alpha * dGC
            if roundoff:
                rn = float(self._incremental_csr(GCnew, GC_pre)[0].norm())
                ok = math.isfinite(rn) and rn < r0
                e_new = float(self.get_incremental_energy(GCnew, GC_pre, deltaT)) if ok else e0
            else:
                e_new = float(self.get_incremental_energy(GCnew, GC_pre, deltaT))
                ok = math.isfinite(e_new) and e_new <= e0 + c1 * deltaE * alpha
            if ok and alpha * step_max <= self._maximum_step_length:
                return alpha, GCnew, e_new
            alpha *= 0.5
            if alpha < 1e-12:
                return 0.0, GC_now.clone(), e0

    def _solve_iteration(self, GC0, GC_pre=None, deltaT=None, tol_error=None):
        """Newton on the step's incremental energy; returns GC or False."""
        if GC_pre is None:                        # the static signature (GC, tol_error)
            return super()._solve_iteration(GC0, tol_error)
        deltaT = self._deltaT if deltaT is None else deltaT
        tol_error = self.tol_error if tol_error is None else tol_error
        GC_now = GC0.clone()
        self._iter_now = 0
        self.history = []
        energy = float(self.get_incremental_energy(GC_now, GC_pre, deltaT))
        dGC = torch.zeros_like(GC0)
        low_alpha, alpha = 0, 0.0
        while True:
            if self._iter_now > self.maximum_iteration:
                self.assembly.GC = GC_now
                return False
            R, Kv = self._incremental_csr(GC_now, GC_pre)
            self._iter_now += 1
            rmax = float(R.abs().max()) if R.numel() else 0.0
            self.history.append(dict(iter=self._iter_now, rmax=rmax, rnorm=float(R.norm())))
            req = self._linear_request(Kv, -R, self._iter_now, alpha, dGC)
            self._run_linear(req)
            dGC = self._linear_finish(req, Kv, -R)
            alpha, GCnew, energy_new = self._dyn_line_search(GC_now, GC_pre, dGC, R, energy, deltaT)
            self.history[-1].update(alpha=alpha)
            if alpha == 0 and rmax > tol_error:
                self.assembly.GC = GC_now
                return False
            if alpha == 0:
                break
            if alpha < 0.01:
                low_alpha += 1
            else:
                low_alpha = max(0, low_alpha - 5)
            if low_alpha > 10:
                if rmax < 1e-3:
                    self.assembly.GC = GC_now
                    break
                return False
            energy = float(self.get_incremental_energy(GCnew, GC_pre, deltaT))
            GC_now = GCnew
            if float(dGC.abs().max()) < tol_error and rmax < tol_error:
                break
        return GC_now


class DynamicExplicitSolver(BaseSolver):
    """Central difference with lumped mass (dynamic_explicit.py:10-167).

    The reference advances each step from the last *stored* displacement
    (dynamic_explicit.py:100), which only follows the central-difference
    recurrence when a state is stored at every step; this solver always
    advances from the previous step.
    """

    def __init__(self, time_end: float = 1.0, time_per_storage: float = 1e-4, fp32: bool = False) -> None:
        super().__init__()
        self._time_end = time_end
        self._time_per_storage = time_per_storage
        self._next_storage_time = 0.0
        self._GC_list = None
        self._GV_list = None
        self._GA_list = None
        self._time_list = []
        self._deltaT = 0.0
        self.fp32 = fp32

    def initialize(self, assembly, *args, **kwargs):
        super().initialize(assembly)
        self.assembly.initialize_dynamic()
        self._deltaT = self.estimate_critical_timestep()
        if self._deltaT <= 0:
            raise ValueError("Critical timestep must be positive.")
        self._GC_list, self._GV_list, self._GA_list, self._time_list = [], [], [], []

    def estimate_critical_timestep(self, safety_factor=0.8) -> float:
        """The reference's placeholder (dynamic_explicit.py:54-64); see cfl_timestep."""
        return safety_factor * 5e-6

    def cfl_timestep(self, factor=0.5) -> float:
        """factor * min_e(l_e / c): l_e = smallest tet altitude 3V/max face area,
        c = sqrt((kappa + 4 mu / 3) / rho) (one C3D4 group)."""
        P = self.assembly.plan
        es = self.assembly._mat_elems
        if len(es) != 1 or es[0].kind != "C3D4":
            raise NotImplementedError("cfl_timestep covers one C3D4 group")
        e = es[0]
        x = P.X[e._elems.to(P.device)]
        v = torch.einsum("ei,ei->e", torch.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], dim=1), x[:, 3] - x[:, 0]).abs() / 6
        fa = []
        for tri in ([0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]):
            a = x[:, tri]
            fa.append(0.5 * torch.cross(a[:, 1] - a[:, 0], a[:, 2] - a[:, 0], dim=1).norm(dim=1))
        hmin = float((3 * v / torch.stack(fa, 1).max(1).values).min())
        mu, kappa = e.materials.parameters()
        c = math.sqrt((kappa + 4 * mu / 3) / float(e.density))
        return factor * hmin / c

    def _fused_group(self):
        """(group, (mu, kappa)) when one fused launch per step covers the
        model (one element group, no loads), else None."""
        es = self.assembly._mat_elems
        if len(es) != 1 or self.assembly._face_loads:
            return None
        return 0, es[0].materials.parameters()

    def solve(self, GC0=None, GV0=None, *args, **kwargs):
        A = self.assembly
        P = A.plan
        dt = float(self._deltaT)
        u = (A.GC.clone() if GC0 is None else A._gc(GC=GC0).clone()).contiguous()
        v = (torch.zeros_like(u) if GV0 is None else A._gc(GC=GV0).clone()).contiguous()
        vh = torch.empty_like(u)
        a = torch.empty_like(u)
        minv = A.lumped_mass_inv()
        fused = self._fused_group()
        if fused is None:
            return self._solve_assembled(u, v, vh, a, minv, dt)
        gi, (mu, kappa) = fused
        # a_0 and vh_{-1/2} (dynamic_explicit.py:80-91)
        P.explicit_run(gi, mu, kappa, minv, dt, 0, u, vh, a, v, fp32=self.fp32, init=True)
        self._GC_list.append(u.clone())
        self._GV_list.append(v.clone())
        self._GA_list.append(a.clone())
        self._time_list.append(0.0)
        # the reference's time / storage bookkeeping (dynamic_explicit.py:97-134)
        current_time, pending = 0.0, 0
        while current_time < self._time_end:
            current_time += dt
            pending += 1
            if current_time >= self._next_storage_time or current_time >= self._time_end:
                P.explicit_run(gi, mu, kappa, minv, dt, pending, u, vh, a, v, fp32=self.fp32, init=False)
                pending = 0
                self._GC_list.append(u.clone())
                self._GV_list.append(v.clone())
                self._GA_list.append(a.clone())
                self._time_list.append(current_time)
                self._next_storage_time += self._time_per_storage
        if pending:
            P.explicit_run(gi, mu, kappa, minv, dt, pending, u, vh, a, v, fp32=self.fp32, init=False)
        self.GC = u
        self.GV, self.GA, self.GV_half = v, a, vh
        return True

    def _solve_assembled(self, u, v, vh, a, minv, dt):
        """The reference's loop for several element groups and loads
        (dynamic_explicit.py:80-134): each step the residual of every group
        and load is assembled by the residual kernels (assemble_force) between
        the two stages of fea_explicit_stage."""
        if self.fp32:
            raise NotImplementedError("the FP32 element force covers the fused one-group path")
        A = self.assembly
        P = A.plan
        R = torch.empty_like(u)
        vhp = torch.empty_like(u)
        A.assemble_csr(u, want_K=False, R=R)
        P.explicit_stage(2, dt, minv, R, None, vh, None, a, v)
        self._GC_list.append(u.clone())
        self._GV_list.append(v.clone())
        self._GA_list.append(a.clone())
        self._time_list.append(0.0)
        current_time = 0.0
        while current_time < self._time_end:
            P.explicit_stage(0, dt, minv, None, u, vh, vhp, a, None)
            A.assemble_csr(u, want_K=False, R=R)
            P.explicit_stage(1, dt, minv, R, None, vh, vhp, a, v)
            current_time += dt
            if current_time >= self._next_storage_time or current_time >= self._time_end:
                self._GC_list.append(u.clone())
                self._GV_list.append(v.clone())
                self._GA_list.append(a.clone())
                self._time_list.append(current_time)
                self._next_storage_time += self._time_per_storage
        self.GC = u
        self.GV, self.GA, self.GV_half = v, a, vh
        return True

    def get_lumped_mass_inv(self, GC=None):
        return self.assembly.lumped_mass_inv()


class _LinearSolverModule:
    """``_linear_solver`` namespace (FEA/solver/_linear_solver.py)."""

    @staticmethod
    def conjugate_gradient(A_indices, A_values, b, x0=None, tol: float = 1e-3, max_iter: int = 1500):
        """Plain CG on a COO matrix with the reference's stop test ||r||^2/||b||^2 < tol
        (_linear_solver.py:6-42), run by the device PCG kernels without preconditioner."""
        from .plan import vptr, stream
        import ctypes as C
        b = torch.as_tensor(b, dtype=torch.float64)
        dev = b.device if b.is_cuda else torch.device("cuda")
        b = b.to(dev).contiguous()
        n = b.shape[0]
        A = torch.sparse_coo_tensor(A_indices.to(dev), A_values.to(dev, torch.float64), (n, n)).coalesce()
        Ac = A.to_sparse_csr()
        ip = Ac.crow_indices().to(torch.int64).contiguous()
        ix = Ac.col_indices().to(torch.int32).contiguous()
        vv = Ac.values().contiguous()
        x = torch.zeros_like(b) if (x0 is None or x0.numel() == 0) else x0.to(dev, torch.float64).clone().contiguous()
        w = torch.empty(L.fea_pcg_work_len(n), dtype=torch.float64, device=dev)
        it, rr = C.c_int32(0), C.c_double(0.0)
        st = L.fea_pcg_solve(n, vptr(ip), vptr(ix), vptr(vv), vptr(b), vptr(x), float(tol), int(max_iter), 20, 0,
                             vptr(w), w.numel(), C.byref(it), C.byref(rr), stream())
        if st not in (L.FEA_OK, L.FEA_ENOTCONV):
            L.check(st, "conjugate_gradient")
        return x


_linear_solver = _LinearSolverModule()
