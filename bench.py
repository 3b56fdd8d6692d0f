#!/usr/bin/env python
"""Element residual + tangent + reduced-CSR assembly throughput (GElem/s).

Workload (one GPU): a 64^3 C3D8 block on [0,1]^3, nodes jittered by
U(-0.1h, 0.1h) (seed 0), compressible Neo-Hookean mu = 1, kappa = 50, the
x = 0 face clamped, follower pressure p = 0.02 on the x = 1 face (Q4, the
reference's Pressure load convention);
262,144 elements, 274,625 nodes, 811,200 free DOFs, 63,695,790 nonzeros.
One step = one full assembly of the reduced residual R and tangent K at a
seeded displacement state (all element groups and the pressure load), i.e.
what the Newton solver does per iteration.  The K values (510 MB) exceed the
126 MB L2, so no flush is needed between steps.

`value` is device-timed (inputs resident in HBM).  `e2e` goes through the
public API ``Assembly.assemble_Stiffness_Matrix`` with the displacement
copied from pinned host memory and the residual read back every step.
Under torchrun (N > 1) every rank assembles its own block (weak scaling,
no collective in the data path); times are the max over ranks.

``--impl reference`` times the CPU restatement of the reference algorithm
(oracle/, in the reference's own output form) on the same full mesh with all
host threads; that process never imports fea_b200.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "elem tangent+assembly GElem/s"
PRESSURE = 0.02
UNIT = "GElem/s"


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="fea_b200", choices=["fea_b200", "reference"])
    ap.add_argument("--n", type=int, default=64, help="elements per side of the C3D8 block")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--workload", default="assembly", choices=["assembly", "pcg", "explicit", "newton", "adjoint", "serving", "newmark", "pcgb"],
                    help="assembly (default, the headline line) or one of the other measured forms")
    ap.add_argument("--explicit-n", type=int, default=70, help="cells per side of the Kuhn-tet cube")
    ap.add_argument("--explicit-steps", type=int, default=10000)
    ap.add_argument("--pcg-max-iter", type=int, default=50000, help="iteration cap of each PCG solve")
    ap.add_argument("--adjoint-n", type=int, default=40, help="elements per side of the compliance block")
    ap.add_argument("--pcgb-slots", type=int, default=24)
    ap.add_argument("--pcgb-rounds", type=int, default=10)
    ap.add_argument("--newmark-n", type=int, default=48, help="elements per side of the Newmark block")
    ap.add_argument("--newmark-dt", type=float, default=0.01)
    ap.add_argument("--newmark-steps", type=int, default=10)
    ap.add_argument("--fd-samples", type=int, default=200, help="coordinates checked by central differences")
    ap.add_argument("--serve-requests", type=int, default=512)
    ap.add_argument("--serve-rates", default="inf", help="comma-separated Poisson arrival rates (requests/s)")
    ap.add_argument("--serve-min-elems", type=int, default=2000)
    ap.add_argument("--serve-max-elems", type=int, default=200000)
    ap.add_argument("--serve-slots", type=int, default=48)
    ap.add_argument("--serve-round", type=int, default=32, help="PCG iterations per captured round")
    ap.add_argument("--serve-plain", type=int, default=1, help="also time the one-at-a-time path")
    ap.add_argument("--serve-sample", type=int, default=48,
                    help="requests of the serving record in the default line (0: none)")
    return ap.parse_args()


def workload(n):
    """Mesh, clamp set, pressure surface and state of the benchmark."""
    from fea_b200 import meshes
    X, el = meshes.hex_block(n, jitter=0.1, seed=0)
    E = el.shape[0]
    i_el = np.arange(E) // (n * n)
    end = np.nonzero(i_el == n - 1)[0]
    clamp = np.arange((n + 1) * (n + 1))           # node plane i = 0
    faces = el[end][:, [1, 2, 6, 5]]                # face 3 (x = max) of the end elements
    return X, el, clamp, end, faces


FP64_NOMINAL_TFLOPS = 37.0   # B200 FP64 (vector and tensor alike), NVIDIA's nominal figure


def fp64_roofline(E, B, hbm_gbs, kern_ms, nn=8, ng=8):
    """The assembly's flop side: F = E g (60 nn^2 + 108 nn + 300) FP64 flops
    for the full element tangent in the reference's formulation (1.05e10 at
    64^3), its rate over the volume kernels' time against the nominal FP64
    peak, and the combined roofline max(B / BW, F / FP64) of the two bounds."""
    F = float(E) * ng * (60 * nn * nn + 108 * nn + 300)
    t = kern_ms * 1e-3
    t_hbm = B / (hbm_gbs * 1e9)
    t_fp64 = F / (FP64_NOMINAL_TFLOPS * 1e12)
    return {"bound": "fp64", "flops": F, "achieved_tflops": F / t / 1e12, "peak_tflops": FP64_NOMINAL_TFLOPS,
            "frac": F / t / 1e12 / FP64_NOMINAL_TFLOPS,
            "peak_source": "nominal B200 FP64 (no measured FP64 peak on this pool)",
            "combined_roofline_ms": 1e3 * max(t_hbm, t_fp64), "combined_frac": max(t_hbm, t_fp64) / t}


def algorithmic_bytes(E, nn, nnz, N, n):
    """Per-assembly algorithmic bytes: connectivity, the reference's int32
    element-to-slot map, K values, coordinates + displacement, residual."""
    return E * 4 * nn + E * 4 * (3 * nn) ** 2 + 8 * nnz + 48 * N + 8 * n


def dist_barrier(world):
    """Barrier across the ranks (no-op on one rank)."""
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def dist_max(x, world, device):
    """Max of a per-rank time over all ranks (the job finishes with its slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def job_rate(world, units_per_rank, ms):
    """Whole-job throughput in G units/s: every rank processes its own units
    (weak scaling) in the max-over-ranks time ms."""
    return world * units_per_rank / (ms * 1e-3) / 1e9


def sample_clocks(stop, out, dev):
    cmd = ["nvidia-smi", "-i", str(dev), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
           "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "100"]
    try:
        p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return
    def reader():
        for line in p.stdout:
            out.append(line.strip())
    t = threading.Thread(target=reader, daemon=True)
    t.start()
    stop.wait()
    p.terminate()
    try:
        p.wait(timeout=5)
    except subprocess.TimeoutExpired:
        p.kill()
    t.join(timeout=2)


def summarize_clocks(lines):
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        f = [x.strip() for x in ln.split(",")]
        if len(f) < 8:
            continue
        try:
            sm.append(float(f[0]))
            mx = float(f[1])
        except ValueError:
            continue
        for nm, v in zip(names, f[4:8]):
            if v.lower().startswith("active"):
                reasons.add(nm)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def reference_workload(n):
    """The benchmark's mesh, clamp set and pressure faces built with the
    oracle's own generator, so that a process that times the reference
    algorithm never imports fea_b200 (nor maps its library).  The same X and
    connectivity as ``workload`` (checked by a CPU test)."""
    import torch
    from oracle import fea_oracle as O
    X, el = O.hex_block(n, jitter=0.1, seed=0)
    E = el.shape[0]
    end = torch.nonzero(torch.arange(E) // (n * n) == n - 1).flatten()
    clamp = torch.arange((n + 1) * (n + 1))            # node plane i = 0
    faces = el[end][:, [1, 2, 6, 5]]                   # face 3 (x = max) of the end elements
    return X, el, clamp, faces


class ReferenceAssembly:
    """One step of the reference arm: ``Assembly.assemble_Stiffness_Matrix``
    on the full benchmark mesh in the reference's own form (element R and K,
    slot scatter, the pressure load, Dirichlet mask and ``unique`` relabel
    into an uncoalesced reduced COO; assembly.py:283-387), run by the oracle
    on the host cores with all threads.  Set-up (mesh, element pattern and
    slot map: the reference's ``initialize``) happens once, outside the
    timed steps."""

    def __init__(self, n):
        import torch
        from oracle import fea_oracle as O
        torch.set_num_threads(os.cpu_count() or 1)
        X, el, clamp, faces = reference_workload(n)
        self.model = O.Model(X, [O.Group("C3D8", el, 1.0, 50.0)], [O.PressureLoad(faces, PRESSURE)],
                             [(clamp, (0, 1, 2))])
        free = self.model.free_mask()
        self.pattern = [O.element_pattern(el)]
        idx = self.pattern[0][0]
        self.E, self.N = int(el.shape[0]), int(X.shape[0])
        self.ndof = int(free.sum())
        self.nnz = int((free[idx[0]] & free[idx[1]]).sum())   # pressure pairs lie inside elements
        self.gc = 1e-3 * torch.randn(self.ndof, generator=torch.Generator().manual_seed(0), dtype=torch.float64)
        self.threads = torch.get_num_threads()

    def step(self):
        return self.model.stiffness_coo(self.gc, self.pattern)


def bench_config(n, E, N, ndof, nnz, world):
    """The ``config`` of the headline line, identical for both arms."""
    return {"workload": "c3d8_%dcube_jitter_neohookean_assembly" % n, "elements": E, "nodes": N,
            "ndof": ndof, "nnz": nnz, "parallelism": "replica per GPU" if world > 1 else "single GPU",
            "l2": "K values %.0f MB > 126 MB L2, no flush" % (8 * nnz / 1e6)}


def cpu_baseline(n):
    """The reference arm's step, timed once after one untimed step, on the
    whole benchmark mesh (about 10-30 s of host work with set-up)."""
    ref = ReferenceAssembly(n)
    ref.step()
    t0 = time.perf_counter()
    ref.step()
    dt = time.perf_counter() - t0
    return {"value": ref.E / dt / 1e9, "unit": UNIT, "cores": ref.threads, "kind": "port",
            "sample": "one full assemble_Stiffness_Matrix step of the same %d-element mesh in the reference's "
                      "form (R + K + slot scatter + pressure + Dirichlet mask + unique relabel), after one "
                      "untimed step; %.2f s; %s" % (ref.E, dt, cpu_model())}


def cpu_model():
    """The host CPU's model name (first processor in /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.lower().startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown CPU"


def _timed_difference(run, seconds, cap):
    """Time `run(k)`, which returns (seconds, units done), at k = 1 and
    k = 1 + m, m sized from the first call so that the second takes about
    `seconds`: per-unit time with the set-up of each call cancelled (after
    one untimed call that warms the thread pool and caches).  Returns
    (seconds per unit, units timed, seconds of the long call)."""
    run(1)
    t1, u1 = run(1)
    m = max(2, min(cap, int(seconds / max(t1 / 2, 1e-6))))
    t2, u2 = run(1 + m)
    return max(t2 - t1, 1e-9) / max(u2 - u1, 1), u2 - u1, t2


def cpu_cg_iteration(indptr, indices, values, b, seconds):
    """Oracle port of the reference's conjugate_gradient on the same reduced
    system, on the host cores: time per iteration."""
    import torch
    from oracle import fea_oracle as O
    torch.set_num_threads(os.cpu_count() or 1)
    ip, ix, v, bb = indptr.cpu(), indices.cpu().to(torch.int64), values.cpu(), b.cpu()

    def run(k):
        # the stop test only ends a run whose residual would otherwise reach
        # denormal values, which are slow on the host and not the reference's cost
        t = time.perf_counter()
        _, it = O.conjugate_gradient(ip, ix, v, bb, tol=1e-30, max_iter=k)
        return time.perf_counter() - t, it

    per, m, total = _timed_difference(run, seconds, 2000)
    return {"value": per * 1e3, "unit": "ms per CG iteration", "cores": torch.get_num_threads(), "kind": "port",
            "sample": "%d iterations of the reference's CG (CSR SpMV + vector updates) on the same %d-row, "
                      "%d-nonzero system, minus a 1-iteration call; %.1f s; %s"
                      % (m, bb.shape[0], v.shape[0], total, cpu_model())}


def cpu_explicit_step(X, el, dt, seconds):
    """Oracle port of the reference's central-difference loop (lumped mass,
    residual-only element pass with the residual index precomputed) on the
    same mesh, on the host cores: time per step."""
    import torch
    from oracle import fea_oracle as O
    torch.set_num_threads(os.cpu_count() or 1)
    m = O.Model(torch.from_numpy(np.asarray(X)), [O.Group("C3D4", torch.from_numpy(np.asarray(el)), 1.0, 10.0, 1.0)],
                [], [])
    n = int(m.free_mask().sum())
    gc0 = torch.zeros(n, dtype=torch.float64)
    gv0 = 0.01 * torch.randn(n, generator=torch.Generator().manual_seed(0), dtype=torch.float64)

    def run(k):
        t = time.perf_counter()
        O.explicit_run(m, gc0, gv0, dt, k)
        return time.perf_counter() - t, k

    per, steps, total = _timed_difference(run, seconds, 50)
    return {"value": 1.0 / per, "unit": "steps/s", "cores": torch.get_num_threads(), "kind": "port",
            "sample": "%d steps of the reference's loop on the same %d-element mesh, minus a 1-step run "
                      "(lumped mass and first force pass cancel); %.1f s; %s" % (steps, len(el), total, cpu_model())}


def run_reference(a):
    """The reference arm: rank 0 times W + K full steps of the reference
    algorithm (``ReferenceAssembly``) on the benchmark mesh and prints the
    headline line with ``impl: reference``; other ranks exit without work.
    This process never imports fea_b200."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ref = ReferenceAssembly(a.n)
    for _ in range(a.warmup):
        ref.step()
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        ref.step()
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    v = ref.E / (ms * 1e-3) / 1e9
    cb = {"value": v, "unit": UNIT, "cores": ref.threads, "kind": "port",
          "sample": "%d full assemble_Stiffness_Matrix steps of the same %d-element mesh in the reference's form "
                    "(R + K + slot scatter + pressure + Dirichlet mask + unique relabel), %.1f s timed, after %d "
                    "untimed; %s" % (a.steps, ref.E, sum(times), a.warmup, cpu_model())}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(a.n, ref.E, ref.N, ref.ndof, ref.nnz, a.gpus),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def build_block_model(n, p=0.02, rho=None):
    import fea_b200 as F
    X, el, clamp, end, faces = workload(n)
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=np.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 50.0))
    if rho is not None:
        e.set_density(rho)
    part.add_element(e)
    part.set_nodes["clamp"] = clamp
    part.add_surface_set("end", [(end, 3)])
    asm = F.Assembly()
    asm.add_part(part, "block")
    asm.add_instance(F.Instance(part), "block")
    load = F.loads.Pressure("block", "end", p)
    asm.add_load(load, "traction")
    asm.add_boundary(F.boundarys.Boundary_Condition("block", "clamp"), "clamp")
    asm.initialize()
    return asm, el, X, load


def run_pcg(a):
    """FP64 Jacobi-PCG (node-row and plain-CSR SpMV) and FP32-SpMV inner CG
    with FP64 refinement on the reduced 64^3 system K(u0) x = -R(u0) at the
    initial state, to a relative residual of 1e-8 (squared scaled ratio
    1e-16); errors against an FP64 solve converged to 1e-12."""
    import torch
    asm, el, X, _ = build_block_model(a.n)
    P = asm.plan
    R, K = asm.assemble_csr(asm.GC)
    b = (-R).contiguous()
    xref = torch.zeros_like(b)
    it_ref, rr_ref, _ = P.pcg(K, b, xref, 1e-24, a.pcg_max_iter, check_every=50)
    K32 = P.to_f32(K)
    P.fill_f32(K)                                    # builds the padded layout's column lists once
    out = {}
    for mode in ("fp64", "fp64_csr", "mixed", "mixed_plan_layout", "mixed_inner_tol"):
        x = torch.zeros_like(b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if mode == "mixed":                          # padded FP32 layout (values converted inside)
            it, outer, rr, st = P.pcg_mixed(K, None, b, x, 1e-16, 0.0, a.pcg_max_iter, check_every=50)
        elif mode == "mixed_inner_tol":
            it, outer, rr, st = P.pcg_mixed(K, None, b, x, 1e-16, 1e-4, a.pcg_max_iter, check_every=50)
        elif mode == "mixed_plan_layout":
            it, outer, rr, st = P.pcg_mixed(K, K32, b, x, 1e-16, 0.0, a.pcg_max_iter, check_every=50)
        else:
            it, rr, st = P.pcg(K, b, x, 1e-16, a.pcg_max_iter, check_every=50, generic=(mode == "fp64_csr"))
            outer = 1
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        r = b - P.spmv(K, x)
        out[mode] = {"iterations": it, "outer": outer, "ms": ms, "ms_per_iter": ms / max(it, 1),
                     "relres": float(r.norm() / b.norm()),
                     "err_vs_fp64_1e-12": float((x - xref).norm() / xref.norm()), "status": st}
    nnz, n = P.nnz, P.ndof
    act = P.mask != 0
    idx_bytes = 4 * int(P.rowlen[act].to(torch.int64).sum())
    # per iteration: values + column lists once per node + 13 FP64 vector passes
    bytes64 = 8 * nnz + idx_bytes + 8 * 13 * n
    bytes64_csr = 12 * nnz + 8 * (n + 1) + 8 * 13 * n
    bytes32 = 4 * nnz + idx_bytes + 56 * n
    line = {"metric": "PCG time to relres 1e-8 (64^3 C3D8 reduced system)", "unit": "ms",
            "value": out["mixed"]["ms"], "higher_is_better": False, "workload": "pcg", "dtype": "f64/f32",
            "n": n, "nnz": nnz, **out, "mixed_vs_fp64_per_iter": out["mixed"]["ms_per_iter"] / out["fp64"]["ms_per_iter"],
            "reference_iterations": it_ref,
            "iteration_bytes": {"fp64": bytes64, "fp64_csr": bytes64_csr, "fp32_inner": bytes32},
            "achieved_GBs": {"fp64": bytes64 / (out["fp64"]["ms_per_iter"] * 1e-3) / 1e9,
                             "fp64_csr": bytes64_csr / (out["fp64_csr"]["ms_per_iter"] * 1e-3) / 1e9,
                             "mixed": bytes32 / (out["mixed"]["ms_per_iter"] * 1e-3) / 1e9}}
    if not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_cg_iteration(P.indptr, P.indices, K, b, a.cpu_seconds)
    print(json.dumps(line), flush=True)


def run_explicit(a):
    """2.06M-tet cube (70^3 cells, 6 tets each), rho = 1, mu = 1, kappa = 10,
    no boundary conditions, v0 ~ N(0, 0.01^2) per DOF (seed 0), dt = 0.5 x
    min(altitude)/c, c = sqrt((kappa + 4 mu / 3) / rho); FP64 and FP32
    element force (FP64 sums), energy drift and displacement difference."""
    import torch
    import fea_b200 as F
    from fea_b200 import meshes
    X, el = meshes.tet_block(a.explicit_n)
    part = F.Part(X)
    e = F.elements.C3D4(elems=el, elems_index=np.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 10.0))
    e.set_density(1.0)
    part.add_element(e)
    asm = F.Assembly()
    asm.add_part(part, "cube")
    asm.add_instance(F.Instance(part), "cube")
    asm.initialize()
    P = asm.plan
    minv = asm.lumped_mass_inv()
    m = 1.0 / minv
    sol = F.solver.DynamicExplicitSolver()
    sol.assembly = asm
    dt = sol.cfl_timestep(0.5)
    v0 = (0.01 * torch.randn(P.ndof, generator=torch.Generator().manual_seed(0), dtype=torch.float64)).cuda()
    eb = torch.zeros(1, dtype=torch.float64, device="cuda")

    def energy(u, v):
        P.energy_volume(0, 1.0, 10.0, u, eb)
        return float(0.5 * (m * v * v).sum() + eb[0])

    def shadow_energy(u, vh, acc):
        # 1/2 vh_{N+1/2} M vh_{N-1/2} + W(u_N): the quantity central
        # differences conserve without the O((w dt)^2) oscillation of the
        # synchronous kinetic energy of the high-frequency modes
        P.energy_volume(0, 1.0, 10.0, u, eb)
        return float(0.5 * (m * (vh + dt * acc) * vh).sum() + eb[0])

    res = {}
    for fp32 in (False, True):
        u = torch.zeros(P.ndof, dtype=torch.float64, device="cuda")
        v = v0.clone()
        vh = torch.empty_like(u)
        acc = torch.empty_like(u)
        P.explicit_run(0, 1.0, 10.0, minv, dt, 0, u, vh, acc, v, fp32=fp32, init=True)
        E0 = energy(u, v0)
        S0 = shadow_energy(u, vh, acc)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        P.explicit_run(0, 1.0, 10.0, minv, dt, a.explicit_steps, u, vh, acc, v, fp32=fp32, init=False)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        E1 = energy(u, vh + 0.5 * dt * acc)          # v_N = vh_{N-1/2} + dt/2 a_N
        S1 = shadow_energy(u, vh, acc)
        res["fp32" if fp32 else "fp64"] = {"ms_total": ms, "ms_per_step": ms / a.explicit_steps,
                                           "energy_0": S0, "energy_end": S1, "energy_drift": (S1 - S0) / S0,
                                           "sync_energy_change": (E1 - E0) / E0, "u": u}
    du = float((res["fp32"]["u"] - res["fp64"]["u"]).norm() / res["fp64"]["u"].norm())
    for k in res:
        res[k].pop("u")
    E, N = el.shape[0], X.shape[0]
    line = {"metric": "explicit central-difference steps/s (2.06M C3D4)", "unit": "steps/s",
            "value": 1e3 / res["fp64"]["ms_per_step"], "higher_is_better": True, "workload": "explicit",
            "elements": E, "nodes": N, "steps": a.explicit_steps, "dt": dt, "fp64": res["fp64"],
            "fp32": res["fp32"], "fp32_vs_fp64_disp_rel": du,
            "elements_per_s": E * 1e3 / res["fp64"]["ms_per_step"]}
    if not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_explicit_step(X, el, dt, a.cpu_seconds)
    print(json.dumps(line), flush=True)


def run_newton(a):
    """Full static Newton solve of the 64^3 block to 1e-8 relative residual."""
    import torch
    import fea_b200 as F
    asm, el, X, _ = build_block_model(a.n)
    gc0 = asm.GC.clone()
    out = {}
    for prec in ("fp64", "mixed"):
        sol = F.solver.StaticImplicitSolver(rtol=1e-8, maximum_iteration=100, precision=prec)
        sol.initialize(asm)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gc = sol.solve(GC0=gc0.clone())
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if isinstance(gc, bool):
            print(json.dumps({"newton_failed": prec, "history": sol.history}), flush=True)
            raise RuntimeError("Newton solve (%s) failed" % prec)
        R = asm.assemble_force(GC=gc)
        out[prec] = {"seconds": dt, "newton_iters": len(sol.history), "history": sol.history, "gc": gc,
                     "pcg_iters_total": sum(h.get("pcg_iters", 0) for h in sol.history),
                     "final_rel_residual": float(R.norm()) / sol.history[0]["rnorm"]}
    d = float((out["mixed"]["gc"] - out["fp64"]["gc"]).norm() / out["fp64"]["gc"].norm())
    for k in out:
        out[k].pop("gc")
    line = {"metric": "static Newton solve to 1e-8 (64^3 C3D8)", "unit": "s", "value": out["fp64"]["seconds"],
            "higher_is_better": False, "workload": "newton", "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_vs_fp64_disp_rel": d}
    print(json.dumps(line), flush=True)


def run_newmark(a):
    """Implicit Newmark dynamics (DynamicImplicitSolver) of the jittered n^3
    C3D8 block, rho = 1, clamped at x = 0, pressure 0.02 on x = 1 from t = 0,
    from rest: ``--newmark-steps`` steps of dt = ``--newmark-dt``, Newton to
    max|R| < 1e-11 per step."""
    import torch
    import fea_b200 as F
    # warm-up: three untimed steps on a model of its own (clocks, first
    # launches of every kernel, allocator pools)
    asm_w = build_block_model(a.newmark_n, rho=1.0)[0]
    sol_w = F.solver.DynamicImplicitSolver(deltaT=a.newmark_dt, time_end=3 * a.newmark_dt * (1 - 1e-9),
                                           tol_error=1e-11)
    sol_w.initialize(asm_w)
    sol_w.solve(GC0=torch.zeros_like(asm_w.GC))
    torch.cuda.synchronize()
    del sol_w, asm_w
    asm, el, X, _ = build_block_model(a.newmark_n, rho=1.0)
    sol = F.solver.DynamicImplicitSolver(deltaT=a.newmark_dt, time_end=a.newmark_steps * a.newmark_dt * (1 - 1e-9),
                                         tol_error=1e-11)
    sol.initialize(asm)
    gc0 = torch.zeros_like(asm.GC)
    newton, pcg = [], []
    orig = sol._solve_iteration

    def counted(*args, **kw):
        r = orig(*args, **kw)
        newton.append(sol._iter_now)
        pcg.append(sum(h.get("pcg_iters", 0) for h in sol.history))
        return r

    sol._solve_iteration = counted
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sol.solve(GC0=gc0)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    steps = len(sol._GC_list) - 1
    R = sol._incremental_csr(sol._GC_list[-1], sol._GC_list[-2] + a.newmark_dt * sol._GV_list[-2]
                             + 0.25 * a.newmark_dt ** 2 * sol._GA_list[-2])[0]
    line = {"metric": "implicit Newmark steps/s (%d^3 C3D8, dt %g)" % (a.newmark_n, a.newmark_dt),
            "unit": "steps/s", "value": steps / (ms * 1e-3), "higher_is_better": True, "workload": "newmark",
            "ms_per_step": ms / steps, "steps": steps, "elements": int(el.shape[0]), "ndof": int(asm.plan.ndof),
            "newton_iters_per_step": newton, "pcg_iters_per_step": pcg,
            "last_step_max_residual": float(R.abs().max()), "max_displacement": float(sol._GC_list[-1].abs().max()),
            "energy_history": sol.E_history, "timing": "CUDA events around solve(), initial acceleration included, after a three-step warm-up solve"}
    print(json.dumps(line), flush=True)


def run_pcgb(a):
    """Batched PCG kernels of the serving engine alone: ``--pcgb-slots``
    resident C3D4 cantilever systems (60k-120k elements, seeded, K at rest),
    PCG with a tolerance no slot reaches in the timed rounds; device time per
    batched iteration (CUDA events over ``--pcgb-rounds`` graph replays of 32
    iterations) and the bytes it streams (values, column lists once per
    node, 13 vector passes)."""
    import torch
    from fea_b200 import serving, solver as S
    reqs = serving.make_requests(a.pcgb_slots, float("inf"), seed=1, min_elems=60000, max_elems=120000)
    asms, lins, works = [], [], []
    for r in reqs:
        asm = serving.build_assembly(r)
        R, K = asm.assemble_csr(asm.GC)
        b = (-R).contiguous()
        lins.append(S.LinearSolve(K, b, torch.zeros_like(b), 1e-300, 10 ** 8, False))
        asms.append(asm)
    max_items = a.pcgb_slots * max((serving.request_rows(r) // 3 + 15) // 16 + 1 for r in reqs)
    eng = serving.BatchedPCG(a.pcgb_slots, max_items, 32, True)
    for k, (asm, lin) in enumerate(zip(asms, lins)):
        w = torch.empty(serving.BatchedPCG.work_len(asm.plan), dtype=torch.float64, device="cuda")
        works.append(w)
        eng.assign(k, asm.plan, lin, w)
    eng.sync()
    for k in range(a.pcgb_slots):
        eng.start(k)
    for _ in range(3):
        eng.run_round()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.pcgb_rounds):
        eng.run_round()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / (a.pcgb_rounds * 32)
    active = int((eng.poll()[:, 0] == 0).sum())
    nnz = sum(x.plan.nnz for x in asms)
    n = sum(x.plan.ndof for x in asms)
    idx = sum(int(x.plan.rowlen[x.plan.mask != 0].to(torch.int64).sum()) for x in asms)
    byt = 8 * nnz + 4 * idx + 8 * 13 * n
    print(json.dumps({"metric": "batched PCG iteration (%d resident C3D4 slots)" % a.pcgb_slots, "unit": "ms",
                      "value": ms, "higher_is_better": False, "workload": "pcgb", "slots_active": active,
                      "ndof_total": n, "nnz_total": nnz, "bytes_per_iter": byt,
                      "achieved_GBs": byt / (ms * 1e-3) / 1e9}), flush=True)


def run_adjoint(a):
    """Compliance f.u of an n^3 C3D8 block (nodes jittered as in the assembly
    workload, mu = 1, kappa = 50, bottom node plane clamped, pressure 0.03 on
    the top faces): gradients w.r.t. all
    nodal coordinates and mu from the hand-written adjoint behind
    ComplianceFunction; checked against central differences (h = 1e-6) on
    seeded random coordinates and against torch autograd of the oracle's
    residual (lam . dR/dX)."""
    import torch
    import fea_b200 as F
    from fea_b200 import adjoint, meshes
    from oracle import fea_oracle as O
    n = a.adjoint_n
    X, el = meshes.hex_block(n, jitter=0.1, seed=0)
    E, N = el.shape[0], X.shape[0]
    top = np.nonzero(np.arange(E) % n == n - 1)[0]
    clamp = np.nonzero(np.arange(N) % (n + 1) == 0)[0]
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=np.arange(E), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 50.0))
    part.add_element(e)
    part.set_nodes["bottom"] = clamp
    part.add_surface_set("top", [(top, 1)])
    asm = F.Assembly()
    asm.add_part(part, "block")
    asm.add_instance(F.Instance(part), "block")
    asm.add_load(F.loads.Pressure("block", "top", 0.03), "pressure")
    asm.add_boundary(F.boundarys.Boundary_Condition("block", "bottom"), "clamp")
    asm.initialize()
    solver = F.solver.StaticImplicitSolver(rtol=1e-12, maximum_iteration=80)
    solver.initialize(asm)
    # forward solve + adjoint through the autograd Function
    Xt = torch.from_numpy(X).clone().requires_grad_(True)
    mu = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    C = adjoint.ComplianceFunction.apply(Xt, mu, asm, solver)
    C.backward()
    torch.cuda.synchronize()
    t_full = time.perf_counter() - t0
    newton_iters = len(solver.history)
    gstar = asm.GC.clone()
    # adjoint gradient alone at the equilibrium (adjoint PCG + VJP kernels)
    reps = 5
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        Cg, dX, dmu, it_adj, lam = adjoint.compliance_gradient(asm, gstar, return_lambda=True)
    torch.cuda.synchronize()
    t_grad = (time.perf_counter() - t0) / reps
    gX = dX.cpu()
    scale = float(gX.abs().max())
    # central differences, warm-started from the equilibrium
    def comp(Xn, mu_v=1.0):
        adjoint.set_coordinates(asm, Xn)
        asm._mat_elems[0].materials.mu = torch.tensor(mu_v, dtype=torch.float64)
        gc = solver.solve(GC0=gstar.clone())
        if isinstance(gc, bool):
            raise RuntimeError("equilibrium solve failed")
        return float(torch.dot(adjoint.external_force(asm, gc), gc))
    h = 1e-6
    rng = np.random.default_rng(0)
    free_nodes = np.setdiff1d(np.arange(N), clamp)
    nodes = rng.choice(free_nodes, size=a.fd_samples, replace=False)
    comps = rng.integers(0, 3, size=a.fd_samples)
    X0 = torch.from_numpy(X).clone()
    errs, raw = [], []
    t0 = time.perf_counter()
    for nd, k in zip(nodes, comps):
        Xp = X0.clone(); Xp[nd, k] += h
        Xm = X0.clone(); Xm[nd, k] -= h
        fd = (comp(Xp) - comp(Xm)) / (2 * h)
        ad = float(gX[nd, k])
        errs.append(abs(fd - ad) / max(abs(ad), 1e-2 * scale))
        if abs(ad) >= 1e-2 * scale:
            raw.append(abs(fd - ad) / abs(ad))
    fd_mu = (comp(X0, 1.0 + h) - comp(X0, 1.0 - h)) / (2 * h)
    t_fd = time.perf_counter() - t0
    comp(X0, 1.0)
    # lam . dR/dX of the kernels against torch autograd of the oracle residual
    dXk, _ = adjoint.residual_vjp(asm, gstar, lam)
    Xo = torch.from_numpy(X).clone().requires_grad_(True)
    faces = torch.from_numpy(el[top][:, [4, 5, 6, 7]])
    m = O.Model(Xo, [O.Group("C3D8", torch.from_numpy(el), 1.0, 50.0)], [O.PressureLoad(faces, 0.03)],
                [(clamp, (0, 1, 2))])
    Ro, _ = m.assemble(gstar.cpu(), want_K=False)
    (Ro * lam.cpu()).sum().backward()
    auto_rel = float((dXk.cpu() - Xo.grad).norm() / Xo.grad.norm())
    line = {"metric": "compliance gradient evals/s (%d^3 C3D8, dC/dX all nodes + dC/dmu)" % n,
            "value": 1.0 / t_grad, "unit": "evals/s", "higher_is_better": True, "workload": "adjoint",
            "elements": E, "ndof": asm.plan.ndof, "compliance": float(Cg),
            "gradient_s": t_grad, "adjoint_pcg_iters": it_adj,
            "forward_plus_backward_s": t_full, "forward_newton_iters": newton_iters,
            "fd_samples": int(a.fd_samples), "fd_step": h, "fd_seconds": t_fd,
            "fd_max_rel_err": max(errs), "fd_max_rel_err_components_above_1pct": max(raw) if raw else None,
            "fd_components_above_1pct": len(raw),
            "dmu_adjoint": float(dmu[0]), "dmu_fd": fd_mu, "dmu_rel_err": abs(fd_mu - float(dmu[0])) / abs(float(dmu[0])),
            "vjp_vs_oracle_autograd_rel": auto_rel}
    print(json.dumps(line), flush=True)


def serving_run(n_requests, rate, slots, round_iters, min_elems, max_elems, plain=True, seed=0):
    """One stream of seeded cantilever static solves (C3D4, Newton to 1e-8):
    solves/s and p50/p99 latency of the continuous-batching server, and of
    the same requests solved one at a time through StaticImplicitSolver."""
    import torch
    from fea_b200 import serving
    reqs = serving.make_requests(n_requests, rate, seed=seed, min_elems=min_elems, max_elems=max_elems)
    if not math.isfinite(rate):
        for r in reqs:
            r.arrival = 0.0

    def summary(res, wall):
        ok = [r for r in res if r.error is None]
        lat = np.array([r.latency for r in ok])
        span = max(r.done for r in res) - min(r.arrival for r in res)
        return {"solves_per_s": len(ok) / span, "rejected": len(res) - len(ok), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "makespan_s": span, "wall_s": wall,
                "newton_iters": int(sum(r.newton_iters for r in res)), "pcg_iters": int(sum(r.pcg_iters for r in res))}
    # warm-up: one small request through both paths
    w = serving.make_requests(1, float("inf"), seed=99, min_elems=2000, max_elems=2000)
    w[0].arrival = 0.0
    serving.serve(w, max_slots=slots, round_iters=round_iters, keep=False)
    serving.solve_plain(w, keep=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    served, stats = serving.serve(reqs, max_slots=slots, round_iters=round_iters)
    rec = {"rate_per_s": rate, "served": summary(served, time.perf_counter() - t0), "server": stats}
    if plain:
        t0 = time.perf_counter()
        plain_res = serving.solve_plain(reqs)
        rec["plain"] = summary(plain_res, time.perf_counter() - t0)
        rec["speedup_solves_per_s"] = rec["served"]["solves_per_s"] / rec["plain"]["solves_per_s"]
        rec["max_rel_diff_served_vs_plain"] = max(float((x.gc - y.gc).norm() / y.gc.norm())
                                                  for x, y in zip(served, plain_res)
                                                  if x.gc is not None and y.gc is not None)
    return rec


def run_serving(a):
    """The serving workload at every rate of --serve-rates."""
    out = [serving_run(a.serve_requests, float(x), a.serve_slots, a.serve_round, a.serve_min_elems,
                       a.serve_max_elems, plain=bool(a.serve_plain)) for x in a.serve_rates.split(",")]
    line = {"metric": "served static solves/s (C3D4 cantilevers, Newton to 1e-8)", "unit": "solves/s",
            "value": out[0]["served"]["solves_per_s"], "higher_is_better": True, "workload": "serving",
            "requests": a.serve_requests, "elems": [a.serve_min_elems, a.serve_max_elems], "runs": out}
    print(json.dumps(line), flush=True)


def main():
    a = args_()
    if a.impl == "reference":
        run_reference(a)
        return
    if a.workload != "assembly":
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        {"pcg": run_pcg, "explicit": run_explicit, "newton": run_newton, "adjoint": run_adjoint,
         "serving": run_serving, "newmark": run_newmark, "pcgb": run_pcgb}[a.workload](a)
        return
    import torch
    import torch.distributed as dist
    import fea_b200 as F
    from fea_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    X, el, clamp, end, faces = workload(a.n)
    n = a.n
    part = F.Part(X)
    e = F.elements.C3D8(elems=el, elems_index=np.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(1.0, 50.0))
    part.add_element(e)
    part.set_nodes["clamp"] = clamp
    part.add_surface_set("end", [(end, 3)])
    asm = F.Assembly()
    asm.add_part(part, "block")
    asm.add_instance(F.Instance(part), "block")
    asm.add_load(F.loads.Pressure("block", "end", PRESSURE), "traction")
    asm.add_boundary(F.boundarys.Boundary_Condition("block", "clamp"), "clamp")
    asm.initialize()
    P = asm.plan
    E, N, ndof, nnz = el.shape[0], X.shape[0], P.ndof, P.nnz
    gc = (1e-3 * torch.randn(ndof, generator=torch.Generator().manual_seed(0), dtype=torch.float64)).cuda()
    K = torch.empty(nnz, dtype=torch.float64, device="cuda")
    R = torch.empty(ndof, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def barrier():
        dist_barrier(world)

    def max_over_ranks(x):
        return dist_max(x, world, "cuda")

    # element kernel timed live: events around the volume kernel of every step
    mu, kappa = 1.0, 50.0

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        P.assemble_volume(0, mu, kappa, gc, K=K, R=R)
        if ev is not None:
            ev[1].record(stream)
        P.assemble_pressure(0, PRESSURE, asm._Xinst, gc, K=K, R=R)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    clocks_lines, stop = [], threading.Event()
    th = None
    if not a.no_clocks:
        th = threading.Thread(target=sample_clocks, args=(stop, clocks_lines, local), daemon=True)
        th.start()
        time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    l0 = _lib.fea_launch_count()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(a.steps):
        step(evs[k])
    t_end.record(stream)
    torch.cuda.synchronize()
    launches = _lib.fea_launch_count() - l0
    barrier()
    stop.set()
    if th is not None:
        th.join(timeout=10)
    ms = max_over_ranks(t_start.elapsed_time(t_end) / a.steps)
    kern_ms = statistics.mean(s.elapsed_time(t) for s, t in evs)
    value = job_rate(world, E, ms)

    # end to end through the public API, host buffers: every step copies its
    # displacement from pinned host memory and reads its residual back; the
    # copies run on a second stream, double-buffered, so that the next
    # step's upload and this step's download overlap the assembly
    gc_h = gc.cpu().pin_memory()
    r_h = [torch.empty(ndof, dtype=torch.float64).pin_memory() for _ in range(2)]
    gc_d = [torch.empty_like(gc) for _ in range(2)]
    copy = torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_used = [torch.cuda.Event() for _ in range(2)]

    def e2e_steps(nsteps):
        with torch.cuda.stream(copy):
            gc_d[0].copy_(gc_h, non_blocking=True)
            ev_in[0].record(copy)
        for k in range(nsteps):
            b = k % 2
            if k + 1 < nsteps:
                nb = (k + 1) % 2
                with torch.cuda.stream(copy):
                    if k >= 1:
                        copy.wait_event(ev_used[nb])       # step k-1 is done with gc_d[nb]
                    gc_d[nb].copy_(gc_h, non_blocking=True)
                    ev_in[nb].record(copy)
            stream.wait_event(ev_in[b])
            Rr, Ki, Kv = asm.assemble_Stiffness_Matrix(GC=gc_d[b])
            ev_used[b].record(stream)
            with torch.cuda.stream(copy):
                copy.wait_event(ev_used[b])
                r_h[b].copy_(Rr, non_blocking=True)
                Rr.record_stream(copy)
        stream.wait_stream(copy)

    e2e_steps(2)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_steps(a.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / a.steps)
    if not torch.equal(r_h[(a.steps - 1) % 2], asm.assemble_Stiffness_Matrix(GC=gc)[0].cpu()):
        raise RuntimeError("end-to-end residual differs from the device residual")
    barrier()

    B = algorithmic_bytes(E, 8, nnz, N, ndof)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = B / (kern_ms * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "c3d8_rk_traffic.json")
    if os.path.exists(tf):
        try:
            t = json.load(open(tf))
            traffic = float(t["bytes_per_element"]) * E
        except (OSError, KeyError, ValueError):
            traffic = None
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(n, E, N, ndof, nnz, world),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "algorithmic_bytes": B, "kernel_ms": kern_ms,
                     "kernel": "k_hex_elem + k_hex_gat (C3D8 element blocks staged block-major in per-node regions, then a node-row gather with transposed writes into CSR)",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650"},
        "roofline_fp64": fp64_roofline(E, B, hbm, kern_ms),
        "e2e": {"value": job_rate(world, E, e2e_ms), "unit": UNIT, "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": 8 * ndof, "d2h_bytes_per_step": 8 * ndof,
                "api": "Assembly.assemble_Stiffness_Matrix",
                "copies": "pinned host buffers; next step's upload and this step's download on a second "
                          "stream, double-buffered, overlapping the assembly"},
        "gpu_launches": int(launches),
        "clocks": summarize_clocks(clocks_lines),
    }
    if world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n)
    if world == 1 and a.serve_sample > 0:
        # the serving form on a seeded sample of the cantilever stream (all
        # requests at t = 0), served against one at a time on this GPU
        rec = serving_run(a.serve_sample, float("inf"), a.serve_slots, a.serve_round, a.serve_min_elems,
                          a.serve_max_elems)
        line["serving"] = {"requests": a.serve_sample, "arrivals": "all at t = 0", "elems": [a.serve_min_elems,
                           a.serve_max_elems], "sample": "first %d requests of the seeded 512-request stream "
                           "(seed 0)" % a.serve_sample, **rec}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
