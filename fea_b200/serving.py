"""Serving many static solves on one GPU with continuous batching.

A request is a static Newton solve of its own mesh (here: a C3D4 cantilever
with seeded dimensions, size and material, clamped at x = 1 - length and
loaded by a follower pressure on its free end x = 1).  The server

- prepares arriving requests on host threads (mesh, plan, device upload) as
  long as their estimated device memory fits the budget (by default a share
  of the device memory free when serving starts, torch.cuda.mem_get_info);
- keeps every admitted request's mesh, CSR pattern and Newton state resident
  and runs its Newton iteration as a generator
  (``StaticImplicitSolver._newton``), which stops at each tangent solve;
- packs the tangent solves of all admitted requests into one batched
  Jacobi-PCG (``fea_pcgb_*``): a fixed round of iterations over the chunk
  list of all active slots, captured once as a CUDA graph and replayed;
- after each round, resumes the Newton iteration of every slot whose solve
  finished (line search, next assembly) and admits new requests into free
  slots, so requests join and leave while others are on the device.

A slot's PCG arithmetic depends only on its own system, so a request's
result is the same bits whether it is served alone or among others.

The reference has no serving layer; its static solver handles one model at
a time (FEA/solver/static_implicit.py).  ``solve_plain`` is that path on
this GPU: one request after the other through ``StaticImplicitSolver``.
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import dataclasses
import math
import threading
import time

import numpy as np
import torch

from . import _lib as L
from ._trace import nvtx
from .plan import stream, vptr


@dataclasses.dataclass
class BeamRequest:
    rid: int
    length: float
    width: float
    height: float
    n_elems: int
    mu: float
    kappa: float
    pressure: float          # follower pressure on the free end
    arrival: float = 0.0     # seconds after the start of the stream


STABLE_LOAD = 25.0


def load_parameter(length, width, height, mu, kappa, pressure):
    """P L^2 / (E I) of a cantilever under end load P = pressure * w * h
    (E the small-strain Young's modulus of the Neo-Hookean pair, I the
    weaker second moment of the cross-section)."""
    E = 9.0 * kappa * mu / (3.0 * kappa + mu)
    I = min(width * height ** 3, height * width ** 3) / 12.0
    return pressure * width * height * length ** 2 / (E * I)


def make_requests(n, rate, seed=0, min_elems=2000, max_elems=200000):
    """n seeded cantilever requests with Poisson arrivals at `rate` per second:
    length U[4, 16], cross-section U[1, 2]^2, elements U[min, max], mu
    U[0.5, 2], kappa = 20 mu, end pressure U[0.005, 0.05] (the reference's
    Pressure sign: positive pushes on the face), redrawn while the load
    parameter P L^2 / (E I) exceeds STABLE_LOAD (25; seeded draws at 68 had
    an indefinite tangent at rest, none of 24 up to 31 had)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    while len(out) < n:
        L_, w, h = float(rng.uniform(4, 16)), float(rng.uniform(1, 2)), float(rng.uniform(1, 2))
        ne = int(rng.integers(min_elems, max_elems + 1))
        mu = float(rng.uniform(0.5, 2.0))
        p = float(rng.uniform(0.005, 0.05))
        # draws past the stable range of the enclosed-volume load model are
        # redrawn: there the tangent at rest is indefinite and no Newton
        # solve (the reference's direct solve included) converges
        if load_parameter(L_, w, h, mu, 20.0 * mu, p) > STABLE_LOAD:
            continue
        if rate and math.isfinite(rate):
            t += rng.exponential(1.0 / rate)
        out.append(BeamRequest(len(out), L_, w, h, ne, mu, 20.0 * mu, p, t))
    return out


def build_assembly(req: BeamRequest, device=None):
    """The request's model through the reference-mirroring API."""
    import fea_b200 as F
    from . import meshes
    X, el = meshes.tet_beam(req.length, req.width, req.height, req.n_elems)
    part = F.Part(X)
    e = F.elements.C3D4(elems=el, elems_index=np.arange(el.shape[0]), part=part)
    e.set_materials(F.materials.NeoHookean(req.mu, req.kappa))
    part.add_element(e)
    part.set_nodes["root"] = np.nonzero(np.abs(X[:, 0] - (1.0 - req.length)) < 1e-9)[0]
    sets, _ = meshes.plane_faces("C3D4", el, X, 0, 1.0)
    part.add_surface_set("tip", sets)
    asm = F.Assembly(device=device)
    asm.add_part(part, "beam")
    asm.add_instance(F.Instance(part), "beam")
    asm.add_load(F.loads.Pressure("beam", "tip", req.pressure), "tip")
    asm.add_boundary(F.boundarys.Boundary_Condition("beam", "root"), "root")
    asm.initialize()
    return asm


def make_solver(asm):
    import fea_b200 as F
    s = F.solver.StaticImplicitSolver(rtol=1e-8, maximum_iteration=100)
    s.initialize(asm)
    return s


def request_rows(req: BeamRequest):
    """Upper bound of the request's free DOFs (3 per node of its mesh)."""
    from .meshes import beam_dims
    nx, ny, nz = beam_dims(req.length, req.width, req.height, req.n_elems)
    return 3 * (nx + 1) * (ny + 1) * (nz + 1)


def estimate_bytes(req: BeamRequest):
    """Device memory of one admitted request: K values and column indices
    (about 45 per row), the plan's per-element and per-node arrays, Newton
    and PCG vectors."""
    rows = request_rows(req)
    return 12 * 45 * rows + 120 * req.n_elems + 200 * rows + (4 << 20)


@dataclasses.dataclass
class Result:
    rid: int
    gc: torch.Tensor         # None for a rejected request
    newton_iters: int
    pcg_iters: int
    arrival: float
    admitted: float
    done: float
    error: str = None        # why the request was rejected (its solve failed)

    @property
    def latency(self):
        return self.done - self.arrival


def solve_plain(requests, clock=None, keep=True):
    """One request after the other through StaticImplicitSolver (the plain
    GPU path), arrivals honoured: a request starts when it has arrived and
    the previous one has finished.  Returns results in request order."""
    t0 = time.perf_counter() if clock is None else clock
    out = []
    for req in sorted(requests, key=lambda r: r.arrival):
        now = time.perf_counter() - t0
        if now < req.arrival:
            time.sleep(req.arrival - now)
        start = time.perf_counter() - t0
        asm = sol = gc = None
        try:
            asm = build_assembly(req)
            sol = make_solver(asm)
            gc = sol.solve(GC0=asm.GC.clone())
            err = "Newton did not converge" if isinstance(gc, bool) else None
        except Exception as ex:              # the request is rejected; the others go on
            err = "%s: %s" % (type(ex).__name__, ex)
        torch.cuda.synchronize()
        done = time.perf_counter() - t0
        hist = sol.history if sol is not None else []
        out.append(Result(req.rid, gc.cpu() if (keep and err is None) else None, len(hist),
                          sum(h.get("pcg_iters", 0) for h in hist), req.arrival, start, done, err))
        del asm, sol, gc
    return sorted(out, key=lambda r: r.rid)


class BatchedPCG:
    """Device table and slots of the batched PCG (fea_pcgb_*)."""

    def __init__(self, max_slots, max_items, round_iters=32, use_graph=True, device=None):
        self.device = torch.device(device if device is not None else "cuda")
        self.max_slots, self.max_chunks = int(max_slots), int(max_items)
        nbytes = int(L.fea_pcgb_table_bytes(self.max_slots, self.max_chunks))
        self.table = torch.zeros((nbytes + 7) // 8, dtype=torch.float64, device=self.device)
        self.desc = (L.PcgbSlot * self.max_slots)()
        self.keep = [None] * self.max_slots
        self.state = torch.zeros(4 * self.max_slots, dtype=torch.float64, device=self.device)
        self.round_iters = int(round_iters)
        self.use_graph = use_graph
        self.graph = None
        self.rounds = 0
        self._dirty = True
        if use_graph:
            # one uncaptured round on the empty table sizes the launch grids,
            # then the round is captured once; replays read the live table
            self.sync()
            self._iterate()
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, capture_error_mode="thread_local"):
                self._iterate()
            self.graph = g

    def free_slots(self):
        return [k for k in range(self.max_slots) if self.keep[k] is None]

    @staticmethod
    def work_len(plan):
        """Work doubles of a slot on plan's matrix, node-row or CSR SpMV."""
        return int(max(L.fea_pcgb_work_len(plan.ndof, plan.n_nodes), L.fea_pcgb_work_len(plan.ndof, 0)))

    def assign(self, k, plan, lin, work, node_rows=True):
        """Slot k solves lin (a solver.LinearSolve) on plan's matrix; work: pcgb
        work buffer of work_len(plan) doubles.  node_rows: SpMV over the plan's
        node rows (else CSR rows)."""
        d = self.desc[k]
        d.n, d.nnz = plan.ndof, plan.nnz
        d.indptr_dev, d.indices_dev = plan.indptr.data_ptr(), plan.indices.data_ptr()
        d.values_dev, d.b_dev, d.x_dev = lin.K.data_ptr(), lin.b.data_ptr(), lin.x.data_ptr()
        d.work_dev, d.work_len = work.data_ptr(), work.numel()
        d.tol, d.max_iter, d.active = float(lin.tol), int(lin.cap), 1
        if node_rows:
            d.n_nodes = plan.n_nodes
            d.vbase_dev, d.rowlen_dev, d.dbase_dev = plan.vbase.data_ptr(), plan.rowlen.data_ptr(), plan.dbase.data_ptr()
            d.mask_dev = plan.mask.data_ptr()
        else:
            d.n_nodes = 0
            d.vbase_dev = d.rowlen_dev = d.dbase_dev = d.mask_dev = None
        self.keep[k] = (plan, lin, work)
        self._dirty = True

    def release(self, k):
        self.desc[k] = L.PcgbSlot()
        self.keep[k] = None
        self._dirty = True

    def sync(self):
        if self._dirty:
            L.check(L.fea_pcgb_set(vptr(self.table), self.max_slots, self.max_chunks, self.max_slots, self.desc,
                                   stream()), "fea_pcgb_set")
            self._dirty = False

    def start(self, k):
        d = self.desc[k]
        L.check(L.fea_pcgb_start(vptr(self.table), self.max_slots, self.max_chunks, k, d.n, d.nnz, stream()),
                "fea_pcgb_start")

    def _iterate(self):
        L.check(L.fea_pcgb_iterate(vptr(self.table), self.max_slots, self.max_chunks, self.round_iters, stream()),
                "fea_pcgb_iterate")

    def run_round(self):
        with nvtx("fea.pcgb_round"):
            self.sync()
            if self.graph is not None:
                self.graph.replay()
            else:
                self._iterate()
        self.rounds += 1

    def poll(self):
        L.check(L.fea_pcgb_state(vptr(self.table), self.max_slots, self.max_chunks, self.max_slots, vptr(self.state),
                                 stream()), "fea_pcgb_state")
        return self.state.view(-1, 4).cpu().numpy()

    def poll_async(self):
        """Queue the state copy behind the current round; wait() returns it."""
        if not hasattr(self, "_host_state"):
            self._host_state = torch.empty(4 * self.max_slots, dtype=torch.float64, pin_memory=True)
            self._ev = torch.cuda.Event()
        L.check(L.fea_pcgb_state(vptr(self.table), self.max_slots, self.max_chunks, self.max_slots, vptr(self.state),
                                 stream()), "fea_pcgb_state")
        self._host_state.copy_(self.state, non_blocking=True)
        self._ev.record()

    def wait(self):
        self._ev.synchronize()
        return self._host_state.view(-1, 4).numpy()


class _Job:
    __slots__ = ("req", "asm", "solver", "gen", "lin", "work", "slot", "admitted", "bytes")

    def __init__(self, req, asm, solver, admitted, nbytes):
        self.req, self.asm, self.solver = req, asm, solver
        self.gen = solver._newton(asm._gc(GC=asm.GC.clone()), solver.tol_error)
        self.lin, self.work, self.slot = None, None, None
        self.admitted, self.bytes = admitted, nbytes


def _prepare(req, stream_):
    with torch.cuda.stream(stream_):
        asm = build_assembly(req)
        sol = make_solver(asm)
    stream_.synchronize()
    return asm, sol


def admission_budget(fraction=0.8, reserve=2 << 30, device=None):
    """Bytes the server may hand to admitted requests: ``fraction`` of the
    device memory free now (torch.cuda.mem_get_info), less ``reserve`` for
    the batched-PCG table, graphs and the allocator's slack."""
    free, _ = torch.cuda.mem_get_info(device)
    return max(0, int(fraction * free) - int(reserve))


def serve(requests, max_slots=48, round_iters=32, mem_budget=None, use_graph=True, prep_threads=2,
          keep=True):
    """Serve `requests` (arrival times honoured) with continuous batching.
    ``mem_budget`` (bytes) defaults to ``admission_budget()``, measured on
    the device when serving starts.  Returns (results in request order,
    server statistics)."""
    dev = torch.device("cuda")
    if mem_budget is None:
        mem_budget = admission_budget(device=dev)
    # items of the largest admissible batch: SpMV items of 16 nodes (3 rows
    # per node at most) outnumber update items of 256 rows
    max_chunks = max_slots * (max((request_rows(r) // 3 + 15) // 16 + 1 for r in requests) if requests else 1)
    eng = BatchedPCG(max_slots, max_chunks, round_iters, use_graph, dev)
    waiting = sorted(requests, key=lambda r: r.arrival)
    prep_streams = [torch.cuda.Stream() for _ in range(prep_threads)]
    pool = cf.ThreadPoolExecutor(max_workers=prep_threads)
    free_streams = list(prep_streams)
    preparing, ready, queue_slot, results = {}, [], [], {}
    lock = threading.Lock()
    mem_used = 0
    t0 = time.perf_counter()
    busy_rounds = 0

    work_stream = torch.cuda.Stream()
    main = torch.cuda.current_stream()

    def finish(job, value, error=None):
        """Record the job's result (value: GC, or False when Newton failed)."""
        nonlocal mem_used
        if error is None and isinstance(value, bool):
            error = "Newton did not converge"
        work_stream.synchronize()
        results[job.req.rid] = Result(job.req.rid, value.cpu() if (keep and error is None) else None,
                                      len(job.solver.history),
                                      sum(h.get("pcg_iters", 0) for h in job.solver.history), job.req.arrival,
                                      job.admitted, time.perf_counter() - t0, error)
        mem_used -= job.bytes

    timing = {"newton_host_s": 0.0, "wait_s": 0.0, "prep_s": 0.0}

    def advance(job, first=False):
        """Run the job's Newton iteration up to its next tangent solve (on the
        work stream, while the GPU iterates the other slots)."""
        t_a = time.perf_counter()
        try:
            return _advance(job, first)
        except Exception as ex:              # a failing request is rejected; the others go on
            finish(job, False, "%s: %s" % (type(ex).__name__, ex))
            return False
        finally:
            timing["newton_host_s"] += time.perf_counter() - t_a

    def _advance(job, first):
        with torch.cuda.stream(work_stream):
            try:
                job.lin = next(job.gen) if first else job.gen.send(None)
            except StopIteration as stop:
                finish(job, stop.value)
                return False
            if job.work is None:
                job.work = torch.empty(BatchedPCG.work_len(job.asm.plan), dtype=torch.float64, device=dev)
        queue_slot.append(job)
        return True

    slots = [None] * max_slots
    finished = []                      # jobs whose solve ended in the last polled round
    in_flight = False
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    timing.update(round_gpu_s=0.0, slot_rounds=0)
    while waiting or preparing or ready or queue_slot or finished or in_flight or any(j is not None for j in slots):
        now = time.perf_counter() - t0
        # admit arrived requests into preparation while memory allows
        while waiting and waiting[0].arrival <= now and free_streams:
            nb = estimate_bytes(waiting[0])
            if nb > mem_budget:               # could never be admitted: rejected at admission
                req = waiting.pop(0)
                results[req.rid] = Result(req.rid, None, 0, 0, req.arrival, now, time.perf_counter() - t0,
                                          "needs %d bytes, more than the memory budget %d" % (nb, mem_budget))
                continue
            if mem_used + nb > mem_budget and (preparing or ready or queue_slot or any(slots)):
                break
            req = waiting.pop(0)
            st_ = free_streams.pop()
            mem_used += nb
            preparing[pool.submit(_prepare, req, st_)] = (req, st_, nb, now)
        for fut in [f for f in preparing if f.done()]:
            req, st_, nb, adm = preparing.pop(fut)
            free_streams.append(st_)
            try:
                asm, sol = fut.result()
            except Exception as ex:          # the model could not be built: rejected
                results[req.rid] = Result(req.rid, None, 0, 0, req.arrival, adm, time.perf_counter() - t0,
                                          "%s: %s" % (type(ex).__name__, ex))
                mem_used -= nb
                continue
            with torch.cuda.stream(work_stream):
                ready.append(_Job(req, asm, sol, adm, nb))
        # host work of the jobs that left the batch, overlapping the round in flight
        for job in ready:
            advance(job, first=True)
        ready.clear()
        for job in finished:
            advance(job)
        finished.clear()
        if in_flight:
            t_w = time.perf_counter()
            state = eng.wait()
            timing["wait_s"] += time.perf_counter() - t_w
            timing["round_gpu_s"] += ev_a.elapsed_time(ev_b) * 1e-3
            in_flight = False
            busy_rounds += 1
            for k, job in enumerate(slots):
                if job is None or state[k, 0] == 0.0:
                    continue
                lin = job.lin
                lin.it, lin.status, lin.rr = int(state[k, 1]), int(state[k, 2]), float(state[k, 3])
                slots[k] = None
                eng.release(k)
                finished.append(job)
        # free slots to waiting solves
        fresh = []
        for k in range(max_slots):
            if slots[k] is None and queue_slot:
                job = queue_slot.pop(0)
                job.slot = k
                slots[k] = job
                eng.assign(k, job.asm.plan, job.lin, job.work)
                fresh.append(k)
        if not any(j is not None for j in slots):
            if not finished:
                if waiting and not preparing:
                    time.sleep(max(0.0, min(0.002, waiting[0].arrival - (time.perf_counter() - t0))))
                else:
                    time.sleep(0.0005)
            continue
        eng.sync()
        if fresh:
            main.wait_stream(work_stream)
            for k in fresh:
                eng.start(k)
        timing["slot_rounds"] += sum(j is not None for j in slots)
        ev_a.record()
        eng.run_round()
        ev_b.record()
        eng.poll_async()
        in_flight = True
    pool.shutdown()
    stats = {"rounds": busy_rounds, "graph": eng.graph is not None, "max_slots": max_slots,
             "round_iters": round_iters, "mem_budget": int(mem_budget), "wall_s": time.perf_counter() - t0,
             **timing}
    return [results[r.rid] for r in sorted(requests, key=lambda r: r.rid)], stats

