"""Serving: batched PCG slots and continuous batching of static solves.

Tolerances: a slot of the batched PCG reaches the same solution as the
single-system PCG to 1e-10 relative; a served request's result is
bitwise identical alone and among others; served and plain converged
displacements agree to 1e-7 relative (both are Newton solves to a relative
residual of 1e-8), and a served result agrees with the FP64 oracle's
direct-solve Newton solution to 1e-8."""
import pytest
import torch

from tests.helpers import rel

pytestmark = pytest.mark.gpu


def _small_requests(n, seed):
    from fea_b200 import serving
    reqs = serving.make_requests(n, float("inf"), seed=seed, min_elems=2000, max_elems=9000)
    for r in reqs:
        r.arrival = 0.0
    return reqs


def test_batched_pcg_slots_match_single_solves():
    from fea_b200 import serving
    reqs = _small_requests(3, seed=1)
    systems = []
    for r in reqs:
        asm = serving.build_assembly(r)
        R, K = asm.assemble_csr(asm.GC)
        systems.append((asm, (-R).contiguous(), K.clone()))
    eng = serving.BatchedPCG(4, 4 * 1024, round_iters=16)
    xs, works = [], []
    import fea_b200._lib as L
    from fea_b200.solver import LinearSolve
    for k, (asm, b, K) in enumerate(systems):
        x = torch.zeros_like(b)
        w = torch.empty(serving.BatchedPCG.work_len(asm.plan), dtype=torch.float64, device="cuda")
        eng.assign(k, asm.plan, LinearSolve(K, b, x, 1e-24, 20000, True), w, node_rows=(k != 1))
        xs.append(x)
        works.append(w)
    eng.sync()
    for k in range(3):
        eng.start(k)
    for _ in range(2000):
        eng.run_round()
        st = eng.poll()
        if st[:3, 0].all():
            break
    assert st[:3, 0].all() and (st[:3, 2] == 0).all()
    for k, (asm, b, K) in enumerate(systems):
        x1 = torch.zeros_like(b)
        it, rr, status = asm.plan.pcg(K, b, x1, 1e-24, 20000)
        assert status == 0
        assert rel(xs[k], x1) < 1e-10
        r = b - asm.plan.spmv(K, xs[k])
        assert float(r.norm() / b.norm()) < 1e-10
    # the first system alone in the engine gives the same bits
    asm, b, K = systems[0]
    eng1 = serving.BatchedPCG(1, 1024, round_iters=16)
    x = torch.zeros_like(b)
    w = torch.empty(serving.BatchedPCG.work_len(asm.plan), dtype=torch.float64, device="cuda")
    eng1.assign(0, asm.plan, LinearSolve(K, b, x, 1e-24, 20000, True), w)
    eng1.sync()
    eng1.start(0)
    while True:
        eng1.run_round()
        if eng1.poll()[0, 0]:
            break
    assert torch.equal(x, xs[0])


def test_served_results_same_alone_and_in_the_mix():
    from fea_b200 import serving
    reqs = _small_requests(5, seed=2)
    mixed, stats = serving.serve(reqs, max_slots=4, round_iters=16)
    assert stats["rounds"] > 0
    for r in (reqs[0], reqs[3]):
        alone, _ = serving.serve([r], max_slots=4, round_iters=16)
        assert torch.equal(alone[0].gc, mixed[r.rid].gc)
        assert alone[0].newton_iters == mixed[r.rid].newton_iters
    plain = serving.solve_plain(reqs)
    for a, b in zip(mixed, plain):
        assert a.rid == b.rid
        assert rel(a.gc, b.gc) < 1e-7
        assert a.latency > 0 and b.latency > 0


def test_served_result_matches_the_fp64_oracle():
    """A served request against the oracle's Newton solve of the same model
    (reference algorithm, direct solves, residual to 1e-12 of the first)."""
    import numpy as np
    from fea_b200 import meshes, serving
    from oracle import fea_oracle as O
    reqs = _small_requests(3, seed=5)
    served, _ = serving.serve(reqs, max_slots=4, round_iters=16)
    r = min(reqs, key=lambda q: q.n_elems)
    X, el = meshes.tet_beam(r.length, r.width, r.height, r.n_elems)
    root = np.nonzero(np.abs(X[:, 0] - (1.0 - r.length)) < 1e-9)[0]
    _, faces = meshes.plane_faces("C3D4", el, X, 0, 1.0)
    m = O.Model(torch.from_numpy(X), [O.Group("C3D4", torch.from_numpy(el), r.mu, r.kappa)],
                [O.PressureLoad(torch.from_numpy(faces), r.pressure)], [(root, (0, 1, 2))])
    gc, it = O.newton_solve(m, m.initial_gc(), rtol=1e-12, linear="direct")
    assert rel(served[r.rid].gc, gc) < 1e-8
