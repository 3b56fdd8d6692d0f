"""Failure detection without faulting the GPU: failures are made on the host
(an indefinite or NaN system, an iteration cap, an inverted element, a
poisoned serving request) and the CUDA path must report them through its
status codes and exceptions, return, and leave the device usable; a
rejected serving request must not change the other requests' results.
"""
import math

import pytest
import torch

from tests.helpers import fea_model

pytestmark = pytest.mark.gpu


def _system(golden):
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    asm = c.assembly
    R, K = asm.assemble_csr(asm.GC)
    return asm, K, (-R).contiguous()


def test_pcg_reports_breakdown_on_an_indefinite_system(golden):
    from fea_b200 import _lib as L
    asm, K, b = _system(golden)
    P = asm.plan
    x = torch.zeros_like(b)
    it, rr, st = P.pcg(-K, b, x, 1e-20, 1000, raise_on_breakdown=False)
    assert st == L.FEA_EBREAKDOWN and it <= 1
    with pytest.raises(L.FeaError):
        P.pcg(-K, b, torch.zeros_like(b), 1e-20, 1000, raise_on_breakdown=True)
    # the device is still usable: the same system solves
    x = torch.zeros_like(b)
    it, rr, st = P.pcg(K, b, x, 1e-20, 5000)
    assert st == L.FEA_OK


def test_pcg_reports_nan_input_and_the_iteration_cap(golden):
    from fea_b200 import _lib as L
    asm, K, b = _system(golden)
    P = asm.plan
    bn = b.clone()
    bn[3] = float("nan")
    it, rr, st = P.pcg(K, bn, torch.zeros_like(b), 1e-20, 1000, raise_on_breakdown=False)
    assert st == L.FEA_EBREAKDOWN
    it, rr, st = P.pcg(K, b, torch.zeros_like(b), 1e-30, 7)
    assert st == L.FEA_ENOTCONV and it == 7
    with pytest.raises(L.FeaError):
        P.pcg(K, b, torch.zeros_like(b), 1e-30, 7, raise_on_cap=True)


def test_inverted_element_gives_nan_and_newton_raises(golden):
    """An element turned inside out (J < 0) has no Neo-Hookean energy: R is NaN
    there, as in the reference (J ** (-2/3) of a negative J), and the Newton
    step raises the reference's ValueError on the non-finite direction."""
    import fea_b200 as F
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8", solver=F.solver.StaticImplicitSolver(maximum_iteration=5))
    c.initialize()
    asm = c.assembly
    X = torch.from_numpy(g["X"])
    el = torch.from_numpy(g["elems"])
    U = torch.zeros_like(X)
    e0 = el.shape[0] // 2                       # an interior element: mirror its top nodes through its bottom
    top, bot = el[e0, 4:], el[e0, :4]
    U[top, 2] = -2.0 * (X[top, 2] - X[bot, 2])
    rgc = asm._GC2RGC(torch.zeros(asm.plan.ndof, dtype=torch.float64))
    rgc[0] = U.to(rgc[0].device)
    gc = asm._RGC2GC(rgc)
    R = asm.assemble_force(GC=gc)
    assert not bool(torch.isfinite(R).all())
    with pytest.raises(ValueError):
        c.solver.solve(GC0=gc)


def test_serving_rejects_a_poisoned_request_and_keeps_the_others():
    from fea_b200 import serving
    reqs = serving.make_requests(4, float("inf"), seed=11, min_elems=2000, max_elems=5000)
    for r in reqs:
        r.arrival = 0.0
    good, _ = serving.serve([r for r in reqs if r.rid != 2], max_slots=4, round_iters=16)
    reqs[2].pressure = float("nan")
    mixed, _ = serving.serve(reqs, max_slots=4, round_iters=16)
    assert mixed[2].error is not None and mixed[2].gc is None
    for a, b in zip(good, [m for m in mixed if m.rid != 2]):
        assert a.rid == b.rid and b.error is None
        assert torch.equal(a.gc, b.gc)
    plain = serving.solve_plain(reqs)
    assert plain[2].error is not None and all(p.error is None for p in plain if p.rid != 2)
    assert all(math.isfinite(p.latency) for p in plain)


def test_serving_rejects_a_request_beyond_the_memory_budget():
    from fea_b200 import serving
    reqs = serving.make_requests(3, float("inf"), seed=12, min_elems=2000, max_elems=4000)
    for r in reqs:
        r.arrival = 0.0
    reqs[1].n_elems = 40000
    budget = max(serving.estimate_bytes(r) for r in (reqs[0], reqs[2])) * 2
    assert serving.estimate_bytes(reqs[1]) > budget
    res, _ = serving.serve(reqs, max_slots=4, round_iters=16, mem_budget=budget)
    assert res[1].error is not None and "memory budget" in res[1].error and res[1].gc is None
    assert res[0].error is None and res[2].error is None
    alone, _ = serving.serve([reqs[0], reqs[2]], max_slots=4, round_iters=16)
    assert torch.equal(alone[0].gc, res[0].gc) and torch.equal(alone[1].gc, res[2].gc)
