"""Device-side line search of the Newton solver (static_implicit.py:97-169):
trial energies of a ladder of steps evaluated on the device and the first
accepted step selected and applied there.  The ladder's energies equal the
total potential at those points, and the Newton solve with the device
search takes the same steps as the host search and converges to the
reference's solution."""
import numpy as np
import pytest
import torch

from tests.helpers import fea_model, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,kind", [("hex5", "C3D8"), ("cfg1", "C3D4")])
def test_ladder_energies_are_the_total_potential(golden, name, kind):
    from fea_b200 import _lib as L
    g = golden(name)
    c, e, _ = fea_model(g, kind)
    c.initialize()
    A = c.assembly
    P = A.plan
    gc = torch.from_numpy(g["state"]).cuda()
    R = A.assemble_force(GC=gc)
    dgc = 1e-2 * torch.randn(gc.shape, generator=torch.Generator().manual_seed(3), dtype=torch.float64).cuda()
    e0 = A._total_Potential_Energy(GC=gc).reshape(1)
    st = torch.empty(L.FEA_LS_NSTATE, dtype=torch.float64, device="cuda")
    P.ls_prepare(dgc, R, e0, st)
    h = st.tolist()
    de = float((dgc * R).sum())
    assert h[L.FEA_LS_SIGN] == (-1.0 if de > 0 else 1.0)
    assert abs(h[L.FEA_LS_DE] + abs(de)) <= 1e-12 * abs(de)
    assert h[L.FEA_LS_SMAX] == float(dgc.abs().max()) and h[L.FEA_LS_E0] == float(e0)
    for k0 in (0, 8):
        E = torch.empty(L.FEA_LS_M, dtype=torch.float64, device="cuda")
        mu, kappa = e.materials.parameters()
        P.ls_energy_volume(0, mu, kappa, gc, dgc, st, k0, E, False)
        for fi, ld in enumerate(A._face_loads):
            P.ls_energy_pressure(fi, float(ld.pressure), A._Xinst, gc, dgc, st, k0, E, True)
        for k in range(L.FEA_LS_M):
            a = h[L.FEA_LS_SIGN] * 2.0 ** -(k0 + k)
            ref = float(A._total_Potential_Energy(GC=gc + a * dgc))
            assert abs(float(E[k]) - ref) <= 1e-12 * abs(ref), (k0, k)


def test_select_takes_the_first_armijo_step_and_applies_it(golden):
    """A step too long for alpha = 1: the device picks the same halving as
    the host loop and moves gc by exactly that step."""
    import fea_b200 as F
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    A = c.assembly
    gc = torch.from_numpy(g["state"]).cuda()
    R = A.assemble_force(GC=gc)
    dgc = -0.5 * R / R.abs().max()                      # a descent direction, far too long
    E0 = A._total_Potential_Energy(GC=gc)
    s = F.solver.StaticImplicitSolver()
    s.initialize(A)
    a_d, gc_d, e_d = s._line_search_device(gc, dgc, R, E0)
    a_h, gc_h, e_h = s._line_search_host(gc, dgc, R, E0)
    assert a_d == a_h and 0.0 < a_d < 1.0
    step = gc + a_d * dgc
    assert float((gc_d - step).abs().max()) <= 1e-15 * float(step.abs().max())
    assert rel(gc_d, gc_h) < 1e-15
    assert abs(float(e_d) - float(e_h)) <= 1e-12 * abs(float(e_h))


@pytest.mark.parametrize("name,kind", [("hex5", "C3D8"), ("cfg1", "C3D4")])
def test_newton_with_device_line_search_matches_host_search(golden, name, kind):
    import fea_b200 as F
    g = golden(name)
    runs = []
    for dev in (True, False):
        c, e, ld = fea_model(g, kind, solver=F.solver.StaticImplicitSolver(rtol=1e-11, maximum_iteration=60,
                                                                            device_line_search=dev))
        c.initialize()
        if name == "cfg1":
            gc = c.assembly.GC.clone()
            for k in range(1, 6):
                ld.pressure = float(g["p"]) * k / 5
                gc = c.solver.solve(GC0=gc)
                assert not isinstance(gc, bool)
            ref = g["gc_increments"][-1]
        else:
            gc = c.solver.solve()
            ref = g["gc_converged"]
        runs.append(([h.get("alpha") for h in c.solver.history], gc))
        assert rel(gc, ref) < 1e-8
    (a1, g1), (a2, g2) = runs
    assert len(a1) == len(a2) and all(x == y or abs(x - y) <= 1e-15 for x, y in zip(a1, a2) if x is not None)
    assert rel(g1, g2) < 1e-10
