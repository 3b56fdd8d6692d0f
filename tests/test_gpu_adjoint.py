"""Hand-written adjoint against the reference's autograd and finite differences."""
import numpy as np
import pytest
import torch

from tests.helpers import fea_model, rel

pytestmark = pytest.mark.gpu


def test_residual_vjp_matches_reference_autograd(golden):
    """lam . dR/dX and lam . dR/dmu at the converged state equal the
    reference's autograd of (R . lam) (tests/gradient_test/test_grad.py recipe)."""
    from fea_b200 import adjoint
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    gc = torch.from_numpy(g["gc_converged"]).cuda()
    lam = torch.from_numpy(g["adj_lambda"]).cuda()
    dX, dmu = adjoint.residual_vjp(c.assembly, gc, lam)
    assert rel(dX, g["adj_gX"]) < 1e-12
    assert abs(float(dmu[0]) - float(g["adj_gmu"])) <= 1e-12 * abs(float(g["adj_gmu"]))


def _solve(c, X=None, mu=None):
    import fea_b200 as F
    from fea_b200 import adjoint
    asm = c.assembly
    if X is not None:
        adjoint.set_coordinates(asm, X)
    if mu is not None:
        asm._mat_elems[0].materials.mu = torch.tensor(mu, dtype=torch.float64)
    s = F.solver.StaticImplicitSolver(rtol=1e-14, maximum_iteration=60)
    s.initialize(asm)
    gc = s.solve(GC0=torch.zeros_like(asm.GC))
    assert not isinstance(gc, bool)
    f = adjoint.external_force(asm, gc)
    return float(torch.dot(f, gc)), gc


def test_compliance_gradient_vs_central_differences(golden):
    from fea_b200 import adjoint
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    X0 = torch.from_numpy(g["X"]).clone()
    mu0 = float(g["mu"])
    C0, gc = _solve(c)
    C, dX, dmu, it = adjoint.compliance_gradient(c.assembly, gc)
    assert abs(float(C) - C0) <= 1e-14 * abs(C0)
    h = 1e-6
    rng = np.random.default_rng(0)
    N = X0.shape[0]
    nodes = rng.choice(N, size=8, replace=False)
    comps = rng.integers(0, 3, size=8)
    scale = float(dX.abs().max())
    for nd, k in zip(nodes, comps):
        Xp = X0.clone(); Xp[nd, k] += h
        Xm = X0.clone(); Xm[nd, k] -= h
        fd = (_solve(c, X=Xp)[0] - _solve(c, X=Xm)[0]) / (2 * h)
        ad = float(dX[nd, k])
        # central differences at h = 1e-6 carry ~1e-9 of the largest component
        # in truncation and round-off; components below 1 % of the largest
        # are compared against 1e-6 of that 1 %
        assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-2 * scale), (nd, k, fd, ad)
    _solve(c, X=X0)
    fd = (_solve(c, mu=mu0 + h)[0] - _solve(c, mu=mu0 - h)[0]) / (2 * h)
    assert abs(fd - float(dmu[0])) <= 1e-6 * abs(float(dmu[0]))


def test_autograd_function_wraps_the_adjoint(golden):
    import fea_b200 as F
    from fea_b200 import adjoint
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    X = torch.from_numpy(g["X"]).clone().requires_grad_(True)
    mu = torch.tensor(float(g["mu"]), dtype=torch.float64, requires_grad=True)
    solver = F.solver.StaticImplicitSolver(rtol=1e-14, maximum_iteration=60)
    solver.initialize(c.assembly)
    C = adjoint.ComplianceFunction.apply(X, mu, c.assembly, solver)
    C.backward()
    C0, gc = _solve(c, X=torch.from_numpy(g["X"]), mu=float(g["mu"]))
    _, dX, dmu, _ = adjoint.compliance_gradient(c.assembly, gc)
    assert abs(float(C) - C0) <= 1e-12 * abs(C0)
    assert rel(X.grad, dX) < 1e-10
    assert abs(float(mu.grad) - float(dmu[0])) <= 1e-10 * abs(float(dmu[0]))
