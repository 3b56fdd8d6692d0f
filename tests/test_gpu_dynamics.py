"""Implicit Newmark dynamics through the CUDA path against the reference's
DynamicImplicitSolver (golden histories) and the oracle.

Tolerances: consistent mass <= 1e-13 relative (pattern equal to the
stiffness pattern, as the reference stores it); displacement and velocity
histories <= 1e-6 relative and accelerations <= 1e-5 relative per stored
time: every Newton step of both stops at max|R| < tol = 1e-8, the reference
with direct solves, this path with device PCG, and the acceleration divides
the displacement difference by beta dt^2.
"""
import numpy as np
import pytest
import torch

from tests.helpers import fea_model, rel

pytestmark = pytest.mark.gpu


NEWMARK = ["newmark_tet2", "newmark_hex2"]


def _newmark_model(g):
    import fea_b200 as F
    dt, steps = float(g["dt"]), int(g["steps"])
    sol = F.solver.DynamicImplicitSolver(deltaT=dt, time_end=steps * dt * (1 - 1e-9), tol_error=float(g["tol"]))
    c, e, load = fea_model(g, str(g["kind"]), solver=sol)
    c.initialize()
    return c


@pytest.mark.parametrize("name", NEWMARK)
def test_consistent_mass_vs_golden(golden, name):
    g = golden(name)
    c = _newmark_model(g)
    idx, vals = c.assembly.assemble_mass_matrix(GC_now=None)
    n = g["GC"].shape[1]
    dense = torch.zeros(n, n, dtype=torch.float64)
    dense.index_put_((idx[0].cpu(), idx[1].cpu()), vals.cpu(), accumulate=True)
    ref = torch.zeros(n, n, dtype=torch.float64)
    ip, ix, vv = g["mass_indptr"], g["mass_indices"], g["mass_values"]
    rows = np.repeat(np.arange(n), np.diff(ip))
    ref[torch.from_numpy(rows), torch.from_numpy(ix.astype(np.int64))] = torch.from_numpy(vv)
    assert rel(dense, ref) < 1e-13
    np.testing.assert_array_equal(c.assembly.plan.indptr.cpu().numpy(), ip)
    np.testing.assert_array_equal(c.assembly.plan.indices.cpu().numpy(), ix)


@pytest.mark.parametrize("name", NEWMARK)
def test_newmark_histories_vs_reference(golden, name):
    g = golden(name)
    c = _newmark_model(g)
    n = g["GC"].shape[1]
    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert c.solver.solve(GC0=z, GV0=z) is True
    s = c.solver
    assert len(s._GC_list) == g["GC"].shape[0]
    assert abs(s._time_list[-1] - float(g["time"][-1])) < 1e-12
    scale_u = np.abs(g["GC"]).max()
    for k in range(len(s._GC_list)):
        assert np.abs(s._GC_list[k].cpu().numpy() - g["GC"][k]).max() <= 1e-6 * scale_u
        assert np.abs(s._GV_list[k].cpu().numpy() - g["GV"][k]).max() <= 1e-6 * np.abs(g["GV"]).max()
        assert np.abs(s._GA_list[k].cpu().numpy() - g["GA"][k]).max() <= 1e-5 * np.abs(g["GA"]).max()
    # each step's last Newton residual is below the tolerance
    assert s.history[-1]["rmax"] < float(g["tol"])


@pytest.mark.parametrize("name", NEWMARK)
def test_newmark_energy_and_incremental_system(golden, name):
    """The incremental system is the gradient and Hessian of the incremental
    energy: central differences of the energy along a random direction match
    R . d, and of R match K d."""
    g = golden(name)
    c = _newmark_model(g)
    s = c.solver
    n = g["GC"].shape[1]
    gen = torch.Generator().manual_seed(3)
    x = (1e-3 * torch.randn(n, generator=gen, dtype=torch.float64)).cuda()
    pre = (1e-3 * torch.randn(n, generator=gen, dtype=torch.float64)).cuda()
    d = torch.randn(n, generator=gen, dtype=torch.float64).cuda()
    R, Ki, Kv = s.get_incremental_stiffness_matrix(x, pre)
    h = 1e-6
    ep = float(s.get_incremental_energy(x + h * d, pre))
    em = float(s.get_incremental_energy(x - h * d, pre))
    assert abs((ep - em) / (2 * h) - float(torch.dot(R, d))) <= 1e-6 * abs(float(torch.dot(R, d)))
    Rp = s.get_incremental_stiffness_matrix(x + h * d, pre)[0]
    Rm = s.get_incremental_stiffness_matrix(x - h * d, pre)[0]
    Kd = c.assembly.plan.spmv(Kv, d)
    assert rel((Rp - Rm) / (2 * h), Kd) < 1e-6
