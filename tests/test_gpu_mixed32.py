"""The FP32 inner solver on the padded node layout (fea_f32_layout_fill,
fea_pcg_solve_mixed_nodes32): the layout holds the plan's FP32 values and
columns (padding zeros), the mixed solve meets its FP64 stop test and the
direct solution to 1e-8 with and without inner_tol, and the Newton solver's mixed mode uses
it."""
import numpy as np
import pytest
import torch

from oracle import fea_oracle as O
from tests.helpers import fea_model, rel

pytestmark = pytest.mark.gpu


def test_padded_layout_holds_the_plan_matrix(golden):
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    P = c.assembly.plan
    R, K = c.assembly.assemble_csr(torch.from_numpy(g["state"]).cuda())
    desc, cbase, qbase, cols, vals = P.f32_layout()
    P.fill_f32(K)
    ip, ix = P.indptr.cpu().numpy(), P.indices.cpu().numpy()
    Kc = K.cpu().numpy()
    mask, rowlen, rdof = P.mask.cpu().numpy(), P.rowlen.cpu().numpy(), P.rdof.cpu().numpy()
    cb, qb, cl, vl = cbase.cpu().numpy(), qbase.cpu().numpy(), cols.cpu().numpy(), vals.cpu().numpy()
    assert np.all(cb % 4 == 0) and np.all(qb % 4 == 0)
    for nd in range(P.n_nodes):
        if mask[nd] == 0:
            assert cb[nd + 1] == cb[nd]
            continue
        L, L4 = int(rowlen[nd]), int(cb[nd + 1] - cb[nd])
        assert L4 == (L + 3) // 4 * 4
        f = bin(int(mask[nd])).count("1")
        for j in range(f):
            row = int(rdof[nd]) + j
            a, b = int(ip[row]), int(ip[row + 1])
            assert np.array_equal(cl[cb[nd]:cb[nd] + L], ix[a:b]) and not cl[cb[nd] + L:cb[nd + 1]].any()
            v = vl[qb[nd] + j * L4:qb[nd] + (j + 1) * L4]
            assert np.array_equal(v[:L], Kc[a:b].astype(np.float32)) and not v[L:].any()


@pytest.mark.parametrize("inner_tol", [0.0, 1e-4])
def test_mixed_padded_layout_solve_matches_direct(golden, inner_tol):
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    P = c.assembly.plan
    R, K = c.assembly.assemble_csr(torch.from_numpy(g["state"]).cuda())
    b = (-R).contiguous()
    x = torch.zeros_like(b)
    it, outer, rr, st = P.pcg_mixed(K, None, b, x, 1e-22, inner_tol, 20000, check_every=20)
    assert st == 0 and outer >= 1
    ip, ix, Kc = P.indptr.cpu(), P.indices.cpu().long(), K.cpu()
    xd = O.direct_solve(ip, ix, Kc, b.cpu())
    # the true FP64 residual meets the stop test (r.D^-1 r)/(b.D^-1 b) < tol,
    # and the displacements are within the 1e-8 of the solver contract
    A = torch.sparse_csr_tensor(ip, ix, Kc, (b.numel(), b.numel()))
    rows = torch.repeat_interleave(torch.arange(b.numel()), ip[1:] - ip[:-1])
    dinv = 1.0 / Kc[ix == rows]
    r = b.cpu() - A @ x.cpu()
    assert float((r * dinv * r).sum() / (b.cpu() * dinv * b.cpu()).sum()) < 1e-20
    assert rel(x, xd) < 1e-8
    if inner_tol > 0:
        x0 = torch.zeros_like(b)
        it0, outer0, _, st0 = P.pcg_mixed(K, None, b, x0, 1e-22, 0.0, 20000, check_every=20)
        assert st0 == 0 and outer <= outer0


def test_newton_mixed_mode_on_padded_layout(golden):
    import fea_b200 as F
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8", solver=F.solver.StaticImplicitSolver(rtol=1e-11, maximum_iteration=60,
                                                                          precision="mixed"))
    c.initialize()
    gc = c.solver.solve()
    assert not isinstance(gc, bool)
    assert rel(gc, g["gc_converged"]) < 1e-8
