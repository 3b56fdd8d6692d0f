"""The node partition of one system, on one GPU: a rank's plan over its
elements (owned plus the one-element halo) assembles its owned rows of R and
K exactly as the whole-mesh plan does (same columns, bit-identical values),
so sharded assembly needs no exchange.  The sharded PCG itself is covered on
gloo CPU ranks (tests/test_sharded_pcg.py)."""
import numpy as np
import pytest
import torch

from oracle import fea_oracle as O

pytestmark = pytest.mark.gpu


def test_rank_plans_assemble_owned_rows_like_the_whole_mesh():
    from fea_b200 import distributed as D
    from fea_b200.plan import DevicePlan
    n = 5
    X, el = O.hex_block(n, jitter=0.1, seed=4)
    E, N = el.shape[0], X.shape[0]
    top = torch.nonzero(torch.arange(E) % n == n - 1).flatten()
    faces = el[top][:, [4, 5, 6, 7]].numpy()
    free = np.ones((N, 3), bool)
    free[np.arange(N) % (n + 1) == 0] = False                       # bottom clamped
    mask = (free @ np.array([1, 2, 4])).astype(np.uint8)
    full = DevicePlan(X, mask, [("C3D8", el.numpy())], [("Q4", faces)])
    gc = 1e-3 * torch.randn(full.ndof, generator=torch.Generator().manual_seed(2), dtype=torch.float64).cuda()
    Xi = X.cuda()

    def assemble(P, g):
        K = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
        R = torch.empty(P.ndof, dtype=torch.float64, device="cuda")
        P.assemble_volume(0, 1.0, 50.0, g, K=K, R=R)
        P.assemble_pressure(0, 0.03, Xi, g, K=K, R=R)
        return R.cpu(), K.cpu()

    Rf, Kf = assemble(full, gc)
    ipf, ixf = full.indptr.cpu(), full.indices.cpu().long()
    rdof_full = np.concatenate([[0], np.cumsum(free.sum(1))])
    row_start, node_start = D.partition_rows(free.sum(1), 2)
    for r in range(2):
        lo, hi = int(node_start[r]), int(node_start[r + 1])
        sel = D.rank_elements(el.numpy(), lo, hi)
        sub_el = el.numpy()[sel]
        present = np.zeros(N, bool)
        present[np.unique(sub_el)] = True
        smask = np.where(present, mask, 0).astype(np.uint8)
        fsel = D.rank_elements(faces, lo, hi)
        P = DevicePlan(X, smask, [("C3D8", sub_el)], [("Q4", faces[fsel])])
        # sub-plan DOF -> global DOF (same node-major order over the present nodes)
        g2l = np.full(full.ndof, -1, np.int64)
        nodes_dofs = [(nd, k) for nd in range(N) for k in range(3) if smask[nd] >> k & 1]
        l2g = np.array([rdof_full[nd] + int(np.sum(free[nd, :k])) for nd, k in nodes_dofs], np.int64)
        g2l[l2g] = np.arange(l2g.shape[0])
        Rs, Ks = assemble(P, gc[torch.from_numpy(l2g).cuda()])
        ips, ixs = P.indptr.cpu(), P.indices.cpu().long()
        for grow in range(int(row_start[r]), int(row_start[r + 1])):
            lrow = int(g2l[grow])
            cols_l = ixs[int(ips[lrow]):int(ips[lrow + 1])]
            cols_g = torch.from_numpy(l2g)[cols_l]
            assert torch.equal(cols_g, ixf[int(ipf[grow]):int(ipf[grow + 1])])
            assert torch.equal(Ks[int(ips[lrow]):int(ips[lrow + 1])], Kf[int(ipf[grow]):int(ipf[grow + 1])])
            assert float(Rs[lrow]) == float(Rf[grow])
