"""One reduced system over two gloo ranks on CPU: node-range partition, halo
exchange of the search direction, two scalar all-reduces per iteration.  The
sharded Jacobi-PCG reproduces the single-rank solve of the same system (the
oracle's reduced K and R of a jittered C3D8 block with pressure), and the
shards' rows and halos cover the matrix exactly once."""
import os
import sys

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _system():
    sys.path.insert(0, ROOT)
    from oracle import fea_oracle as O
    n = 4
    X, el = O.hex_block(n, jitter=0.1, seed=3)
    E = el.shape[0]
    top = torch.nonzero(torch.arange(E) % n == n - 1).flatten()
    faces = el[top][:, [4, 5, 6, 7]]
    bottom = torch.nonzero(torch.arange(X.shape[0]) % (n + 1) == 0).flatten()
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 50.0)], [O.PressureLoad(faces, 0.03)], [(bottom, (0, 1, 2))])
    gc = 1e-3 * torch.randn(int(m.free_mask().sum()), generator=torch.Generator().manual_seed(1), dtype=torch.float64)
    R, (ip, ix, v) = m.assemble(gc)
    node_dofs = m.free_mask().view(-1, 3).sum(1).numpy()
    return ip, ix, v, -R, node_dofs


def _single(ip, ix, v, b, tol):
    """The same Jacobi-PCG on one rank (plain torch, the same recurrence)."""
    A = torch.sparse_csr_tensor(ip, ix, v, (b.shape[0], b.shape[0]))
    rows = torch.repeat_interleave(torch.arange(b.shape[0]), ip[1:] - ip[:-1])
    d = torch.zeros_like(b)
    d[rows[ix == rows]] = v[ix == rows]
    dinv = 1.0 / d
    x = torch.zeros_like(b)
    r = b.clone(); z = dinv * r; p = z.clone()
    rz, bb = float(r @ z), float(b @ (dinv * b))
    for it in range(1, 5000):
        q = A @ p
        a = rz / float(p @ q)
        x += a * p; r -= a * q; z = dinv * r
        rzn = float(r @ z)
        if rzn / bb < tol:
            return x, it
        p = z + rzn / rz * p; rz = rzn
    return x, 5000


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from fea_b200 import distributed as D
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ip, ix, v, b, node_dofs = _system()
        row_start, node_start = D.partition_rows(node_dofs, world)
        S = D.ShardedSystem.from_plan_rows(rank, world, row_start, ip, ix)
        lo, hi = int(ip[S.row0]), int(ip[S.row1])
        x = torch.zeros(S.nloc, dtype=torch.float64)
        it, rr, st = D.sharded_pcg(S, v[lo:hi], b[S.row0:S.row1], x, 1e-24, 5000)
        out[rank] = (x.numpy(), it, st, S.row0, S.row1, S.halo_cols.numpy(), {k: w.numpy() for k, w in S.send.items()})
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_partition_rows_balances_contiguous_node_ranges():
    sys.path.insert(0, ROOT)
    from fea_b200 import distributed as D
    nd = np.array([3, 0, 3, 2, 3, 3, 1, 3])
    rows, nodes = D.partition_rows(nd, 3)
    assert rows[0] == 0 and rows[-1] == nd.sum() and nodes[-1] == nd.shape[0]
    assert np.all(np.diff(rows) >= 0) and np.all(np.diff(nodes) >= 0)
    assert np.array_equal(rows, np.concatenate([[0], np.cumsum(nd)])[nodes])


def test_sharded_pcg_two_gloo_ranks_matches_single_rank():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(world, 29531, out), nprocs=world, start_method="spawn")
    ip, ix, v, b, node_dofs = _system()
    xs, it1 = _single(ip, ix, v, b, 1e-24)
    x = np.concatenate([out[r][0] for r in range(world)])
    assert out[0][2] == 0 and out[1][2] == 0 and out[0][1] == out[1][1]
    assert np.linalg.norm(x - xs.numpy()) <= 1e-10 * np.linalg.norm(xs.numpy())
    assert abs(out[0][1] - it1) <= 2
    # rows split once; each rank's halo is exactly what the other sends it
    assert out[0][3] == 0 and out[0][4] == out[1][3] and out[1][4] == b.shape[0]
    h1 = out[1][5]
    assert np.array_equal(np.sort(out[0][6][1] + out[0][3]), h1)
    h0 = out[0][5]
    assert np.array_equal(np.sort(out[1][6][0] + out[1][3]), h0)
