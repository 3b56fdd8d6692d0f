"""CPU checks of the C ABI: the library loads, exports every declared symbol,
and its host-side plan reproduces the reference's reduced pattern."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from oracle import fea_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "fea_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fea_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from fea_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTED) == names
    assert _lib.fea_version() == 1


def _plan(N, mask, groups, faces=()):
    from fea_b200.plan import HostPlan, KIND
    return HostPlan(N, mask, [(KIND[k], c) for k, c in groups], [(KIND[k], c) for k, c in faces])


@pytest.mark.parametrize("name,kind", [("cfg1", "C3D4"), ("tet3", "C3D4"), ("hex5", "C3D8")])
def test_host_plan_csr_bit_exact(golden, name, kind):
    from fea_b200 import _lib as L
    g = golden(name)
    N = g["X"].shape[0]
    mask = np.zeros(N, np.uint8)
    mask[np.unique(g["elems"])] = 7
    mask[g["fixed"]] = 0
    faces = g["pressure_faces"]
    hp = _plan(N, mask, [(kind, g["elems"])], [("T3" if faces.shape[1] == 3 else "Q4", faces)])
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDPTR), g["indptr"])
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDICES), g["indices"])
    assert hp.scalar(L.FEA_S_NDOF) == g["R"].shape[0]


@pytest.mark.parametrize("dofs", [(0,), (1, 2), (0, 2)])
def test_host_plan_partial_dirichlet_vs_oracle(dofs):
    from fea_b200 import _lib as L
    X, el = O.hex_block(3, jitter=0.1, seed=3)
    fixed = torch.nonzero(X[:, 0] < 1e-9).flatten().numpy()
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 10.0)], [], [(fixed, dofs)])
    R, (ip, ix, vv) = m.assemble(torch.zeros(int(m.free_mask().sum()), dtype=torch.float64))
    mask = np.full(X.shape[0], 7, np.uint8)
    for d in dofs:
        mask[fixed] &= ~np.uint8(1 << d)
    hp = _plan(X.shape[0], mask, [("C3D8", el.numpy())])
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDPTR), ip.numpy())
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDICES), ix.numpy())


def test_host_plan_mixed_groups_and_shared_nodes():
    """A tet block glued to a hex block: one pattern over both groups."""
    from fea_b200 import _lib as L
    Xh, eh = O.hex_block(2)
    Xt, et = O.tet_block(2)
    Xt = Xt + torch.tensor([1.0, 0.0, 0.0], dtype=torch.float64)
    # merge coincident nodes on x = 1
    key = lambda x: tuple(np.round(x, 9))
    ids = {key(x): i for i, x in enumerate(Xh.numpy())}
    Xall = list(Xh.numpy())
    remap = []
    for x in Xt.numpy():
        k = key(x)
        if k not in ids:
            ids[k] = len(Xall)
            Xall.append(x)
        remap.append(ids[k])
    et = torch.tensor(np.array(remap)[et.numpy()])
    X = torch.tensor(np.array(Xall))
    m = O.Model(X, [O.Group("C3D8", eh, 1.0, 5.0), O.Group("C3D4", et, 1.0, 5.0)], [], [])
    R, (ip, ix, vv) = m.assemble(torch.zeros(X.shape[0] * 3, dtype=torch.float64))
    hp = _plan(X.shape[0], np.full(X.shape[0], 7, np.uint8), [("C3D8", eh.numpy()), ("C3D4", et.numpy())])
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDPTR), ip.numpy())
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDICES), ix.numpy())


def test_host_plan_chunks_cover_all_nodes_and_incidences(golden):
    from fea_b200 import _lib as L
    g = golden("cfg1")
    N = g["X"].shape[0]
    mask = np.full(N, 7, np.uint8)
    hp = _plan(N, mask, [("C3D4", g["elems"])])
    cp = hp.array(L.G_BASE + L.A_CHUNKPTR)
    cl = hp.array(L.G_BASE + L.A_CHUNKLIST)
    ci = hp.array(L.G_BASE + L.A_CHUNKINC)
    ni = hp.array(L.G_BASE + L.A_NODEINC)
    dim = hp.array(L.G_BASE + L.A_CHUNKDIM).reshape(-1, 3)
    assert np.array_equal(cl, np.arange(N))          # every node listed once, in order
    assert cp[0] == 0 and cp[-1] == N and ci[0] == 0 and ci[-1] == ni[-1] == g["elems"].size
    assert np.all(np.diff(ci) <= hp.scalar(L.G_BASE + L.S_THREADS))
    assert np.all(ni[cl[cp[:-1]]] == ci[:-1])
    assert np.all(dim[:, 2] == 1)                    # all-free rows are contiguous
    assert dim[:, :2].sum(1).max() == hp.scalar(L.G_BASE + L.S_SMEM)
    inc = hp.array(L.G_BASE + L.A_INC)
    e, a = inc >> 4, inc & 15
    node = g["elems"][e, a]
    assert np.all(np.diff(node) >= 0)                 # incidences sorted by node
    boff = hp.array(L.G_BASE + L.A_BOFF).reshape(-1, 4)
    vbase = hp.array(L.FEA_A_VBASE)
    ip = hp.array(L.FEA_A_INDPTR)
    ix = hp.array(L.FEA_A_INDICES)
    rd = hp.array(L.FEA_A_RDOF)
    # every row offset addresses the column block of the element node in the CSR row
    for q in range(0, inc.size, 97):
        n = node[q]
        for b in range(4):
            c = g["elems"][e[q], b]
            assert ix[vbase[n] + boff[q, b]] == rd[c]


def test_face_chunks_list_only_surface_nodes(golden):
    from fea_b200 import _lib as L
    g = golden("hex5")
    N = g["X"].shape[0]
    mask = np.full(N, 7, np.uint8)
    mask[g["fixed"]] = 0
    faces = g["pressure_faces"]
    hp = _plan(N, mask, [("C3D8", g["elems"])], [("Q4", faces)])
    cl = hp.array(L.F_BASE + L.A_CHUNKLIST)
    np.testing.assert_array_equal(cl, np.unique(faces))
    assert hp.array(L.F_BASE + L.A_CHUNKINC)[-1] == faces.size


def test_plan_errors():
    from fea_b200 import _lib as L
    el = np.array([[0, 1, 2, 9]], np.int32)
    with pytest.raises(L.FeaError) as ex:
        _plan(4, np.full(4, 7, np.uint8), [("C3D4", el)])
    assert ex.value.status == -2
    # a node with more incidences than a chunk has threads
    X, el = O.tet_block(1)
    hub = np.array([[0, 1, 2, 3]] * 300, np.int32)
    with pytest.raises(L.FeaError) as ex:
        _plan(8, np.full(8, 7, np.uint8), [("C3D4", hub)])
    assert ex.value.status == -3
    # 64-bit node ids beyond int32 are out of range, not wrapped onto small ids
    wide = np.array([[0, 1, 2, 2 ** 32 + 3]], np.int64)
    with pytest.raises(L.FeaError) as ex:
        _plan(4, np.full(4, 7, np.uint8), [("C3D4", wide)])
    assert ex.value.status == -2
    with pytest.raises(L.FeaError) as ex:
        _plan(4, np.full(4, 7, np.uint8), [("C3D4", np.array([[0, 1, 2, 3]]))], [("T3", np.array([[0, 1, -1]]))])
    assert ex.value.status == -2


def test_header_constants_match_the_binding():
    """Every integer #define of the header has the same value in the binding."""
    from fea_b200 import _lib as L
    src = open(os.path.join(ROOT, "include", "fea_b200.h")).read()
    defs = dict(re.findall(r"^#define\s+(FEA_[A-Z0-9_]+)\s+(-?\d+)\b", src, flags=re.M))
    assert "FEA_PLAN_MAX_ELEMS" in defs and "FEA_ETOOBIG" in defs
    bound = {k: v for k, v in defs.items() if hasattr(L, k)}
    assert len(bound) >= 10
    assert all(getattr(L, k) == int(v) for k, v in bound.items()), \
        {k: (getattr(L, k), v) for k, v in bound.items() if getattr(L, k) != int(v)}


def test_plan_rejects_groups_beyond_the_incidence_code():
    """More than FEA_PLAN_MAX_ELEMS elements (faces) in one group: FEA_ETOOBIG
    before the connectivity is read (incidences e * 16 + a fit 32 bits)."""
    from fea_b200 import _lib as L
    conn = np.zeros(8, np.int32)
    mask = np.full(8, 7, np.uint8)
    h = ctypes.c_void_p()
    one = lambda t, *v: (t * 1)(*v)
    for ne, nf in ((L.FEA_PLAN_MAX_ELEMS + 1, 0), (1, L.FEA_PLAN_MAX_ELEMS + 1)):
        st = L.fea_plan_build(8, mask.ctypes.data, 1, one(ctypes.c_int32, L.FEA_C3D8), one(ctypes.c_int64, ne),
                              one(ctypes.c_void_p, conn.ctypes.data), 1, one(ctypes.c_int32, L.FEA_Q4),
                              one(ctypes.c_int64, nf), one(ctypes.c_void_p, conn.ctypes.data), 0, 0, ctypes.byref(h))
        assert st == L.FEA_ETOOBIG and not h.value
    assert (L.FEA_PLAN_MAX_ELEMS - 1) * 16 + 15 <= 2 ** 31 - 1 < L.FEA_PLAN_MAX_ELEMS * 16 + 16


def test_empty_group_and_fully_fixed_mesh():
    from fea_b200 import _lib as L
    hp = _plan(5, np.zeros(5, np.uint8), [("C3D4", np.zeros((0, 4), np.int32))])
    assert hp.scalar(L.FEA_S_NDOF) == 0 and hp.scalar(L.FEA_S_NNZ) == 0
    X, el = O.tet_block(1)
    hp = _plan(8, np.zeros(8, np.uint8), [("C3D4", el.numpy())])
    assert hp.scalar(L.FEA_S_NDOF) == 0 and hp.scalar(L.FEA_S_NNZ) == 0


def test_product_meshes_match_oracle_meshes():
    """The benchmark's mesh generators build the same meshes as the oracle's."""
    from fea_b200 import meshes
    for n in (1, 3):
        X, el = meshes.hex_block(n, jitter=0.1, seed=4)
        Xo, elo = O.hex_block(n, jitter=0.1, seed=4)
        np.testing.assert_array_equal(X, Xo.numpy())
        np.testing.assert_array_equal(el, elo.numpy())
        X, el = meshes.tet_block(n)
        Xo, elo = O.tet_block(n)
        np.testing.assert_array_equal(X, Xo.numpy())
        np.testing.assert_array_equal(el, elo.numpy())
    X, el = meshes.tet_block(2)
    sets, faces = meshes.plane_faces("C3D4", el, X, 2, 1.0)
    ref = O.boundary_faces("C3D4", torch.from_numpy(el), torch.from_numpy(X), 2, 1.0)
    np.testing.assert_array_equal(faces, torch.cat([f for _, _, f in ref]).numpy())


def _upper_staging(hp, el, mask):
    """The C3D8 staging arrays of a plan, the upper-block records decoded."""
    from fea_b200 import _lib as L
    arr = lambda i: hp.array(L.G_BASE + i)
    ub = arr(L.A_UBLK).reshape(-1, 4)
    return dict(nodeinc=arr(L.A_NODEINC), inc=arr(L.A_INC), incpos=arr(L.A_INCPOS).reshape(-1, 8),
                stagepos=arr(L.A_STAGEPOS).reshape(-1, 36), region=arr(L.A_REGION), uptr=arr(L.A_UPTR),
                stride=hp.scalar(L.FEA_S_G_HXSTRIDE, 0), maxval=hp.scalar(L.G_BASE + L.S_MAXVAL, 0),
                row=ub[:, 0], col=ub[:, 1], lc=ub[:, 2] & 0xFFFFFFFF, mc=ub[:, 2] >> 32,
                first=ub[:, 3] & 0xFFFFFFFF, count=ub[:, 3] >> 32,
                adjptr=hp.array(L.FEA_A_ADJPTR), adjcol=hp.array(L.FEA_A_ADJCOL),
                adjoff=hp.array(L.FEA_A_ADJOFF), moff=hp.array(L.FEA_A_MOFF))


def _slots():
    """(lane a, distance d, slot) of the element kernel: lane a computes K_ab,
    b = (a + d) mod 8, for d = 0..3 and d = 4 when a < 4."""
    out = []
    for a in range(8):
        for d in range(5 if a < 4 else 4):
            out.append((a, d, len(out)))
    return out


def _expected_contributions(el, mask):
    """Upper block (r, c) -> [(e, slot)] in staging order: the pair {i, j} of
    element e is counted once, from the incidence (e, i) of its lower node r
    (from i <= j when the element repeats the node), in ascending e, i, j."""
    slot = {}
    for a, d, s in _slots():
        slot[(a, (a + d) % 8)] = s
        slot[((a + d) % 8, a)] = s
    expect = {}
    for e in range(el.shape[0]):
        for i in range(8):
            r = el[e, i]
            if not mask[r]:
                continue
            for j in range(8):
                c = el[e, j]
                if mask[c] and (c > r or (c == r and j >= i)):
                    expect.setdefault((r, c), []).append((e, slot[(i, j)]))
    return expect


def _staging_case(golden, case):
    """(N, el, mask) of the packed-layout case (the hex5 fixture, partial
    masks) or of a fixed-layout case (a 16^3 structured block, one face
    clamped, part of it in x only)."""
    if case == "packed":
        g = golden("hex5")
        N, el = g["X"].shape[0], g["elems"]
        fixed = g["fixed"]
    else:
        X, el = O.hex_block(16, jitter=0.1, seed=3)
        N, el = X.shape[0], el.numpy()
        fixed = np.nonzero(X[:, 0].numpy() < 1e-9)[0]
    mask = np.full(N, 7, np.uint8)
    mask[fixed] = 0
    mask[fixed[:3]] = 5                               # partial masks too
    return N, el, mask


@pytest.mark.parametrize("case", ["packed", "fixed"])
def test_block_contributor_lists(golden, case):
    """Regions and upper-block records of the C3D8 staging: each node's
    region holds, block-major in adjacency order, the contributions to its
    upper blocks (n, c >= n) in ascending element order, regions start at
    even blocks (packed) or at n * stride (fixed, with 16 record slots per
    node and the residual slots at n * maxval); every element block of two
    active nodes has one staged position and the others none; the records
    carry the row and transpose targets (MOFF: n's value offset in row c)."""
    N, el, mask = _staging_case(golden, case)
    hp = _plan(N, mask, [("C3D8", el)])
    from fea_b200 import _lib as L
    vbase, rowlen = hp.array(L.FEA_A_VBASE), hp.array(L.FEA_A_ROWLEN)
    st = _upper_staging(hp, el, mask)
    expect = _expected_contributions(el, mask)
    sp, region, uptr, S = st["stagepos"], st["region"], st["uptr"], st["stride"]
    assert (S > 0) == (case == "fixed")
    seen = np.zeros(sp.shape, bool)
    for n in range(N):
        assert region[n] % 2 == 0
        if S:
            assert region[n] == n * S and uptr[n] == 16 * n
        u = uptr[n]
        t = 0
        for p in range(st["adjptr"][n], st["adjptr"][n + 1]):
            c = st["adjcol"][p]
            if c < n:
                continue
            assert st["row"][u] == vbase[n] + st["adjoff"][p]
            q = np.nonzero(st["adjcol"][st["adjptr"][c]:st["adjptr"][c + 1]] == n)[0][0] + st["adjptr"][c]
            assert st["moff"][p] == st["adjoff"][q]
            assert st["col"][u] == (vbase[c] + st["moff"][p] if c != n else -1)
            assert st["lc"][u] == rowlen[c] and st["mc"][u] == mask[c]
            lst = expect.get((n, c), [])
            assert st["first"][u] == t and st["count"][u] == len(lst)
            for k, (e, s) in enumerate(lst):
                assert sp[e, s] == region[n] + t + k
                seen[e, s] = True
            t += len(lst)
            u += 1
        if S:
            assert t <= S and u <= uptr[n] + 16
            assert np.all(st["row"][u:uptr[n] + 16] == -1) and np.all(st["col"][u:uptr[n] + 16] == -1)
        else:
            assert u == uptr[n + 1]
            assert region[n + 1] - region[n] == (t + 1) // 2 * 2
    assert np.all(sp[~seen] == -1) and np.all(sp[seen] >= 0)
    assert np.unique(sp[seen]).size == int(seen.sum())
    # residual slots: one per incidence of an active node, node by node
    inc, nodeinc, ip = st["inc"], st["nodeinc"], st["incpos"]
    for n in range(N):
        for k, q in enumerate(range(nodeinc[n], nodeinc[n + 1])):
            e, a = inc[q] >> 4, inc[q] & 15
            assert ip[e, a] == (n * st["maxval"] + k if S else q)


def test_face_chunks_take_one_warp_unless_a_node_has_more_faces():
    """Face lists are chunked by 32 incidences (one-warp CTAs), by 128 when a
    node lies on more than 32 faces: a fan of 40 triangles around one apex
    node of a tet fan."""
    from fea_b200 import _lib as L
    X, el = O.hex_block(2)
    N = X.shape[0]
    mask = np.full(N, 7, np.uint8)
    quads = el.numpy()[:, :4].astype(np.int32)                  # bottom faces of the elements
    hp = _plan(N, mask, [("C3D8", el.numpy())], [("Q4", quads)])
    assert hp.scalar(L.F_BASE + L.S_THREADS, 0) == 32
    M = 40
    apex, ring = 0, np.arange(1, M + 1)
    tets = np.stack([np.full(M, apex), ring, np.roll(ring, -1), np.full(M, M + 1)], 1).astype(np.int32)
    tris = tets[:, :3].copy()
    mask = np.full(M + 2, 7, np.uint8)
    hp = _plan(M + 2, mask, [("C3D4", tets)], [("T3", tris)])
    assert hp.scalar(L.F_BASE + L.S_THREADS, 0) == 128


def test_serving_requests_are_seeded_and_bounded():
    from fea_b200 import meshes, serving
    a = serving.make_requests(20, 5.0, seed=3)
    b = serving.make_requests(20, 5.0, seed=3)
    assert [vars(x) for x in a] == [vars(x) for x in b]
    assert all(4 <= r.length <= 16 and 1 <= r.width <= 2 and 1 <= r.height <= 2 for r in a)
    assert all(2000 <= r.n_elems <= 200000 and abs(r.kappa - 20 * r.mu) < 1e-12 for r in a)
    assert all(0.005 <= r.pressure <= 0.05 for r in a)
    assert all(serving.load_parameter(r.length, r.width, r.height, r.mu, r.kappa, r.pressure)
               <= serving.STABLE_LOAD for r in a)
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    for r in a[:4]:
        X, el = meshes.tet_beam(r.length, r.width, r.height, r.n_elems)
        assert serving.request_rows(r) == 3 * X.shape[0]
        assert 0.5 * r.n_elems <= el.shape[0] <= 2.0 * r.n_elems
        assert abs(X[:, 0].max() - 1.0) < 1e-12 and abs(X[:, 0].min() - (1.0 - r.length)) < 1e-9


def _hand_csr(n, free):
    """CSR of an n^3 C3D8 block built from the neighbour rule alone: nodes
    (i,j,k) and (i',j',k') share an element iff every index differs by at
    most 1; DOFs numbered in node order over the free ones."""
    N = (n + 1) ** 3
    ijk = [(i // (n + 1) ** 2, i // (n + 1) % (n + 1), i % (n + 1)) for i in range(N)]
    dof = {}
    for a in range(N):
        for d in range(3):
            if free[a][d]:
                dof[(a, d)] = len(dof)
    indptr, indices = [0], []
    for a in range(N):
        for d in range(3):
            if not free[a][d]:
                continue
            cols = sorted(dof[(c, e)] for c in range(N) for e in range(3)
                          if free[c][e] and all(abs(p - q) <= 1 for p, q in zip(ijk[a], ijk[c])))
            indices += cols
            indptr.append(len(indices))
    return np.array(indptr), np.array(indices)


@pytest.mark.parametrize("clamp", [False, True])
def test_csr_of_eight_hex_mesh_by_hand(clamp):
    """2x2x2 C3D8 block (8 elements, 27 nodes): all free, 8 corner nodes
    couple to 8 nodes, 12 edge nodes to 12, 6 face nodes to 18 and the centre
    to 27, so nnz = 9 (64 + 144 + 108 + 27) = 3087; with x = 0 clamped the
    9 nodes there drop out of rows and columns."""
    from fea_b200 import _lib as L
    X, el = O.hex_block(2)
    N = X.shape[0]
    fixed = np.nonzero(X[:, 0].numpy() < 1e-9)[0] if clamp else np.zeros(0, np.int64)
    free = [[i not in set(fixed.tolist())] * 3 for i in range(N)]
    ip, ix = _hand_csr(2, free)
    if not clamp:
        assert ip[-1] == 3087 and len(ip) == 82
    else:
        assert len(ip) == 3 * 18 + 1
    mask = np.full(N, 7, np.uint8)
    mask[fixed] = 0
    hp = _plan(N, mask, [("C3D8", el.numpy())])
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDPTR), ip)
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDICES), ix)
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 10.0)], [], [(fixed, (0, 1, 2))] if clamp else [])
    _, (oip, oix, _) = m.assemble(torch.zeros(int(m.free_mask().sum()), dtype=torch.float64))
    np.testing.assert_array_equal(oip.numpy(), ip)
    np.testing.assert_array_equal(oix.numpy(), ix)


@pytest.mark.parametrize("n,dofs,collapse", [(3, (0, 1, 2), False), (3, (1,), False), (3, (0, 1, 2), True),
                                             (14, (0, 2), False)])
def test_upper_staging_emulated_gives_reference_K(n, dofs, collapse):
    """The C3D8 assembly as the kernels perform it, emulated on the CPU with
    the oracle's element blocks: each element block written to its staged
    position, oriented to its upper node block, then per node the upper
    block sums into the node's rows and their transposes into the column
    nodes' rows.  The CSR values equal the oracle's reduced K
    and R; also with a collapsed element (two of its corners one node), whose
    repeated node puts two blocks of the element on the diagonal, and on a
    14^3 block, which takes the fixed layout."""
    from fea_b200 import _lib as L
    X, el = O.hex_block(n, jitter=0.1, seed=5)
    if collapse:
        el = el.clone()
        el[13, 6] = el[13, 7]                   # the centre element's top edge 6-7 collapsed
    fixed = torch.nonzero(X[:, 0] < 1e-9).flatten().numpy()
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 10.0)], [], [(fixed, dofs)])
    nfree = int(m.free_mask().sum())
    gc = 0.01 * torch.randn(nfree, generator=torch.Generator().manual_seed(2), dtype=torch.float64)
    Rref, (ip, ix, vref) = m.assemble(gc)
    N = X.shape[0]
    mask = np.full(N, 7, np.uint8)
    for d in dofs:
        mask[fixed] &= ~np.uint8(1 << d)
    el = el.numpy()
    hp = _plan(N, mask, [("C3D8", el)])
    st = _upper_staging(hp, el, mask)
    vbase, rowlen, rdof = hp.array(L.FEA_A_VBASE), hp.array(L.FEA_A_ROWLEN), hp.array(L.FEA_A_RDOF)
    Re, Ke = O.element_residual_tangent("C3D8", X, torch.from_numpy(el), m.gc_to_u(gc), 1.0, 10.0)
    Re, Ke = Re.numpy(), Ke.numpy()                    # [a,j,e], [a,j,b,k,e]
    S, Q = st["stride"], st["maxval"]
    assert (S > 0) == (n == 14)
    blocks = np.full((int(st["region"][-1]), 3, 3), np.nan)
    rslot = np.full((N * Q if S else int(st["nodeinc"][-1]), 3), np.nan)
    for e in range(el.shape[0]):                       # element kernel, phase 3
        for a, d, s in _slots():
            pos = st["stagepos"][e, s]
            if pos < 0:
                continue
            b = (a + d) % 8
            Kab = Ke[a, :, b, :, e]
            if d == 0 or el[e, b] > el[e, a]:
                blocks[pos] = Kab
            elif el[e, b] < el[e, a]:
                blocks[pos] = Kab.T
            else:
                blocks[pos] = Kab + Kab.T
        for a in range(8):
            if st["incpos"][e, a] >= 0:
                rslot[st["incpos"][e, a]] = Re[a, :, e]
    K = np.full(int(vbase[-1]), np.nan)
    R = np.full(nfree, np.nan)
    free = lambda mk: [j for j in range(3) if mk >> j & 1]
    for n in range(N):                                  # gather, one lane group per node
        if not mask[n]:
            continue
        Sn = blocks[st["region"][n]:st["region"][n + 1]]
        for u in range(st["uptr"][n], st["uptr"][n + 1]):
            if st["row"][u] < 0:                        # unused record slot (fixed layout)
                break
            f, cnt, mc = st["first"][u], st["count"][u], st["mc"][u]
            blk = np.zeros((3, 3))
            for t in range(f, f + cnt):
                blk = blk + Sn[t]
            for rj, j in enumerate(free(mask[n])):
                for rk, k in enumerate(free(mc)):
                    K[st["row"][u] + rj * rowlen[n] + rk] = blk[j, k]
            if st["col"][u] >= 0:
                for rk, k in enumerate(free(mc)):
                    for cj, j in enumerate(free(mask[n])):
                        K[st["col"][u] + rk * st["lc"][u] + cj] = blk[j, k]
            else:
                nq = st["nodeinc"][n + 1] - st["nodeinc"][n]
                r0 = n * Q if S else st["nodeinc"][n]
                r = rslot[r0:r0 + nq].sum(0)
                for rr, j in enumerate(free(mask[n])):
                    R[rdof[n] + rr] = r[j]
    assert not np.isnan(K).any() and not np.isnan(R).any()
    np.testing.assert_array_equal(hp.array(L.FEA_A_INDPTR), ip.numpy())
    np.testing.assert_allclose(K, vref.numpy(), rtol=0, atol=1e-13 * np.abs(vref.numpy()).max())
    np.testing.assert_allclose(R, Rref.numpy(), rtol=0, atol=1e-13 * np.abs(Rref.numpy()).max())


def test_nvtx_ranges_are_opt_in():
    """FEA_B200_NVTX=1 turns the host-side NVTX ranges on; unset, they cost
    nothing and push nothing."""
    import subprocess
    import sys
    code = ("import fea_b200._trace as t\n"
            "with t.nvtx('fea.test'):\n"
            "    pass\n"
            "print(int(t.ENABLED))\n")
    env = dict(os.environ, FEA_B200_NVTX="1")
    on = subprocess.run([sys.executable, "-c", code], env=env, cwd=ROOT, capture_output=True, text=True)
    env.pop("FEA_B200_NVTX")
    off = subprocess.run([sys.executable, "-c", code], env=env, cwd=ROOT, capture_output=True, text=True)
    assert on.returncode == 0 and on.stdout.strip() == "1"
    assert off.returncode == 0 and off.stdout.strip() == "0"


def test_missing_library_fails_loudly_with_the_build_command(tmp_path):
    """Without libfea_b200.so the package import raises ImportError (no
    fallback), naming the build script to run by path."""
    import shutil
    import subprocess
    import sys
    pkg = tmp_path / "fea_b200"
    pkg.mkdir()
    for f in os.listdir(os.path.join(ROOT, "fea_b200")):
        if f.endswith(".py"):
            shutil.copy(os.path.join(ROOT, "fea_b200", f), pkg / f)
    r = subprocess.run([sys.executable, "-c", "import fea_b200"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode != 0
    last = r.stderr.strip().splitlines()[-1]
    assert last.startswith("ImportError: fea_b200: native library")
    assert "python " + str(pkg / "_build.py") in last
