"""Seeded synthetic meshes for the benchmark workloads.

- hex_block: structured C3D8 block, nodes optionally jittered by U(-j h, j h)
  (the 64^3 jittered block of the assembly benchmark).
- tet_block: every hex cell Kuhn-split into 6 positively oriented C3D4 (the
  unit-cube and explicit-dynamics workloads).
- plane_faces: element faces lying on a coordinate plane, as surface-set
  entries (element labels, face id) plus the face node lists.
- tet_beam: a Kuhn-split box of about a given number of C3D4 elements with
  near-cubic cells (the serving workload's cantilevers).
Node numbering is (i, j, k) lexicographic with k fastest.
"""
from __future__ import annotations

import numpy as np

from .elements import FACES


def grid_nodes(nx, ny, nz, lengths=(1.0, 1.0, 1.0)):
    g = [np.linspace(0.0, L, n + 1) for L, n in zip(lengths, (nx, ny, nz))]
    X, Y, Z = np.meshgrid(*g, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)


def _ids(nx, ny, nz):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    return i.ravel(), j.ravel(), k.ravel(), (lambda a, b, c: (a * (ny + 1) + b) * (nz + 1) + c)


def hex_block(n, jitter=0.0, seed=0, dims=None, lengths=(1.0, 1.0, 1.0)):
    nx, ny, nz = dims if dims is not None else (n, n, n)
    X = grid_nodes(nx, ny, nz, lengths)
    if jitter:
        h = np.array([lengths[0] / nx, lengths[1] / ny, lengths[2] / nz])
        X = X + np.random.default_rng(seed).uniform(-1, 1, X.shape) * jitter * h
    i, j, k, f = _ids(nx, ny, nz)
    el = np.stack([f(i, j, k), f(i + 1, j, k), f(i + 1, j + 1, k), f(i, j + 1, k),
                   f(i, j, k + 1), f(i + 1, j, k + 1), f(i + 1, j + 1, k + 1), f(i, j + 1, k + 1)], 1)
    return X, el.astype(np.int64)


def tet_block(n, dims=None, lengths=(1.0, 1.0, 1.0)):
    nx, ny, nz = dims if dims is not None else (n, n, n)
    X = grid_nodes(nx, ny, nz, lengths)
    i, j, k, f = _ids(nx, ny, nz)
    step = {1: (1, 0, 0), 2: (0, 1, 0), 4: (0, 0, 1)}
    tets = []
    for path in [(1, 2, 4), (1, 4, 2), (2, 1, 4), (2, 4, 1), (4, 1, 2), (4, 2, 1)]:
        c = np.zeros(3, dtype=np.int64)
        t = [f(i, j, k)]
        for s in path:
            c = c + np.array(step[s])
            t.append(f(i + c[0], j + c[1], k + c[2]))
        tets.append(np.stack(t, 1))
    el = np.stack(tets, 1).reshape(-1, 4)
    x = X[el]
    vol = np.einsum("ei,ei->e", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]), x[:, 3] - x[:, 0])
    neg = vol < 0
    el[neg] = el[neg][:, [0, 2, 1, 3]]
    return X, el.astype(np.int64)


def plane_faces(kind, elems, X, axis, value, tol=1e-9):
    """[(element positions, face id)] and the concatenated face node lists."""
    on = np.abs(X[:, axis] - value) < tol
    sets, faces = [], []
    for fid, loc in FACES[kind].items():
        fn = elems[:, loc]
        m = on[fn].all(axis=1)
        if m.any():
            sets.append((np.nonzero(m)[0], fid))
            faces.append(fn[m])
    return sets, (np.concatenate(faces) if faces else np.zeros((0, len(FACES[kind][0])), np.int64))


def beam_dims(length, width, height, n_elems):
    """Cells per side of tet_beam: about n_elems / 6 cells, as cubic as possible."""
    cells = max(1.0, n_elems / 6.0)
    s = (cells / (length * width * height)) ** (1.0 / 3.0)
    return tuple(max(1, int(round(v * s))) for v in (length, width, height))


def tet_beam(length, width, height, n_elems):
    """C3D4 mesh of [1 - length, 1] x [-width/2, width/2] x [-height/2, height/2]
    with about n_elems elements (6 per cell, cells as close to cubes as the
    counts allow).  The free end x = 1 lies close to the origin but not
    through it: the enclosed-volume pressure load inverts [x, x_xi, x_eta]
    per face, which is singular for a face whose plane holds the origin."""
    dims = beam_dims(length, width, height, n_elems)
    X, el = tet_block(0, dims=dims, lengths=(length, width, height))
    X = X - np.array([length - 1.0, width / 2.0, height / 2.0])
    return X, el
