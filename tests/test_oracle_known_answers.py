"""Known-answer checks of the oracle itself (CPU): rigid rotation, the
closed-form uniaxial Neo-Hookean stress, the patch test on a jittered C3D8
block, the lumped mass total rho * volume, and R and K as central
differences of the energy and of R.  The same checks run through the CUDA
path in test_gpu_parity.py."""
import numpy as np
import pytest
import torch

from oracle import fea_oracle as O

MU, KAPPA = 1.3, 20.0


def _block(kind, n, jitter=0.0, rho=1.0):
    X, el = O.hex_block(n, jitter=jitter, seed=9) if kind == "C3D8" else O.tet_block(n)
    return O.Model(X, [O.Group(kind, el, MU, KAPPA, rho)], [], [])


def rotation(a=0.7, b=0.3):
    c, s = np.cos(a), np.sin(a)
    Qz = torch.tensor([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]], dtype=torch.float64)
    c, s = np.cos(b), np.sin(b)
    Qx = torch.tensor([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]], dtype=torch.float64)
    return Qz @ Qx


def uniaxial_P11(lam, mu=MU, kappa=KAPPA):
    """P11 of W = mu/2 (J^-2/3 I1 - 3) + kappa/2 (J-1)^2 at F = diag(lam, 1, 1):
    dW/dF11 = mu J^-2/3 (lam - I1 / (3 J)) + kappa (J - 1) with J = lam, I1 = lam^2 + 2."""
    return mu * lam ** (-2.0 / 3.0) * (lam - (lam ** 2 + 2.0) / (3.0 * lam)) + kappa * (lam - 1.0)


def uniaxial_W(lam, mu=MU, kappa=KAPPA):
    return mu / 2 * (lam ** (-2.0 / 3.0) * (lam ** 2 + 2.0) - 3.0) + kappa / 2 * (lam - 1.0) ** 2


def interior_nodes(n):
    i = np.arange((n + 1) ** 3)
    ijk = np.stack([i // (n + 1) ** 2, i // (n + 1) % (n + 1), i % (n + 1)], 1)
    return torch.from_numpy(np.all((ijk > 0) & (ijk < n), axis=1))


PATCH_F = [[1.04, 0.02, -0.01], [0.015, 0.97, 0.03], [-0.02, 0.01, 1.02]]


@pytest.mark.parametrize("kind", ["C3D8", "C3D4"])
def test_rigid_rotation_zero_residual(kind):
    m = _block(kind, 3, jitter=0.1 if kind == "C3D8" else 0.0)
    u = m.X @ rotation().T - m.X
    R, _ = m.assemble(u.reshape(-1), want_K=False)
    assert float(R.abs().max()) < 1e-13
    assert abs(float(m.energy(u.reshape(-1)))) < 1e-13


@pytest.mark.parametrize("kind", ["C3D8", "C3D4"])
def test_uniaxial_stretch_closed_form(kind):
    lam = 1.05
    m = _block(kind, 3)
    u = torch.zeros_like(m.X)
    u[:, 0] = (lam - 1.0) * m.X[:, 0]
    R, _ = m.assemble(u.reshape(-1), want_K=False)
    R = R.reshape(-1, 3)
    P11 = uniaxial_P11(lam)
    face = (m.X[:, 0] - 1.0).abs() < 1e-12
    assert abs(float(R[face, 0].sum()) - P11) < 1e-12 * P11
    assert abs(float(R[:, 0].sum())) < 1e-12 * P11
    assert abs(float(m.energy(u.reshape(-1))) - uniaxial_W(lam)) < 1e-12 * uniaxial_W(lam)


def test_patch_test_jittered_c3d8():
    n = 4
    m = _block("C3D8", n, jitter=0.15)
    u = m.X @ torch.tensor(PATCH_F, dtype=torch.float64).T - m.X
    R, _ = m.assemble(u.reshape(-1), want_K=False)
    R = R.reshape(-1, 3)
    scale = float(R.abs().max())
    assert scale > 1e-3
    assert float(R[interior_nodes(n)].abs().max()) < 1e-12 * scale


@pytest.mark.parametrize("kind", ["C3D8", "C3D4"])
def test_lumped_mass_totals_rho_volume(kind):
    rho = 2.5
    m = _block(kind, 3, jitter=0.1 if kind == "C3D8" else 0.0, rho=rho)
    mass = (1.0 / m.lumped_mass_inv()).reshape(-1, 3)
    _, w, _ = O.preload_gaussian(kind, m.X, m.groups[0].elems)
    vol = float(w.sum())
    assert abs(vol - 1.0) < 0.05
    for d in range(3):
        assert abs(float(mass[:, d].sum()) - rho * vol) < 1e-12 * rho * vol


@pytest.mark.parametrize("kind", ["C3D8", "C3D4"])
def test_residual_and_tangent_are_derivatives(kind):
    """At a finite-strain state, the central difference (h = 1e-6) of the
    energy along a random direction d equals R . d, and that of R equals K d."""
    m = _block(kind, 2, jitter=0.1 if kind == "C3D8" else 0.0)
    g = torch.Generator().manual_seed(3)
    u = 0.05 * torch.randn(m.X.shape, generator=g, dtype=torch.float64).reshape(-1)
    d = torch.randn(u.shape, generator=g, dtype=torch.float64)
    R, (ip, ix, v) = m.assemble(u)
    h = 1e-6
    dE = float(m.energy(u + h * d) - m.energy(u - h * d)) / (2 * h)
    assert abs(dE - float((R * d).sum())) < 1e-8 * abs(dE)
    Kd = O.csr_matvec(ip, ix, v, d)
    fd = (m.assemble(u + h * d, want_K=False)[0] - m.assemble(u - h * d, want_K=False)[0]) / (2 * h)
    assert float((fd - Kd).norm()) < 1e-8 * float(Kd.norm())


@pytest.mark.parametrize("name,kind", [("tet3", "C3D4"), ("hex5", "C3D8")])
def test_tangent_with_follower_pressure_is_derivative(golden, name, kind):
    """The same check on the committed fixtures, whose follower pressure adds
    its own, unsymmetric, part to R and K."""
    from tests.helpers import oracle_model
    g = golden(name)
    m = oracle_model(g, kind)
    x = torch.from_numpy(g["state"])
    d = torch.randn(x.shape, generator=torch.Generator().manual_seed(5), dtype=torch.float64)
    _, (ip, ix, v) = m.assemble(x)
    Kd = O.csr_matvec(ip, ix, v, d)
    h = 1e-6
    fd = (m.assemble(x + h * d, want_K=False)[0] - m.assemble(x - h * d, want_K=False)[0]) / (2 * h)
    assert float((fd - Kd).norm()) < 1e-8 * float(Kd.norm())


@pytest.mark.parametrize("name", ["cfg1", "tet3", "hex5"])
def test_node_level_pattern_matches_reference_csr(golden, name):
    """The node-level restatement of the pattern (used where the DOF-level
    sort is too large) gives the reference's reduced CSR bit for bit."""
    g = golden(name)
    N = g["X"].shape[0]
    free = np.zeros((N, 3), dtype=bool)
    free[np.unique(g["elems"])] = True
    free[np.asarray(g["fixed"], dtype=np.int64)] = False
    ip, ix = O.reduced_pattern_csr([g["elems"]], free, N)
    np.testing.assert_array_equal(ip, g["indptr"])
    np.testing.assert_array_equal(ix, g["indices"])


@pytest.mark.parametrize("dofs", [(0, 1, 2), (2,), (0, 2)])
def test_node_level_pattern_matches_oracle_with_partial_bcs(dofs):
    X, el = O.hex_block(3, jitter=0.1, seed=4)
    Xt, et = O.tet_block(2)
    et = et + X.shape[0]                                  # a second group on nodes of its own
    Xa = torch.cat([X, Xt + 2.0])
    fixed = np.arange(0, Xa.shape[0], 5)
    m = O.Model(Xa, [O.Group("C3D8", el, 1.0, 50.0), O.Group("C3D4", et, 1.0, 10.0)], [], [(fixed, dofs)])
    R, (ip, ix, v) = m.assemble(torch.zeros(int(m.free_mask().sum()), dtype=torch.float64))
    ip2, ix2 = O.reduced_pattern_csr([el.numpy(), et.numpy()], m.free_mask().numpy(), Xa.shape[0])
    np.testing.assert_array_equal(ip2, ip.numpy())
    np.testing.assert_array_equal(ix2, ix.numpy())
