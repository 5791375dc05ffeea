"""The host side of the adjoint linear solve (wcns_b200.adjoint): restarted,
right-preconditioned GMRES on small dense systems, including one whose
preconditioned Richardson iteration -- the form of wcns_adjoint_iterate --
grows, and the face mask of the physical-boundary regions."""
import numpy as np

from wcns_b200 import adjoint, cases


def _system(n, seed, shift):
    rng = np.random.default_rng(seed)
    a = np.eye(n) * shift + rng.standard_normal((n, n)) / np.sqrt(n)
    return a


def test_gmres_solves_a_nonsymmetric_system():
    a = _system(120, 1, 3.0)
    m = np.diag(1.0 / np.diag(a))
    b = np.random.default_rng(2).standard_normal(120)
    x, hist = adjoint.gmres(lambda v: a @ v, lambda v: m @ v, b, restart=20, tol=1e-11, maxiter=400)
    assert hist[-1] <= 1e-11
    np.testing.assert_allclose(a @ x, b, rtol=0, atol=1e-9 * np.linalg.norm(b))


def test_gmres_converges_where_richardson_grows():
    """x <- x + M (b - A x) grows when an eigenvalue of I - M A lies
    outside the unit disc; GMRES with the same M and A converges."""
    n = 60
    rng = np.random.default_rng(3)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.linspace(0.2, 1.5, n)
    lam[-1] = 2.3  # 1 - 2.3 = -1.3: Richardson with M = I grows
    a = q @ np.diag(lam) @ q.T + 0.05 * rng.standard_normal((n, n)) / np.sqrt(n)
    ident = lambda v: v
    b = rng.standard_normal(n)
    x = np.zeros(n)
    for _ in range(200):
        x = x + (b - a @ x)
    assert np.linalg.norm(b - a @ x) > np.linalg.norm(b)
    x, hist = adjoint.gmres(lambda v: a @ v, ident, b, restart=30, tol=1e-10, maxiter=300)
    assert hist[-1] <= 1e-10
    np.testing.assert_allclose(a @ x, b, rtol=0, atol=1e-8 * np.linalg.norm(b))


def test_gmres_zero_right_hand_side():
    x, hist = adjoint.gmres(lambda v: 2.0 * v, lambda v: v, np.zeros(5))
    assert np.all(x == 0.0) and hist == [0.0]


def test_face_mask_zeroes_the_physical_faces_only():
    case = cases.vortex_case(ni=25, nj=13, nk=9, nsteps=1)  # x, z periodic; y far field
    keep = adjoint.face_mask(case)[0]
    assert keep.shape == (9, 13, 25)
    assert np.all(keep[:, 0, :] == 0.0) and np.all(keep[:, -1, :] == 0.0)
    assert np.all(keep[:, 1:-1, :] == 1.0)
    plate = cases.small_plate_case()
    masks = adjoint.face_mask(plate)
    assert [m.shape for m in masks] == [(nk, nj, ni) for ni, nj, nk in plate.dims]
    assert all(0.0 < m.mean() < 1.0 for m in masks)
