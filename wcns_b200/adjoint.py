"""The adjoint linear solve of the inviscid residual, by restarted GMRES.

The device iteration `wcns_adjoint_iterate` is a Richardson iteration,
psi <- psi + Z P^T Z (r_Q^T psi + g): r is the inviscid residual (the step's
dq, +dF), r_Q its Jacobian with respect to the conserved variables at the
interior points, P one LU-SGS pair (lusgs_l then lusgs_u, LHS.f90:381-577)
and Z the mask that zeroes the points of physical-boundary faces as
set_nonconnect_boundary_dq_0 (CIC.f90:2-17) does.  Where the linearised step
of that pair has a spectral radius at or just above one, the iteration stalls
or grows.  GMRES does not need a contraction: it solves

    Z r_Q^T Z psi = -Z g

with the same operators, right-preconditioned by M = Z P^T Z, and needs only
that the preconditioned operator is nonsingular on the masked space.  (On a
fully periodic block it is not: a conservative difference sums to zero over
the block, so constant adjoints are in the null space and g must be
orthogonal to them.)

Every operator application runs on the device through the C ABI
(`wcns_rhs_invis_adjoint` with the interface ghosts folded,
`wcns_lusgs_operator` transposed); the Krylov vectors live in host memory,
one flat float64 vector over the blocks' five interior arrays.  The context
must hold the linearisation point with its ghosts, time step and spectral
radii (the phases boundary_all, initial_q_dq_c_t and timestep_tgh), as
`wcns_adjoint_iterate` prepares them.
"""
from __future__ import annotations

import numpy as np

from .cases import GAMMA, Case


def face_mask(case: Case):
    """Per block an array (nk, nj, ni): 0 at the points of faces whose
    boundary region is physical (bctype > 0), 1 elsewhere -- the points
    whose dq the step keeps."""
    out = []
    for nb, (ni, nj, nk) in enumerate(case.dims, start=1):
        keep = np.ones((nk, nj, ni))
        for rec in case.regions[case.regions[:, 0] == nb]:
            if rec[7] <= 0:
                continue
            (i0, i1), (j0, j1), (k0, k1) = (sorted((abs(int(rec[1 + 2 * a])), abs(int(rec[2 + 2 * a])))) for a in range(3))
            keep[k0 - 1:k1, j0 - 1:j1, i0 - 1:i1] = 0.0
        out.append(keep)
    return out


class AdjointSystem:
    """The masked adjoint operator and its preconditioner on a context `g`
    (a solver.Wcns) of `case`, on flat vectors of 5 x (interior points) per
    block, block after block."""

    def __init__(self, g, case: Case):
        self.g, self.case = g, case
        self.dims = list(case.dims)
        self.keep = face_mask(case)
        self.sizes = [5 * ni * nj * nk for ni, nj, nk in self.dims]
        self.n = int(sum(self.sizes))
        self.mask = np.concatenate([np.tile(k.ravel(), 5) for k in self.keep])
        # the linearisation point's r, u, v, w at the interior points
        self.prim = [[self._interior([g.get(f, nb)], nb)[0] for f in ("r", "u", "v", "w")]
                     for nb in range(1, len(self.dims) + 1)]

    # flat vector <-> per block ghosted arrays
    def _split(self, v):
        out, o = [], 0
        for (ni, nj, nk), s in zip(self.dims, self.sizes):
            out.append(v[o:o + s].reshape(5, nk, nj, ni))
            o += s
        return out

    def _ghosted(self, a5, nb):
        ni, nj, nk = self.dims[nb - 1]
        out = []
        for m in range(5):
            b = np.zeros((nk + 6, nj + 6, ni + 6))
            b[3:3 + nk, 3:3 + nj, 3:3 + ni] = a5[m]
            out.append(b)
        return out

    def _interior(self, arrs, nb):
        ni, nj, nk = self.dims[nb - 1]
        return np.stack([a[3:3 + nk, 3:3 + nj, 3:3 + ni] for a in arrs])

    def _to_conserved(self, qbar, nb):
        """(d prim / d Q)^T qbar at the block's interior points (the
        transform of `wcns_adjoint_iterate`, prim = (r, u, v, w, p))."""
        r, u, v, w = self.prim[nb - 1]
        g1 = GAMMA - 1.0
        return np.stack([qbar[0] - (u * qbar[1] + v * qbar[2] + w * qbar[3]) / r + 0.5 * g1 * (u * u + v * v + w * w) * qbar[4],
                         qbar[1] / r - g1 * u * qbar[4], qbar[2] / r - g1 * v * qbar[4], qbar[3] / r - g1 * w * qbar[4],
                         g1 * qbar[4]])

    def apply_a(self, v):
        """Z r_Q^T Z v."""
        v = v * self.mask
        for nb, a5 in enumerate(self._split(v), start=1):
            self.g.adj_set("lam", nb, self._ghosted(a5, nb))
        self.g.rhs_invis_adjoint(fold=True)
        out = [self._to_conserved(self._interior(self.g.adj_get("qbar", nb), nb), nb).ravel()
               for nb in range(1, len(self.dims) + 1)]
        return np.concatenate(out) * self.mask

    def apply_m(self, v):
        """Z P^T Z v."""
        v = v * self.mask
        for nb, a5 in enumerate(self._split(v), start=1):
            self.g.adj_set("b", nb, self._ghosted(a5, nb))
        self.g.lusgs_operator(transpose=True)
        out = [self._interior(self.g.adj_get("x", nb), nb).ravel() for nb in range(1, len(self.dims) + 1)]
        return np.concatenate(out) * self.mask

    def flatten(self, per_block):
        """Per block five arrays (nk, nj, ni) -> a flat vector."""
        return np.concatenate([np.stack(a5).ravel() for a5 in per_block])

    def unflatten(self, v):
        return [list(a) for a in self._split(v)]


def gmres(apply_a, apply_m, b, restart=30, tol=1e-8, maxiter=600):
    """Right-preconditioned restarted GMRES for A x = b with x = M y:
    Arnoldi with modified Gram-Schmidt and Givens rotations.  Returns (x,
    relative residual norms ||b - A x|| / ||b||, one per inner iteration)."""
    n = b.shape[0]
    x = np.zeros(n)
    bnorm = float(np.linalg.norm(b))
    hist = []
    if bnorm == 0.0:
        return x, [0.0]
    r = b.copy()
    it = 0
    while it < maxiter:
        beta = float(np.linalg.norm(r))
        if beta / bnorm <= tol:
            break
        V = np.zeros((restart + 1, n))
        Z = np.zeros((restart, n))
        H = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        s = np.zeros(restart + 1)
        s[0] = beta
        V[0] = r / beta
        k_done = 0
        for k in range(restart):
            Z[k] = apply_m(V[k])
            w = apply_a(Z[k])
            for j in range(k + 1):
                H[j, k] = float(np.dot(w, V[j]))
                w = w - H[j, k] * V[j]
            H[k + 1, k] = float(np.linalg.norm(w))
            if H[k + 1, k] > 0.0:
                V[k + 1] = w / H[k + 1, k]
            for j in range(k):  # earlier rotations on the new column
                t = cs[j] * H[j, k] + sn[j] * H[j + 1, k]
                H[j + 1, k] = -sn[j] * H[j, k] + cs[j] * H[j + 1, k]
                H[j, k] = t
            den = np.hypot(H[k, k], H[k + 1, k])
            cs[k], sn[k] = (1.0, 0.0) if den == 0.0 else (H[k, k] / den, H[k + 1, k] / den)
            H[k, k] = den
            H[k + 1, k] = 0.0
            s[k + 1] = -sn[k] * s[k]
            s[k] = cs[k] * s[k]
            it += 1
            k_done = k + 1
            hist.append(abs(s[k + 1]) / bnorm)
            if hist[-1] <= tol or it >= maxiter:
                break
        y = np.linalg.solve(np.triu(H[:k_done, :k_done]), s[:k_done]) if k_done else np.zeros(0)
        x = x + y @ Z[:k_done]
        r = b - apply_a(x)
        hist[-1] = float(np.linalg.norm(r)) / bnorm  # the true residual at the restart
    return x, hist


def solve(g, case: Case, gvec, restart=30, tol=1e-8, maxiter=600):
    """psi with Z r_Q^T Z psi = -Z g: `gvec` per block five arrays (nk, nj,
    ni) of the objective's gradient with respect to the conserved variables;
    returns (psi per block, relative residual history)."""
    S = AdjointSystem(g, case)
    b = -S.flatten(gvec) * S.mask
    x, hist = gmres(S.apply_a, S.apply_m, b, restart=restart, tol=tol, maxiter=maxiter)
    return S.unflatten(x), hist
