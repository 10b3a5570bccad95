"""The algebra of the shifted energy scan, on the CPU against the oracle (no device code).

Between the energies of one J-pi block the R-matrix C(E) of the oracle's own assembly
(src/rmatrix_hp.F90:246-293) changes only by a common shift of its diagonal and by the closed
channels' Bloch terms:
    C(E) = C0 + delta(E) I + Q D(E) Q^T,   Q = blockdiag(q2),
with C0 the assembly at the first energy without Bloch terms, delta the common change of the
channels' diagonal energy terms (-k^2 open, +k^2 closed), D = diag(-xc_c / a) over the closed
channels, and the mesh's Bloch matrix equal to q2 q2^T.  With C0 = P H P^H (Hessenberg form),
    Y = (H + delta I)^-1 P^H Q,  S = Q^T P Y,  T = I - D (I + S D)^-1 S,  R = S T,
which is Q^T C(E)^-1 Q; U follows as for the LU path.  The library's shifted scan forms delta
and D on the host this way and evaluates these expressions on the device (hessenberg.cuh).
"""
import numpy as np
import scipy.linalg

from hprmat_b200 import workloads
from oracle import rmatrix_oracle as orc

NR, RMAX = 30, 20.0


def _hess_solve(H, delta, Z):
    """(H + delta I)^-1 Z as hess_solve_kernel computes it: elimination down the rows with a
    working row, pivoting between the working row and the next row of H (the larger |re| + |im|,
    the working row on ties), the right-hand sides following row by row; the steps' multipliers
    and swaps (lm, sw) are kept for re-solves; then back substitution with the upper factor."""
    n = H.shape[0]
    U = np.zeros_like(H)
    lm = np.zeros(n, complex)
    sw = np.zeros(n, bool)
    cur = H[0].copy()
    cur[0] += delta
    zc = Z[0].copy()
    Y = np.zeros_like(Z)
    for k in range(n - 1):
        nxt = H[k + 1].copy()
        nxt[k + 1] += delta
        ak, bk = cur[k], nxt[k]
        swap = abs(bk.real) + abs(bk.imag) > abs(ak.real) + abs(ak.imag)
        piv, oth = (bk, ak) if swap else (ak, bk)
        l = oth / piv
        p_row, o_row = (nxt, cur) if swap else (cur, nxt)
        U[k, k:] = p_row[k:]
        cur = o_row - l * p_row
        lm[k], sw[k] = l, swap
        zp, zo = (Z[k + 1], zc) if swap else (zc, Z[k + 1])
        Y[k] = zp
        zc = zo - l * zp
    U[n - 1, n - 1] = cur[n - 1]
    Y[n - 1] = zc
    return np.linalg.solve(np.triu(U), Y), (U, lm, sw)


def _hess_resolve(factors, Z):
    """A re-solve with the kept steps: the forward pass over the right-hand sides, then back."""
    U, lm, sw = factors
    n = U.shape[0]
    y = Z.copy()
    zc = y[0].copy()
    for k in range(n - 1):
        zb = y[k + 1].copy()
        zp, zo = (zb, zc) if sw[k] else (zc, zb)
        y[k] = zp
        zc = zo - lm[k] * zp
    y[n - 1] = zc
    return np.linalg.solve(np.triu(U), y)


def _kk(qk):
    """The diagonal energy term of each channel in the assembly: -k^2 open, +k^2 closed."""
    return np.where(qk > 0, -qk * qk, qk * qk)


def test_shifted_form_reproduces_the_oracle():
    w = workloads.production(seed=501, nch=6, nr=NR, rmax=RMAX, energy=1.0, name="shifted-algebra")
    nch, n = w.nch, w.nch * NR
    mesh = orc.rmat_ini(NR, 1, RMAX)
    q2 = mesh.q2[:, 0]
    assert np.allclose(mesh.blo0, np.outer(q2, q2), rtol=1e-13, atol=1e-15)
    Q = np.zeros((n, nch))
    for c in range(nch):
        Q[c * NR:(c + 1) * NR, c] = q2

    kin = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in (2.0, 9.0, 17.5, 28.0)]
    assert any((qk < 0).any() for qk, _ in kin) and any((qk > 0).any() for qk, _ in kin)
    qk_ref = kin[0][0]
    C0 = orc.assemble(mesh, 1, nch, w.lval, qk_ref, np.zeros((nch, 2)), w.cpot)
    H, P = scipy.linalg.hessenberg(C0, calc_q=True)
    assert np.abs(np.tril(H, -2)).max() == 0.0
    W = P.conj().T @ Q

    for qk, eta in kin:
        bnd = orc.boundary_values(nch, w.lval, qk, eta, RMAX)
        C = orc.assemble(mesh, 1, nch, w.lval, qk, bnd.xc, w.cpot)
        shift = _kk(qk) - _kk(qk_ref)
        assert np.allclose(shift, shift[0], rtol=0, atol=1e-12 * max(1.0, np.abs(_kk(qk)).max()))
        delta = shift[0]
        D = np.diag(np.where(qk < 0, -bnd.xc[:, 0] / RMAX, 0.0))
        assert np.allclose(C, C0 + delta * np.eye(n) + Q @ D @ Q.T, rtol=0, atol=1e-12 * np.abs(C).max())

        Y, factors = _hess_solve(H, delta, W)
        Yl = np.linalg.solve(H + delta * np.eye(n), W)
        assert np.linalg.norm(Y - Yl) <= 1e-11 * np.linalg.norm(Yl)
        Z = np.random.default_rng(3).standard_normal((n, 2)) + 0j
        assert np.linalg.norm(_hess_resolve(factors, Z) - np.linalg.solve(H + delta * np.eye(n), Z)) <= \
            1e-11 * np.linalg.norm(np.linalg.solve(H + delta * np.eye(n), Z))
        S = Q.T @ P @ Y
        T = np.eye(nch) - D @ np.linalg.solve(np.eye(nch) + S @ D, S)
        R = S @ T
        R_direct = Q.T @ np.linalg.solve(C, Q)
        assert np.linalg.norm(R - R_direct) <= 1e-10 * np.linalg.norm(R_direct)

        u = orc.collision_matrix(R / RMAX, bnd, qk)
        ref = orc.rmatrix(nch, w.lval, qk, eta, RMAX, mesh, w.cpot)
        no = ref.nopen
        assert np.linalg.norm(u[:no, :no] - ref.cu) <= 1e-10 * np.linalg.norm(ref.cu)
