"""The blocked Householder reduction of the shifted scan, restated in NumPy step by step as the
device kernels compute it (hessenberg.cuh: hb_col_cluster_kernel, hb_gemv_kernel,
hb_prep_kernel and the panel GEMMs of hess_reduce_blocked), on the CPU.

Convention: for x with ||x|| > 0, gamma = -e^{i arg x0} ||x||, u = (x - gamma e1) / ||x - gamma e1||,
H = I - 2 u u^H (tau = 2).  Panels of b columns keep the reflectors in V, their product
H_1 .. H_b = I - V T V^H (T upper triangular) and Y = A0 V T for the matrix A0 at the panel's start.
The checks: H upper Hessenberg, P unitary, A = P H P^H.
"""
import numpy as np
import pytest

from hprmat_b200 import workloads
from oracle import rmatrix_oracle as orc

KB = 32  # panel width (kHbB)


def _reduce_blocked(A0):
    A = np.array(A0, dtype=np.complex128)
    n = A.shape[0]
    ncols = n - 2
    V = np.zeros((n, n), complex)           # column c: reflector of column c (rows c+1 ..)
    Ts = []
    for k in range(0, ncols, KB):
        b = min(KB, ncols - k)
        T = np.zeros((KB, KB), complex)
        Y = np.zeros((n, KB), complex)
        for i in range(b):
            c = k + i
            # column c brought up to date: x = A0[:, c] - Y[:, <i] conj(V[c, k + <i])
            x = A[:, c] - Y[:, :i] @ V[c, k:k + i].conj()
            if i > 0:
                # w = V[k+1.., <i]^H x[k+1..];  z = T^H w;  x[k+1..] -= V[k+1.., <i] z
                w = V[k + 1:, k:k + i].conj().T @ x[k + 1:]
                z = T[:i, :i].conj().T @ w
                x[k + 1:] -= V[k + 1:, k:k + i] @ z
            # the reflector of x[c+1 ..]
            ss = float(np.sum(np.abs(x[c + 1:]) ** 2))
            x0 = x[c + 1]
            a0 = abs(x0)
            u = np.zeros(n, complex)
            gamma = x0
            if ss > 0.0:
                nrm = np.sqrt(ss)
                ph = x0 / a0 if a0 > 0 else 1.0
                gamma = -ph * nrm
                winv = 1.0 / np.sqrt(2.0 * ss + 2.0 * nrm * a0)
                u[c + 1:] = x[c + 1:]
                u[c + 1] -= gamma
                u *= winv
            V[:, c] = u
            A[:, c] = np.where(np.arange(n) <= c, x, 0)
            A[c + 1, c] = gamma
            # s = V[:, <i]^H u;  T[<i, i] = -2 T[<i, <i] s, T[i, i] = 2 (0 for an identity reflector)
            s = V[:, k:k + i].conj().T @ u
            T[:i, i] = -2.0 * (T[:i, :i] @ s)
            T[i, i] = 2.0 if ss > 0.0 else 0.0
            # y_i = 2 (A0[:, c+1 ..] u - Y[:, <i] s): the GEMV over the trailing columns (of A0)
            Y[:, i] = 2.0 * (A[:, c + 1:] @ u[c + 1:] - Y[:, :i] @ s)
        Ts.append(T)
        if k + b < n:
            # A[:, k+b ..] -= Y V[k+b .., ]^H;  W = -V[k+1 .., ]^H A[k+1 .., k+b ..];  A[k+1 .., k+b ..] -= (-V T^H) W
            Vp = V[:, k:k + b]
            A[:, k + b:] -= Y[:, :b] @ Vp[k + b:, :].conj().T
            W = -(Vp[k + 1:, :].conj().T @ A[k + 1:, k + b:])
            VT = -(Vp @ T[:b, :b].conj().T)
            A[k + 1:, k + b:] -= VT[k + 1:, :] @ W
    # P = Q_0 Q_1 ..., Q_p = I - V_p T_p V_p^H, backwards from the identity
    P = np.eye(n, dtype=complex)
    for p in range(len(Ts) - 1, -1, -1):
        k = p * KB
        b = min(KB, ncols - k)
        Vp = V[:, k:k + b]
        W = -(Vp[k + 1:, :].conj().T @ P[k + 1:, k + 1:])
        VTn = -(Vp @ Ts[p][:b, :b])
        P[k + 1:, k + 1:] -= VTn[k + 1:, :] @ W
    return A, P


def _cases():
    rng = np.random.default_rng(7)
    out = [rng.standard_normal((100, 100)) + 1j * rng.standard_normal((100, 100)),
           rng.standard_normal((66, 66)) + 1j * rng.standard_normal((66, 66))]
    w = workloads.production(seed=41, nch=4, nr=30, rmax=20.0)
    mesh = orc.rmat_ini(30, 1, 20.0)
    bnd = orc.boundary_values(w.nch, w.lval, w.qk, w.eta, 20.0)
    out.append(orc.assemble(mesh, 1, w.nch, w.lval, w.qk, bnd.xc, w.cpot))
    return out


@pytest.mark.parametrize("case", range(3))
def test_blocked_reduction_formulas(case):
    A0 = _cases()[case]
    n = A0.shape[0]
    H, P = _reduce_blocked(A0)
    assert np.abs(np.tril(H, -2)).max() == 0.0
    assert np.abs(P.conj().T @ P - np.eye(n)).max() <= 1e-13
    assert np.linalg.norm(P @ H @ P.conj().T - A0) <= 1e-14 * np.linalg.norm(A0) * n ** 0.5
