"""The plain FP64 LU's paired block steps, restated in NumPy (CPU) as the device sequence runs them
(solver.cu: factor_impl's pair_first / pair_second; lu.cuh: panel, trsm modes, gathers).

A block step s factors the panel of columns [k0, k0 + nb) with partial pivoting (the larger
|re| + |im|, the lowest row on ties), interchanging rows only inside the panel and right of it:
L of a step stays in that step's row order, and a solve applies each step's interchanges to the
right-hand side just before that step's block column.  Steps s and s + 1 share one trailing
update of inner dimension 2 nb: step s + 1's interchanges reach step s's multipliers through a
gathered operand, the rows k1 .. k2 get step s's product in step s + 1's order, and the stored
factors are the single-step path's.  Checked: both sequences give the same factors, and the
interleaved solve with them matches numpy's solution.
"""
import numpy as np
import pytest

NB = 8


def _panel(W, k0, ncols):
    """Partial pivoting on columns [k0, k0 + ncols) of W (in place, panel columns only); returns
    the step's row map (new row r <- old row perm[r], rows k0 ..)."""
    n = W.shape[0]
    perm = np.arange(n)
    for j in range(k0, k0 + ncols):
        col = W[j:, j]
        p = j + int(np.argmax(np.abs(col.real) + np.abs(col.imag)))
        if p != j:
            W[[j, p], k0:k0 + ncols] = W[[p, j], k0:k0 + ncols]
            perm[[j, p]] = perm[[p, j]]
        piv = W[j, j]
        if piv != 0:
            W[j + 1:, j] /= piv
        W[j + 1:, j + 1:k0 + ncols] -= np.outer(W[j + 1:, j], W[j, j + 1:k0 + ncols])
    return perm


def _swap_cols(W, perm, k0, c0, c1):
    """The step's interchanges on columns [c0, c1): rows k0 .. take rows perm[k0 ..]."""
    W[k0:, c0:c1] = W[perm[k0:], c0:c1]


def _l11_solve(W, k0, ncols, c0, c1):
    """U12 = L11^-1 W[k0:k0+ncols, c0:c1] with the unit lower triangle of the step."""
    L11 = np.tril(W[k0:k0 + ncols, k0:k0 + ncols], -1) + np.eye(ncols)
    W[k0:k0 + ncols, c0:c1] = np.linalg.solve(L11, W[k0:k0 + ncols, c0:c1])


def _lu_single(A):
    W = A.copy()
    n = W.shape[0]
    perms = []
    for k0 in range(0, n, NB):
        nc = min(NB, n - k0)
        perms.append(_panel(W, k0, nc))
        k1 = k0 + nc
        if k1 >= n:
            break
        _swap_cols(W, perms[-1], k0, k1, n)
        _l11_solve(W, k0, nc, k1, n)
        W[k1:, k1:] -= W[k1:, k0:k1] @ W[k0:k1, k1:]
    return W, perms


def _lu_paired(A):
    W = A.copy()
    n = W.shape[0]
    nsteps = (n + NB - 1) // NB
    perms = []
    s = 0
    while s < nsteps:
        k0 = s * NB
        nc = min(NB, n - k0)
        perms.append(_panel(W, k0, nc))
        k1 = k0 + nc
        if k1 >= n:
            break
        if s + 2 < nsteps:
            # pair_first: only the next panel's columns
            _swap_cols(W, perms[s], k0, k1, k1 + NB)
            _l11_solve(W, k0, NB, k1, k1 + NB)
            W[k1:, k1:k1 + NB] -= W[k1:, k0:k1] @ W[k0:k1, k1:k1 + NB]
            # panel s + 1
            perms.append(_panel(W, k1, NB))
            k2 = k1 + NB
            p1 = perms[s + 1]
            # pair_second: step s's interchanges and U12; step s + 1's interchanges
            _swap_cols(W, perms[s], k0, k2, n)
            _l11_solve(W, k0, NB, k2, n)
            _swap_cols(W, p1, k1, k2, n)
            # rows k1 .. k2 minus L21(s) in step s + 1's order times U12(s)
            F = W[p1[k1:k2], k0:k1]
            W[k1:k2, k2:] -= F @ W[k0:k1, k2:]
            _l11_solve(W, k1, NB, k2, n)
            # A22 -= [P L21(s) | L21(s+1)] [U12(s); U12(s+1)], rows k2 ..
            LL = np.concatenate([W[p1[k2:], k0:k1], W[k2:, k1:k2]], axis=1)
            W[k2:, k2:] -= LL @ W[k0:k2, k2:]
            s += 2
        else:
            _swap_cols(W, perms[s], k0, k1, n)
            _l11_solve(W, k0, nc, k1, n)
            W[k1:, k1:] -= W[k1:, k0:k1] @ W[k0:k1, k1:]
            s += 1
    return W, perms


def _solve(W, perms, b):
    """Forward with each step's interchanges applied just before its block column, then back."""
    n = W.shape[0]
    x = b.astype(np.complex128).copy()
    for s, perm in enumerate(perms):
        k0 = s * NB
        nc = min(NB, n - k0)
        x[k0:] = x[perm[k0:]]
        L11 = np.tril(W[k0:k0 + nc, k0:k0 + nc], -1) + np.eye(nc)
        x[k0:k0 + nc] = np.linalg.solve(L11, x[k0:k0 + nc])
        x[k0 + nc:] -= W[k0 + nc:, k0:k0 + nc] @ x[k0:k0 + nc]
    return np.linalg.solve(np.triu(W), x)


@pytest.mark.parametrize("n", [37, 56, 61, 90])
def test_paired_steps_match_single_steps_and_solve(n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    W1, p1 = _lu_single(A)
    W2, p2 = _lu_paired(A)
    assert len(p1) == len(p2) and all(np.array_equal(x, y) for x, y in zip(p1, p2))
    assert np.linalg.norm(W1 - W2) <= 1e-12 * np.linalg.norm(W1)
    xr = np.linalg.solve(A, b)
    for W, perms in ((W1, p1), (W2, p2)):
        x = _solve(W, perms, b)
        assert np.linalg.norm(x - xr) <= 1e-11 * np.linalg.norm(xr)
