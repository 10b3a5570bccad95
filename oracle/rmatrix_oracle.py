"""Oracle (test infrastructure only): FP64 CPU restatement of HPRMAT's R-matrix path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may use
this module, and only as the checker or as the timed CPU baseline -- never as the product.

This is the reference's "Type 1" path (dense LAPACK ZGESV), restated in NumPy with the
same LAPACK routine (``scipy.linalg.lapack.zgesv``, OpenBLAS) and the same argument
pattern.  Reference paths are relative to the HPRMAT project root:

* ``legzo``                  -- ``src/rmatrix_hp.F90:741-783``
* ``rmat_ini``               -- ``src/rmatrix_hp.F90:61-159``
* ``boundary_values``        -- ``src/rmatrix_hp.F90:224-244``
* ``assemble``               -- ``src/rmatrix_hp.F90:246-293``
* ``solve_rmatrix_dense``    -- ``src/rmatrix_hp.F90:441-477`` (= ``src/rmat_solvers.F90:98-148``)
* ``solve_rmatrix_4``        -- ``src/rmatrix_hp.F90:590-632``
* ``rmatrix``                -- ``src/rmatrix_hp.F90:175-368`` (propagation for ns > 1 at
  ``:326-345``, collision matrix at ``:348-368``)
* ``solve_rmatrix_mixed``    -- ``src/rmat_solvers.F90:157-296`` (CGETRF + FP64 refinement)
* ``rmatrix_wf``             -- ``src/rmatrix_hp.F90:378-431`` with C^-1 as
  ``rmat_pierre/rmatrix.f:270-318`` (wave functions at the mesh points)
* ``spline``/``splint``/``wf_print`` -- ``src/rmatrix_hp.F90:678-734, 786-841``

Arrays follow the Fortran layout: C(E) is column-major with row index
``(channel-1)*nr + i``; ``cpot`` has shape ``(ncp1, ndim, ndim)`` (Fortran order,
``cpot[ir, c, c']``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.linalg.lapack as lapack

from .special_functions import coulfg, whit


def legzo(n: int):
    """Gauss-Legendre nodes/weights on (0, 1) (src/rmatrix_hp.F90:741-783)."""
    pi = 3.1415926535898
    one = 1.0
    x = np.zeros(n + 1)  # 1-based
    w = np.zeros(n + 1)
    n0 = (n + 1) // 2
    for nr in range(1, n0 + 1):
        z = math.cos(pi * (nr - 0.25) / (n + 0.5))
        while True:
            z0 = z
            p = 1.0
            for i in range(1, nr):
                p = p * (z - x[i])
            f0 = 1.0
            if nr == n0 and n != 2 * (n // 2):
                z = 0.0
            f1 = z
            pf = pd = 0.0
            for k in range(2, n + 1):
                pf = (2 - one / k) * z * f1 - (1 - one / k) * f0
                pd = k * (f1 - z * pf) / (1 - z * z)
                f0 = f1
                f1 = pf
            if z == 0:
                break
            fd = pf / p
            q = 0.0
            for i in range(1, nr):
                wp = 1.0
                for j in range(1, nr):
                    if j != i:
                        wp = wp * (z - x[j])
                q = q + wp
            gd = (pd - q * fd) / p
            z = z - fd / gd
            if not (abs(z - z0) > abs(z) * 1.0e-15):
                break
        x[nr] = z
        x[n + 1 - nr] = -z
        w[nr] = 2 / ((1 - z * z) * pd * pd)
        w[n + 1 - nr] = w[nr]
    xs = (1 + x[n:0:-1]) / 2
    ws = w[n:0:-1] / 2
    return xs.copy(), ws.copy()


@dataclass
class Mesh:
    nr: int
    ns: int
    rmax: float
    rmax0: float
    xle: np.ndarray
    wle: np.ndarray
    tc: np.ndarray     # (nr, nr, ns)
    blo0: np.ndarray   # (nr, nr)
    blo1: np.ndarray
    blo2: np.ndarray
    q1: np.ndarray     # (nr, ns)
    q2: np.ndarray     # (nr, ns)
    zrma: np.ndarray   # (nr*ns,)


def rmat_ini(nr: int, ns: int, rmax: float) -> Mesh:
    """Lagrange-Legendre mesh, kinetic + Bloch matrices (src/rmatrix_hp.F90:61-159)."""
    tc = np.zeros((nr, nr, ns))
    blo0 = np.zeros((nr, nr))
    blo1 = np.zeros((nr, nr))
    blo2 = np.zeros((nr, nr))
    q1 = np.zeros((nr, ns))
    q2 = np.zeros((nr, ns))
    rmax0 = rmax / ns
    xle, wle = legzo(nr)
    for is_ in range(1, ns + 1):
        s = is_ - 1
        for i1 in range(1, nr + 1):
            xi = xle[i1 - 1]
            xi2 = xi * (1 - xi)
            if is_ == 1:
                xx = 4 * nr * (nr + 1) + 3 + (1 - 6 * xi) / xi2
                tc[i1 - 1, i1 - 1, 0] = xx / (3 * xi2)
                blo0[i1 - 1, i1 - 1] = 1 / xi2
            else:
                xlb = xi / (1 - xi) * (nr * (nr + 1) - 1 / (1 - xi))
                xla = (1 - xi) / xi * (-nr * (nr + 1) + 1 / xi)
                tc[i1 - 1, i1 - 1, s] = (nr * nr + nr + 6 - 2 / xi2) / (3 * xi2) + xlb - xla
                blo1[i1 - 1, i1 - 1] = (1 - xi) / xi
                blo2[i1 - 1, i1 - 1] = xi / (1 - xi)
            for i2 in range(1, i1):
                xj = xle[i2 - 1]
                xj2 = xj * (1 - xj)
                if is_ == 1:
                    xx = (nr * (nr + 1) + 1 + (xi + xj - 2 * xi * xj) / ((xi - xj) * (xi - xj))
                          - 1 / (1 - xi) - 1 / (1 - xj))
                    tc[i1 - 1, i2 - 1, 0] = xx / math.sqrt(xi2 * xj2)
                    blo0[i1 - 1, i2 - 1] = 1 / math.sqrt(xi2 * xj2)
                else:
                    yy = (math.sqrt(xj2 / (xi2 * xi2 * xi2)) * (2 * xi * xj + 3 * xi - xj - 4 * xi * xi)
                          / ((xj - xi) * (xj - xi)))
                    xlb = math.sqrt(xi * xj / (1 - xi) / (1 - xj)) * (nr * (nr + 1) - 1 / (1 - xj))
                    xla = math.sqrt((1 - xi) * (1 - xj) / xi / xj) * (-nr * (nr + 1) + 1 / xj)
                    tc[i1 - 1, i2 - 1, s] = yy + xlb - xla
                    blo1[i1 - 1, i2 - 1] = math.sqrt((1 - xi) * (1 - xj) / xi / xj)
                    blo2[i1 - 1, i2 - 1] = math.sqrt(xi * xj / (1 - xi) / (1 - xj))
                if (i1 + i2) % 2 == 1:
                    tc[i1 - 1, i2 - 1, s] = -tc[i1 - 1, i2 - 1, s]
                    blo0[i1 - 1, i2 - 1] = -blo0[i1 - 1, i2 - 1]
                    blo1[i1 - 1, i2 - 1] = -blo1[i1 - 1, i2 - 1]
                    blo2[i1 - 1, i2 - 1] = -blo2[i1 - 1, i2 - 1]
                tc[i2 - 1, i1 - 1, s] = tc[i1 - 1, i2 - 1, s]
                blo0[i2 - 1, i1 - 1] = blo0[i1 - 1, i2 - 1]
                blo1[i2 - 1, i1 - 1] = blo1[i1 - 1, i2 - 1]
                blo2[i2 - 1, i1 - 1] = blo2[i1 - 1, i2 - 1]
            if is_ == 1:
                q2[:, 0] = 1 / np.sqrt(xle * (1 - xle))
                q1[:, 0] = 0
            else:
                q2[:, s] = np.sqrt(xle / (1 - xle))
                q1[:, s] = -1 / q2[:, s]
            if nr % 2 == 1:
                q2[:, s] = -q2[:, s]
            q1[0::2, s] = -q1[0::2, s]
            q2[0::2, s] = -q2[0::2, s]
    tc = tc / (rmax0 * rmax0)
    blo0 = blo0 / rmax0
    blo1 = blo1 / rmax0
    blo2 = blo2 / rmax0
    q1 = q1 / math.sqrt(rmax0)
    q2 = q2 / math.sqrt(rmax0)
    zrma = np.concatenate([((is_ - 1) + xle) * rmax0 for is_ in range(1, ns + 1)])
    return Mesh(nr, ns, rmax, rmax0, xle, wle, tc, blo0, blo1, blo2, q1, q2, zrma)


@dataclass
class Boundary:
    """Open-channel Coulomb values and closed-channel Whittaker values (rmatrix_hp.F90:224-244)."""
    nopen: int
    npo_open: list      # 0-based channel indices of open channels, in order
    npo_closed: list
    co: np.ndarray      # (nopen,) G + iF
    cop: np.ndarray     # (nopen,) (G' + iF') * k * a
    xc: np.ndarray      # (nch, 2): a*W'/W and W for closed channels


def boundary_values(nch, lval, qk, eta, rmax) -> Boundary:
    co, cop = [], []
    xc = np.zeros((nch, 2))
    npo_open, npo_closed = [], []
    for i1 in range(nch):
        l = int(lval[i1])
        if qk[i1] > 0:
            npo_open.append(i1)
            fc, gc, dfc, dgc, ifail = coulfg(qk[i1] * rmax, eta[i1], float(l))
            co.append(complex(gc, fc))
            cop.append(complex(dgc, dfc) * qk[i1] * rmax)
        else:
            npo_closed.append(i1)
            qk2 = -qk[i1]
            f, fd, _ = whit(eta[i1], rmax, qk2, -qk2 * qk2, l, 0)
            xc[i1, 0] = rmax * fd[l] / f[l]
            xc[i1, 1] = f[l]
    return Boundary(len(npo_open), npo_open, npo_closed, np.array(co, dtype=np.complex128),
                    np.array(cop, dtype=np.complex128), xc)


def assemble(mesh: Mesh, is_: int, nch, lval, qk, xc, cpot, cpnl=None) -> np.ndarray:
    """C(E) of interval ``is_`` (1-based), src/rmatrix_hp.F90:246-293.  ``cpnl`` (ncp2 >= nr^2,
    ndim, ndim): non-local potential, block (c, c') gains sqrt(w_i w_j) rmax0 cpnl(i nr + j, c, c')
    (0-based i, j; :283-288, one interval)."""
    nr = mesh.nr
    rmax0 = mesh.rmax0
    rmax1 = (is_ - 1) * rmax0
    rmax2 = is_ * rmax0
    ms = (is_ - 1) * nr
    ntot = nch * nr
    ch = np.zeros((ntot, ntot), dtype=np.complex128, order="F")
    s = is_ - 1
    rr = rmax1 + mesh.xle * rmax0
    for i1 in range(nch):
        m1 = i1 * nr
        blk = mesh.tc[:, :, s].astype(np.complex128)
        fac = float(lval[i1] * (lval[i1] + 1))
        d = fac / (rr * rr)
        if qk[i1] > 0:
            d = d - qk[i1] * qk[i1]
        if qk[i1] < 0:
            d = d + qk[i1] * qk[i1]
        blk[np.arange(nr), np.arange(nr)] += d
        if qk[i1] < 0:
            if is_ == 1:
                blk = blk - xc[i1, 0] * mesh.blo0 / rmax2
            else:
                blk = blk - xc[i1, 0] * (mesh.blo2 / rmax2 - mesh.blo1 / rmax1)
        ch[m1:m1 + nr, m1:m1 + nr] = blk
        for i2 in range(nch):
            m2 = i2 * nr
            idx = np.arange(nr)
            ch[m1 + idx, m2 + idx] += cpot[ms + idx, i1, i2]
            if cpnl is not None:
                ii0 = (is_ - 1) * nr * nr
                nl = cpnl[ii0:ii0 + nr * nr, i1, i2].reshape(nr, nr)  # row i, column j
                ch[m1:m1 + nr, m2:m2 + nr] += np.sqrt(np.outer(mesh.wle, mesh.wle)) * rmax0 * nl
    return ch


def _zgesv(a, b):
    lu, piv, x, info = lapack.zgesv(np.asfortranarray(a), np.asfortranarray(b),
                                    overwrite_a=True, overwrite_b=True)
    return x, info


def cond1_estimate(a: np.ndarray) -> float:
    """||A||_1 ||A^-1||_1 by the Hager-Higham 1-norm estimator (N. J. Higham, ACM TOMS 14
    (1988) 381-396; the method of LAPACK's ZLACN2 behind ZGECON) on the zgetrf factors of A:
    x = 1/n; repeat y = A^-1 x, stop when ||y||_1 no longer grows, x = e_j with
    j = argmax |(A^-H sign(y))_j|, stop when j repeats (at most 5 passes); then the extra vector
    x_i = (-1)^i (1 + i/(n-1)), estimate 2 ||A^-1 x||_1 / (3n).  A lower bound of the exact
    value.  Checker for the library's opts.estimate_condition."""
    a = np.asfortranarray(a, dtype=np.complex128)
    n = a.shape[0]
    lu, piv, info = lapack.zgetrf(a)
    if info != 0:
        return math.inf
    anorm = float(np.abs(a).sum(axis=0).max())

    def solve(v, herm):
        x, _ = lapack.zgetrs(lu, piv, v.reshape(-1, 1), trans=2 if herm else 0)
        return x[:, 0]

    x = np.full(n, 1.0 / n, dtype=np.complex128)
    est, jlast = 0.0, -1
    for p in range(5):
        y = solve(x, False)
        e = float(np.abs(y).sum())
        if not np.isfinite(e) or (p > 0 and e <= est):
            break
        est = e
        m = np.abs(y)
        xi = np.where(m > 0, y / np.where(m > 0, m, 1.0), 1.0)
        z = solve(xi, True)
        j = int(np.argmax(np.abs(z)))
        if j == jlast:
            break
        jlast = j
        x = np.zeros(n, dtype=np.complex128)
        x[j] = 1.0
    alt = np.array([(-1.0) ** i * (1.0 + (i / (n - 1) if n > 1 else 0.0)) for i in range(n)], dtype=np.complex128)
    est = max(est, 2.0 * float(np.abs(solve(alt, False)).sum()) / (3.0 * n))
    return anorm * est


def surface_rhs(q2col: np.ndarray, nch: int) -> np.ndarray:
    """X = blockdiag(q2) RHS, one column per channel (src/rmatrix_hp.F90:456-461)."""
    nr = q2col.shape[0]
    x = np.zeros((nch * nr, nch), dtype=np.complex128, order="F")
    for ich in range(nch):
        x[ich * nr:(ich + 1) * nr, ich] = q2col
    return x


def extract_r(x: np.ndarray, bvec: np.ndarray, nch: int, normfac: float = 1.0) -> np.ndarray:
    """R(i, j) = sum_r B(r) X((i-1)*nr + r, j) -- bilinear, no conjugate (rmatrix_hp.F90:466-474)."""
    nr = bvec.shape[0]
    rm = np.zeros((nch, nch), dtype=np.complex128)
    for ich in range(nch):
        rm[ich, :] = bvec @ x[ich * nr:(ich + 1) * nr, :]
    return rm * normfac


def solve_rmatrix_dense(cmat, bvec, nch, nlag, normfac=1.0):
    """Type 1 solver (src/rmatrix_hp.F90:441-477): copy, ZGESV(N, nch), R extraction."""
    a_work = np.array(cmat, dtype=np.complex128, order="F", copy=True)
    xv = surface_rhs(np.asarray(bvec, dtype=np.complex128), nch)
    x, info = _zgesv(a_work, xv)
    if info != 0:
        raise RuntimeError(f"Error in solve_rmatrix_hp ZGESV (info={info})")
    return extract_r(x, np.asarray(bvec, dtype=np.complex128), nch, normfac), x


def solve_rmatrix_mixed(cmat, bvec, nch, nlag, normfac=1.0, max_iter=2, tol=1.0e-10):
    """Type 2 solver (src/rmat_solvers.F90:157-296): CGETRF + FP64 residual refinement."""
    n = nch * nlag
    a_sp = np.asfortranarray(cmat.astype(np.complex64))
    b_dp = surface_rhs(np.asarray(bvec, dtype=np.complex128), nch)
    b_norm = np.linalg.norm(b_dp)
    if b_norm == 0.0:
        b_norm = 1.0
    lu, piv, info = lapack.cgetrf(a_sp)
    if info != 0:
        return solve_rmatrix_dense(cmat, bvec, nch, nlag, normfac)
    w, info = lapack.cgetrs(lu, piv, b_dp.astype(np.complex64))
    x = w.astype(np.complex128)
    steps = 0
    for _ in range(max_iter):
        r = b_dp - cmat @ x
        rel = np.linalg.norm(r) / b_norm
        if rel < tol:
            break
        w, info = lapack.cgetrs(lu, piv, r.astype(np.complex64))
        x = x + w.astype(np.complex128)
        steps += 1
    return extract_r(x, np.asarray(bvec, dtype=np.complex128), nch, normfac), x


def solve_rmatrix_4(cmat, b0, b1, nch, nlag, normfac=1.0):
    """R00, R01, R11 from one ZGESV with 2*nch RHS (src/rmatrix_hp.F90:590-632)."""
    n = nch * nlag
    xv = np.zeros((n, 2 * nch), dtype=np.complex128, order="F")
    for ich in range(nch):
        xv[ich * nlag:(ich + 1) * nlag, ich] = b0
        xv[ich * nlag:(ich + 1) * nlag, ich + nch] = b1
    x, info = _zgesv(np.array(cmat, order="F", copy=True), xv)
    if info != 0:
        raise RuntimeError("Error in solve_rmatrix_hp_4")
    r00 = np.zeros((nch, nch), dtype=np.complex128)
    r01 = np.zeros((nch, nch), dtype=np.complex128)
    r11 = np.zeros((nch, nch), dtype=np.complex128)
    for ich in range(nch):
        blk = x[ich * nlag:(ich + 1) * nlag, :]
        r00[ich, :] = (b0 @ blk[:, :nch]) * normfac
        r01[ich, :] = (b0 @ blk[:, nch:]) * normfac
        r11[ich, :] = (b1 @ blk[:, nch:]) * normfac
    return r00, r01, r11


def collision_matrix(rma: np.ndarray, bnd: Boundary, qk) -> np.ndarray:
    """U from the R-matrix at the channel radius (src/rmatrix_hp.F90:348-368).

    ``rma`` is R/a (crma0 at the last interval), shape (nch, nch).
    """
    no = bnd.nopen
    idx = bnd.npo_open
    crma2 = np.zeros((no, no), dtype=np.complex128)
    for m1, i1 in enumerate(idx):
        for m2, i2 in enumerate(idx):
            crma2[m1, m2] = rma[i1, i2] * math.sqrt(qk[i1] / qk[i2])
    cz = np.zeros((no, no), dtype=np.complex128)
    cu = np.zeros((no, no), dtype=np.complex128)
    for m1 in range(no):
        cz[:, m1] = -crma2[:, m1] * bnd.cop[m1]
        cu[:, m1] = -crma2[:, m1] * np.conj(bnd.cop[m1])
        cz[m1, m1] += bnd.co[m1]
        cu[m1, m1] += np.conj(bnd.co[m1])
    if no == 0:
        return cu
    u, info = _zgesv(cz, cu)
    if info != 0:
        raise RuntimeError("Error in ZGESV for collision matrix")
    return u


@dataclass
class RMatrixResult:
    cu: np.ndarray        # (nopen, nopen) collision matrix
    nopen: int
    rma: np.ndarray       # R/a at the channel radius, (nch, nch)
    boundary: Boundary
    x: np.ndarray | None  # solution of the ns = 1 solve, (N, nch)


def rmatrix(nch, lval, qk, eta, rmax, mesh: Mesh, cpot, solver: str = "dense", cpnl=None) -> RMatrixResult:
    """Collision matrix for one (J, pi, E), src/rmatrix_hp.F90:175-368; ``cpnl``: non-local
    potential (ns = 1 only, :205-209)."""
    if cpnl is not None and mesh.ns != 1:
        raise ValueError("ns must be ns=1 for non-local potentials")
    lval = np.asarray(lval)
    qk = np.asarray(qk, dtype=np.float64)
    eta = np.asarray(eta, dtype=np.float64)
    nr, ns = mesh.nr, mesh.ns
    bnd = boundary_values(nch, lval, qk, eta, rmax)
    crma0_prev = None
    x_last = None
    for is_ in range(1, ns + 1):
        rmax1 = (is_ - 1) * mesh.rmax0
        rmax2 = is_ * mesh.rmax0
        ch = assemble(mesh, is_, nch, lval, qk, bnd.xc, cpot, cpnl)
        bvec = mesh.q2[:, is_ - 1].astype(np.complex128)
        if solver == "dense":
            r11, x_last = solve_rmatrix_dense(ch, bvec, nch, nr)
        elif solver == "mixed":
            r11, x_last = solve_rmatrix_mixed(ch, bvec, nch, nr)
        else:
            raise ValueError(solver)
        if ns > 1:
            r00, r01, r11 = solve_rmatrix_4(ch, mesh.q1[:, is_ - 1], mesh.q2[:, is_ - 1], nch, nr)
        if is_ == 1:
            crma0 = r11 / rmax2
        else:
            cz = r00 + crma0_prev * rmax1
            czi = np.linalg.solve(cz, np.eye(nch, dtype=np.complex128))
            crma0 = (r11 - r01.T @ czi @ r01) / rmax2
        crma0_prev = crma0
    cu = collision_matrix(crma0_prev, bnd, qk)
    return RMatrixResult(cu, bnd.nopen, crma0_prev, bnd, x_last if ns == 1 else None)


def rmatrix_wf(nch, lval, qk, eta, rmax, mesh: Mesh, cpot, nvc, u=None, cpnl=None):
    """U and the internal wave functions (rmatrix with twf = .true., src/rmatrix_hp.F90:378-431).

    ``nvc``: entrance channels, 1-based indices among the open channels.  Per interval the
    dense solve is X = C^-1 [blockdiag(q1) | blockdiag(q2)] (ZGESV, 2 nch right-hand sides),
    giving R00, R01, R11 and the propagated R as ``rmatrix``.  The surface amplitudes cfp of
    the last interval follow from U (:380-386), are carried inwards with
    (R00 + rin R)^-1 R01 (:388-394), and the wave function of interval is is
    C_is^-1 (blockdiag(q2) cfp_is - blockdiag(q1) cfp_is-1) -- C^-1 as in Descouvemont's
    original (rmat_pierre/rmatrix.f:286-301), where ``ch`` holds the inverse; the HPRMAT
    version multiplies by C itself at :407.  Closed-channel amplitudes go to
    cu[nopen + m, ic] (:414-419), and cf is divided by sqrt(rmax0 w_i) (:421-428).

    ``u``: use this collision matrix (nopen x nopen or larger) for the surface amplitudes
    instead of the oracle's own.  Where |U| ~ 1 deep under a barrier (e.g. Ex1, |cop| ~ 1e7)
    the wave function's small components are set by the last bits of U, so a reconstruction
    is compared with the oracle's from the same U.

    Returns (cu (nch, nch) with U in [:nopen, :nopen], nopen, cf (nr ns, nch, len(nvc))).
    """
    lval = np.asarray(lval)
    qk = np.asarray(qk, dtype=np.float64)
    eta = np.asarray(eta, dtype=np.float64)
    nr, ns, rmax0 = mesh.nr, mesh.ns, mesh.rmax0
    n = nch * nr
    bnd = boundary_values(nch, lval, qk, eta, rmax)
    xs, crma, crma0 = [], [], []
    for is_ in range(1, ns + 1):
        s = is_ - 1
        rmax1, rmax2 = (is_ - 1) * rmax0, is_ * rmax0
        ch = assemble(mesh, is_, nch, lval, qk, bnd.xc, cpot, cpnl)
        q1, q2 = mesh.q1[:, s], mesh.q2[:, s]
        rhs = np.zeros((n, 2 * nch), dtype=np.complex128, order="F")
        for c in range(nch):
            rhs[c * nr:(c + 1) * nr, c] = q1
            rhs[c * nr:(c + 1) * nr, nch + c] = q2
        x, info = _zgesv(ch, rhs)
        if info != 0:
            raise RuntimeError(f"singular C(E) in interval {is_}")
        x1, x2 = x[:, :nch], x[:, nch:]
        r00, r01, r11 = extract_r(x1, q1, nch), extract_r(x2, q1, nch), extract_r(x2, q2, nch)
        if is_ == 1:
            c0 = r11 / rmax2
        else:
            cz = r00 + crma0[-1] * rmax1
            c0 = (r11 - r01.T @ np.linalg.solve(cz, r01)) / rmax2
        xs.append((x1, x2))
        crma.append((r00, r01, r11))
        crma0.append(c0)
    no = bnd.nopen
    if u is None:
        u = collision_matrix(crma0[-1], bnd, qk)
    else:
        u = np.asarray(u, dtype=np.complex128)[:no, :no]
    cu = np.zeros((nch, nch), dtype=np.complex128)
    cu[:no, :no] = u
    cf = np.zeros((nr * ns, nch, len(nvc)), dtype=np.complex128)
    for ic, nvex in enumerate(nvc):
        i2 = bnd.npo_open[nvex - 1]
        cfp = np.zeros((nch, ns + 1), dtype=np.complex128)  # column is = 0..ns
        for m1, i1 in enumerate(bnd.npo_open):
            v = -u[m1, nvex - 1] * bnd.cop[m1] * math.sqrt(qk[i2] / qk[i1])
            if i1 == i2:
                v += np.conj(bnd.cop[m1])
            cfp[i1, ns] = v
        cfp[:, ns] /= rmax
        for is_ in range(ns - 1, 0, -1):
            cz = crma[is_][0] + is_ * rmax0 * crma0[is_ - 1]
            cfp[:, is_] = np.linalg.solve(cz, crma[is_][1]) @ cfp[:, is_ + 1]
        for is_ in range(1, ns + 1):
            x1, x2 = xs[is_ - 1]
            v = x2 @ cfp[:, is_] - x1 @ cfp[:, is_ - 1]
            cf[(is_ - 1) * nr:is_ * nr, :, ic] = v.reshape(nch, nr).T
        for m1, i1 in enumerate(bnd.npo_closed):
            cy = np.sum(cf[(ns - 1) * nr:ns * nr, i1, ic] * mesh.q2[:, ns - 1])
            cu[m1 + no, ic] = cy / bnd.xc[i1, 1]
        for is_ in range(ns):
            cf[is_ * nr:(is_ + 1) * nr, :, ic] /= np.sqrt(rmax0 * mesh.wle)[:, None]
    return cu, no, cf


def spline(x, y, ypn=None):
    """Second derivatives of the cubic spline through (x, y) (src/rmatrix_hp.F90:787-816):
    tridiagonal elimination.  Natural at the first point (wf_print's yp1 = 1e30); at the last
    point natural (ypn None: wf_print's yp2 = 1e30) or with first derivative ypn."""
    n = len(x)
    y2 = np.zeros(n)
    u = np.zeros(n)
    for i in range(1, n - 1):
        sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1])
        p = sig * y2[i - 1] + 2.0
        y2[i] = (sig - 1.0) / p
        d = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])
        u[i] = (6.0 * d / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p
    if ypn is None:
        y2[n - 1] = 0.0
    else:
        un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]))
        y2[n - 1] = (un - 0.5 * u[n - 2]) / (0.5 * y2[n - 2] + 1.0)
    for k in range(n - 2, -1, -1):
        y2[k] = y2[k] * y2[k + 1] + u[k]
    return y2


def splint(xa, ya, y2a, x):
    """Cubic-spline value at x (src/rmatrix_hp.F90:818-841): bisection for the bracketing
    interval, then the cubic in the local coordinates."""
    klo, khi = 0, len(xa) - 1
    while khi - klo > 1:
        k = (khi + klo) // 2
        if xa[k] > x:
            khi = k
        else:
            klo = k
    h = xa[khi] - xa[klo]
    a = (xa[khi] - x) / h
    b = (x - xa[klo]) / h
    return a * ya[klo] + b * ya[khi] + ((a ** 3 - a) * y2a[klo] + (b ** 3 - b) * y2a[khi]) * h * h / 6.0


def wf_print(nch, lval, qk, eta, rmax, mesh: Mesh, cu, nopen, cf, iv, nom, npoin, h, ypn=None):
    """Wave function of channel iv (1-based) for entrance nom on r = h, 2h, ..., npoin h
    (src/rmatrix_hp.F90:678-734): the spline of the mesh values inside rmax, the Coulomb
    (open) or Whittaker (closed) form outside.  ypn: the spline's end condition (None:
    natural, as HPRMAT; Descouvemont's original passes an unset yp2, rmat_pierre/rmatrix.f:339,350)."""
    qk = np.asarray(qk, dtype=np.float64)
    zr = mesh.zrma
    nop = sum(1 for w in range(iv) if qk[w] > 0)
    nclo = nopen + sum(1 for w in range(iv) if qk[w] < 0)
    xr, xi = cf[:, iv - 1, nom - 1].real.copy(), cf[:, iv - 1, nom - 1].imag.copy()
    y2r, y2i = spline(zr, xr, ypn), spline(zr, xi, ypn)
    out = np.zeros(npoin, dtype=np.complex128)
    l = int(lval[iv - 1])
    for i in range(1, npoin + 1):
        r = i * h
        if r <= rmax:
            out[i - 1] = complex(splint(zr, xr, y2r, r), splint(zr, xi, y2i, r))
        elif qk[iv - 1] > 0:
            fc, gc, _, _, _ = coulfg(qk[iv - 1] * r, eta[iv - 1], float(l))
            co = complex(gc, fc) * math.sqrt(qk[nom - 1] / qk[iv - 1])
            v = -cu[nop - 1, nom - 1] * co
            if iv == nom:
                v += np.conj(co)
            out[i - 1] = v
        else:
            f, _, _ = whit(eta[iv - 1], r, -qk[iv - 1], -qk[iv - 1] ** 2, l, 0)
            out[i - 1] = cu[nclo - 1, nom - 1] * f[l]
    return out


def rmatrix_adjoint(nch, lval, qk, eta, rmax, mesh: Mesh, cpot, gu):
    """FP64 reference gradient of a real loss L through U (ns = 1, dense NumPy/LAPACK).

    The reference has no derivatives; this is the checker of the device adjoint.  ``gu`` is
    dL/dU in the convention dL = Re sum conj(gu) dU; returns (U, grad) with grad shaped like
    cpot (nr rows used) in the same convention, from
      dU = Z_O^-1 dRt W,  W = diag(cop) U - diag(conj cop),  Rt = R sqrt(k_i/k_j),  R = Q^T X / a,
      dX = -C^-1 dC X,    C^T Y = Q M2^T,  grad(r_i, c, c') = -conj(sum Y[(c,i), :] X[(c',i), :]) / a.
    """
    qk = np.asarray(qk, dtype=np.float64)
    res = rmatrix(nch, lval, qk, eta, rmax, mesh, cpot)
    bnd, no = res.boundary, res.nopen
    nr = mesh.nr
    a = mesh.rmax0
    grad = np.zeros_like(np.asarray(cpot, dtype=np.complex128))
    if no == 0:
        return res.cu, grad
    idx = bnd.npo_open
    s = np.array([[math.sqrt(qk[i1] / qk[i2]) for i2 in idx] for i1 in idx])
    rt = res.rma[np.ix_(idx, idx)] * s
    zo = np.diag(bnd.co) - rt * bnd.cop[None, :]
    u = res.cu
    w = bnd.cop[:, None] * u - np.diag(np.conj(bnd.cop))
    g = np.asarray(gu, dtype=np.complex128)[:no, :no]
    m = (w @ g.conj().T) @ np.linalg.inv(zo)
    m2 = np.zeros((nch, nch), dtype=np.complex128)
    for a1, i1 in enumerate(idx):
        for a2, i2 in enumerate(idx):
            m2[i2, i1] = m[a2, a1] * s[a1, a2]
    q = surface_rhs(mesh.q2[:, 0].astype(np.complex128), nch)   # (N, nch)
    C = assemble(mesh, 1, nch, lval, qk, bnd.xc, cpot)
    y = np.linalg.solve(C.T, q @ m2.T)
    x = res.x
    for c in range(nch):
        for cp in range(nch):
            h = np.sum(y[c * nr:(c + 1) * nr, :] * x[cp * nr:(cp + 1) * nr, :], axis=1)
            grad[:nr, c, cp] = -np.conj(h) / a
    return u, grad
