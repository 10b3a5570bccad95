"""GPU parity of the CUDA path (through the C ABI) against the oracle.

Tolerances: collision matrices agree with the FP64 LAPACK oracle to a relative Frobenius
error of 1e-10 (the target of the solver), for both the plain FP64 LU and the mixed
(3xTF32 tensor-core LU + FP64 refinement) path.  The tensor-core trailing-update kernel is
checked on its own against an FP64 torch product to 3xTF32 accuracy (2e-6 relative).
"""
import math
import os

import numpy as np
import pytest
import torch

from hprmat_b200 import _native as nat
from hprmat_b200 import api, workloads
from oracle import rmatrix_oracle as orc
from tests.example_inputs import ex1_setup, ex2_setup, ex4_setup

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

pytestmark = pytest.mark.gpu

U_TOL = 1e-10


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _oracle_u(w):
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    return orc.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot)


def _refined_u(w):
    """The oracle's U with its zgesv solution refined by residuals in extended precision (three
    steps, after which it no longer changes): the reference for results of a plain FP64 LU,
    which, like the oracle's own, stop at the LU's rounding level."""
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    bnd = orc.boundary_values(w.nch, w.lval, w.qk, w.eta, w.rmax)
    C = orc.assemble(mesh, 1, w.nch, w.lval, w.qk, bnd.xc, w.cpot)
    bvec = mesh.q2[:, 0].astype(np.complex128)
    B = orc.surface_rhs(bvec, w.nch)
    X = np.linalg.solve(C, B)
    for _ in range(3):
        r = (B.astype(np.clongdouble) - C.astype(np.clongdouble) @ X.astype(np.clongdouble)).astype(np.complex128)
        X = X + np.linalg.solve(C, r)
    return orc.collision_matrix(orc.extract_r(X, bvec, w.nch) / w.rmax, bnd, w.qk)


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(precision="mixed")
    yield c
    c.close()


def test_kernels_report_sm100_binary():
    """The CUDA runtime reports the loaded kernels as sm_100 binaries (binaryVersion 100)."""
    assert nat.load().hprmat_b200_dev_binary_version() == 100


@pytest.mark.parametrize("M,N,K", [(64, 64, 16), (1, 1, 1), (77, 33, 5), (300, 129, 64), (1000, 700, 64),
                                   (130, 8, 600), (2053, 37, 64), (4096, 1100, 64)])
def test_fp64_zgemm_kernel_matches_torch(ctx, M, N, K):
    """The FP64 path's complex GEMM update C -= A B (DMMA kernel) against torch's FP64 product,
    with leading dimensions larger than the rows (sub-matrix views, as the LU passes them)."""
    lib = nat.load()
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    lda, ldb, ldc = M + 3, K + 1, M + 5
    A = torch.randn(K, lda, 2, generator=g, dtype=torch.float64)   # column-major complex (lda x K)
    B = torch.randn(N, ldb, 2, generator=g, dtype=torch.float64)
    C = torch.randn(N, ldc, 2, generator=g, dtype=torch.float64)
    dA, dB, dC = A.cuda(), B.cuda(), C.cuda()
    nat.check(lib.hprmat_b200_dev_zgemm(ctx._h, dA.data_ptr(), lda, dB.data_ptr(), ldb, dC.data_ptr(), ldc, M, N, K))
    Az = torch.complex(A[..., 0], A[..., 1]).T[:M, :K]
    Bz = torch.complex(B[..., 0], B[..., 1]).T[:K, :N]
    Cz = torch.complex(C[..., 0], C[..., 1]).T
    ref = Cz.clone()
    ref[:M, :N] -= Az @ Bz
    got = dC.cpu()
    got = torch.complex(got[..., 0], got[..., 1]).T
    assert torch.equal(got[M:, :], ref[M:, :])  # rows beyond M untouched
    err = (got - ref).abs().max().item()
    scale = (Az.abs() @ Bz.abs()).max().item()
    assert err <= 1e-14 * scale, (err, scale)


# ---------------------------------------------------------------- tensor-core kernel
@pytest.mark.parametrize("M,Nc,nb,bn", [(128, 256, 128, 256), (300, 520, 128, 256), (1000, 700, 64, 256),
                                        (77, 33, 32, 256), (640, 128, 128, 128), (129, 200, 64, 128),
                                        (4096, 1100, 128, 128), (2500, 2100, 64, 256)])
def test_tc_update_kernel_matches_fp64(ctx, M, Nc, nb, bn):
    lib = nat.load()
    g = torch.Generator(device="cpu").manual_seed(M + Nc)
    A = torch.randn(M, nb, 2, generator=g, dtype=torch.float32)
    B = torch.randn(Nc, nb, 2, generator=g, dtype=torch.float32)
    C = torch.randn(Nc, M, 2, generator=g, dtype=torch.float32)   # column-major complex (M x Nc)
    plane = max(M, Nc) * nb + 64
    dA = A.cuda().contiguous()
    dB = B.cuda().contiguous()
    dC = C.cuda().contiguous()
    aop = torch.zeros(4 * plane, dtype=torch.float32, device="cuda")
    bop = torch.zeros(4 * plane, dtype=torch.float32, device="cuda")
    h = ctx._h
    nat.check(lib.hprmat_b200_dev_split_planes(h, dA.data_ptr(), M, nb, aop.data_ptr(), plane))
    nat.check(lib.hprmat_b200_dev_split_planes(h, dB.data_ptr(), Nc, nb, bop.data_ptr(), plane))
    nat.check(lib.hprmat_b200_dev_tc_update(h, aop.data_ptr(), bop.data_ptr(), plane, nb, dC.data_ptr(), M, M, Nc,
                                            bn))
    torch.cuda.synchronize()
    Az = torch.complex(A[..., 0].double(), A[..., 1].double())          # M x nb
    Bz = torch.complex(B[..., 0].double(), B[..., 1].double())          # Nc x nb (column j = row j)
    Cz = torch.complex(C[..., 0].double(), C[..., 1].double()).T        # M x Nc
    ref = Cz - Az @ Bz.T
    got = dC.cpu().double()
    got = torch.complex(got[..., 0], got[..., 1]).T
    err = (got - ref).abs().max().item()
    scale = (Az.abs() @ Bz.abs().T).max().item()
    assert err <= 2e-6 * scale, (err, scale)


# ---------------------------------------------------------------- R-matrix path
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_small_workload_u_matches_oracle(ctx, precision):
    w = workloads.small()
    ref = _oracle_u(w)
    ctx.set_precision(precision)
    cu, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    assert nopen == ref.nopen == w.nch
    assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL, ctx.last_stats
    st = ctx.last_stats
    assert st["rel_residual"] < 1e-11


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ex1_and_ex2_through_the_abi(ctx, precision):
    """Reference examples 1 and 2 (ns = 1 cards): product == oracle, and the printed golden
    values of the reference are reproduced."""
    ctx.set_precision(precision)
    mesh = orc.rmat_ini(60, 1, 14.0)
    cpot, kin = ex1_setup(mesh.zrma)
    for e in (10.0, 20.0, 30.0, 40.0, 50.0):
        lval, qk, eta = kin(e, 20)
        cu, nopen = ctx.rmatrix(1, lval, qk, eta, 14.0, 60, 1, cpot)
        ref = orc.rmatrix(1, lval, qk, eta, 14.0, mesh, cpot).cu
        assert abs(cu[0, 0] - ref[0, 0]) <= U_TOL * abs(ref[0, 0])
    mesh = orc.rmat_ini(60, 1, 7.0)
    cpot, kin = ex2_setup(mesh.zrma, 1)
    for e in (12.0, 24.0, 36.0, 48.0):
        lval, qk, eta = kin(e)
        cu, nopen = ctx.rmatrix(2, lval, qk, eta, 7.0, 60, 1, cpot)
        ref = orc.rmatrix(2, lval, qk, eta, 7.0, mesh, cpot).cu
        assert _rel(cu[:2, :2], ref) <= U_TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ex4_closed_channels_single_interval(ctx, precision):
    """Ex4's 12C + alpha couplings with closed channels, one interval (nr = 100, a = 10)."""
    ctx.set_precision(precision)
    mesh = orc.rmat_ini(100, 1, 10.0)
    cpot, kin, nv = ex4_setup(mesh.zrma, 3)
    for e in (4.0, 8.0, 16.0):
        lval, qk, eta = kin(e)
        cu, nopen = ctx.rmatrix(nv, lval, qk, eta, 10.0, 100, 1, cpot)
        ref = orc.rmatrix(nv, lval, qk, eta, 10.0, mesh, cpot)
        assert nopen == ref.nopen
        assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_medium_production_generator(ctx, precision):
    """Production-generator physics at N = 4000 (20 channels x 200 points): open and closed
    channels, Coulomb, complex couplings."""
    w = workloads.production(nch=20)
    ref = _oracle_u(w)
    ctx.set_precision(precision)
    cu, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    assert nopen == ref.nopen
    assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL, ctx.last_stats


@pytest.mark.parametrize("nch", [32, 64, 128])
def test_production_generator_against_fixture(ctx, nch):
    """Production generator at N = 6400, 12800 and 25600 (200 points x nch channels) against
    the committed FP64 oracle collision matrices (tests/golden/make_production_u.py).  N = 6400
    puts 44 panel rows on each of the 148 CTAs, the shape whose shared memory sits just
    under the 48 KB default; N = 25600 (128 channels) is the headline configuration, where the
    call must also end with HPRMAT_B200_OK (refinement converged within its three steps)."""
    fx = np.load(os.path.join(GOLDEN, f"production_u_nch{nch}.npz"))
    w = workloads.production(nch=nch)
    ctx.set_precision("mixed")
    cu, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    st = ctx.last_stats
    assert st["status"] == nat.OK and st["refine_steps"] <= 3, st
    assert nopen == int(fx["nopen"])
    assert _rel(cu[:nopen, :nopen], fx["u"]) <= U_TOL, st


@pytest.mark.parametrize("nch", [50, 80, 128])
def test_sweep_generator_against_fixture(ctx, nch):
    """Precision-sweep generator (closed channels at 40 MeV) at N = 10000, 16000 and 25600
    against committed FP64 oracle collision matrices (tests/golden/make_production_u.py
    --sweep): the mixed path, refined to HPRMAT_B200_OK, within 1e-10 of LAPACK zgesv."""
    fx = np.load(os.path.join(GOLDEN, f"sweep_u_nch{nch}.npz"))
    w = workloads.sweep(nch)
    ctx.set_precision("mixed")
    cu, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    st = ctx.last_stats
    assert st["status"] == nat.OK, st
    assert nopen == int(fx["nopen"])
    assert _rel(cu[:nopen, :nopen], fx["u"]) <= U_TOL, st


@pytest.mark.parametrize("sb,un", [(1, 64), (2, 128), (4, 64), (4, 128)])
def test_wavefront_variants(sb, un):
    """The wavefront solves with other super-block sizes and unit widths (dev tuning hooks),
    on the production generator at N = 4200: 33 blocks of 128 rows, the last one partial and
    without a partner block when the diagonal inverses are doubled."""
    w = workloads.production(nch=21)
    ref = _oracle_u(w)
    c = api.Context(precision="mixed")
    lib = nat.load()
    nat.check(lib.hprmat_b200_dev_set_tuning(c._h, b"wave_sb", sb))
    nat.check(lib.hprmat_b200_dev_set_tuning(c._h, b"wave_un", un))
    cu, nopen = c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    assert nopen == ref.nopen
    assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL, c.last_stats
    c.close()


def test_wavefront_unit_width_switch_on_one_context():
    """Changing the unit width of the wavefront solves on a live context: with 100 right-hand
    sides one 128-column unit and two 64-column units pad to the same width, and the solves must
    still rebuild their operand maps for the new unit (100 channels x 24 points, N = 2400)."""
    w = workloads.production(nch=100, nr=24, rmax=10.0)
    ref = _oracle_u(w)
    c = api.Context(precision="mixed")
    lib = nat.load()
    for un in (128, 64, 128):
        nat.check(lib.hprmat_b200_dev_set_tuning(c._h, b"wave_un", un))
        cu, nopen = c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        assert nopen == ref.nopen
        assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL, (un, c.last_stats)
    c.close()


def test_block_size_change_on_one_context():
    """The block-step solves of the mixed path keep their right-hand-side planes between calls;
    a context that solved with 64-column blocks and then with 128-column ones at the same
    padded width must rebuild them (2 channels x 50 points: two blocks of 64, then one of 128)."""
    import ctypes
    w = workloads.production(nch=2, nr=50, rmax=10.0)
    ref = _oracle_u(w)
    lib = nat.load()
    c = api.Context(precision="mixed", panel_nb=64)
    for nb in (64, 0, 64, 0, 32, 0):
        c.opts.panel_nb = nb
        nat.check(lib.hprmat_b200_set_opts(c._h, ctypes.byref(c.opts)))
        cu, nopen = c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL, (nb, c.last_stats)
        assert c.last_stats["nb"] == (nb or 128)
    c.close()


def test_sweep_maximum_size_mixed_against_fp64():
    """The largest point of the precision sweep, 256 channels x 200 points (N = 51200, closed
    channels at 40 MeV; 69 GB on the device for the mixed path, 90 GB with the FP64 one): the
    panel no longer fits 128 columns, so the mixed path runs with 64-column blocks and the
    block-step solves.  No CPU oracle finishes at this size; the mixed U is checked against
    the device FP64 LU's (an independent algorithm and precision) and must converge within
    the default three refinement steps."""
    w = workloads.sweep(256)
    c = api.Context(precision="mixed")
    cu_m, nopen = c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    st = c.last_stats
    assert st["nb"] == 64 and st["refine_steps"] <= 3 and st["rel_residual"] < 1e-10, st
    c.set_precision("fp64")
    cu_d, nopen_d = c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    assert nopen == nopen_d == int((w.qk > 0).sum())
    assert _rel(cu_m[:nopen, :nopen], cu_d[:nopen, :nopen]) <= U_TOL
    c.close()


def test_sweep_generator_closed_at_40mev(ctx):
    w = workloads.sweep(20)
    ref = _oracle_u(w)
    ctx.set_precision("mixed")
    cu, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL, ctx.last_stats


# ---------------------------------------------------------------- dense solves
def _diag_dominant(n, nrhs, seed):
    """The reference's solver cross-check matrix (examples/Ex0/test_solver.f90:35-84):
    uniform random entries, A_ii += 2N, B_r = 1/sqrt(r)."""
    rng = np.random.default_rng(seed)
    A = rng.random((n, n)) + 1j * rng.random((n, n))
    A[np.arange(n), np.arange(n)] += 2 * n
    B = np.zeros((n, nrhs), np.complex128)
    for c in range(nrhs):
        B[:, c] = 1.0 / np.sqrt(np.arange(1, n + 1)) * (c + 1)
    return np.asfortranarray(A), np.asfortranarray(B)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n,nrhs", [(500, 8), (1000, 1), (2053, 37)])
def test_solve_linear_dense(ctx, precision, n, nrhs):
    A, B = _diag_dominant(n, nrhs, n)
    ctx.set_precision(precision)
    X = ctx.solve_linear(A, B)
    Xr = np.linalg.solve(A, B)
    assert _rel(X, Xr) <= 1e-12


@pytest.mark.parametrize("kappa", [1e2, 1e5, 1e8])
def test_solve_linear_exact_condition_number(ctx, kappa):
    """Householder A = H D H with geometric D (exact kappa), manufactured X = 1, as in
    examples/Ex0/benchmark_mgpu_illcond.f90:41-95."""
    n, nrhs = 1024, 4
    rng = np.random.default_rng(7)
    v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    v /= np.linalg.norm(v)
    H = np.eye(n) - 2 * np.outer(v, v.conj())
    d = kappa ** (-np.arange(n) / (n - 1))
    A = np.asfortranarray((H * d[None, :]) @ H)
    Xt = np.ones((n, nrhs), np.complex128)
    B = np.asfortranarray(A @ Xt)
    ctx.set_precision("mixed", max_refine=3, tol=1e-13)
    X = ctx.solve_linear(A, B, allow_unconverged=True)
    st = ctx.last_stats
    Xr = np.linalg.solve(A, B)
    err_ref = _rel(Xr, Xt)
    # refinement with FP64 residuals reaches a forward error of order kappa * u (u = 2^-53)
    assert _rel(X, Xt) <= max(10 * err_ref, 20 * kappa * 2.0 ** -53), (st, err_ref)


def test_fortran_dropins(ctx):
    lib = nat.load()
    n, nrhs = 700, 5
    A, B = _diag_dominant(n, nrhs, 3)
    Xr = np.linalg.solve(A, B)
    import ctypes
    for fn in ("mixed", "double"):
        Bw = np.array(B, order="F", copy=True)
        Ac = np.array(A, order="F", copy=True)
        info = ctypes.c_int(-7)
        nn, nr = ctypes.c_int(n), ctypes.c_int(nrhs)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if fn == "mixed":
            mr, tol = ctypes.c_int(3), ctypes.c_double(1e-13)
            r = lib.gpu_b200_solve_mixed_(dp(Ac), dp(Bw), ctypes.byref(nn), ctypes.byref(nr), ctypes.byref(mr),
                                          ctypes.byref(tol), ctypes.byref(info))
        else:
            r = lib.gpu_b200_solve_double_(dp(Ac), dp(Bw), ctypes.byref(nn), ctypes.byref(nr), ctypes.byref(info))
        assert r == 0 and info.value == 0
        assert np.array_equal(Ac, A)  # A is read only
        assert _rel(Bw, Xr) <= 1e-12
    assert lib.gpu_b200_finalize_() == 0


def test_solve_rmatrix_matches_oracle(ctx):
    w = workloads.small()
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    bnd = orc.boundary_values(w.nch, w.lval, w.qk, w.eta, w.rmax)
    C = orc.assemble(mesh, 1, w.nch, w.lval, w.qk, bnd.xc, w.cpot)
    bvec = mesh.q2[:, 0].astype(np.complex128)
    ref, _ = orc.solve_rmatrix_dense(C, bvec, w.nch, w.nr, 1.0)
    ctx.set_precision("mixed")
    rm = ctx.solve_rmatrix(C, bvec, w.nch, w.nr, 1.0)
    assert _rel(rm, ref) <= 1e-10


def _growth_matrix(nw=40, n=300, seed=5):
    """blockdiag(W, D): W (nw x nw) has 1 on the diagonal, -1/2 below it and 1 in its last
    column, so partial pivoting swaps nothing and |U| grows as 1.5^k (7.4e6 at nw = 40; the
    classic growth example for GEPP); D is diagonally dominant with entries below 1.  The whole
    matrix is turned by one complex phase.  X = 1 is exact: every row sum of W is exact."""
    A = np.zeros((n, n), np.complex128)
    W = np.eye(nw)
    W[np.tril_indices(nw, -1)] = -0.5
    W[:, -1] = 1.0
    A[:nw, :nw] = W
    rng = np.random.default_rng(seed)
    m = n - nw
    D = (rng.random((m, m)) + 1j * rng.random((m, m))) / (4 * m)
    D[np.arange(m), np.arange(m)] += 0.5
    A[nw:, nw:] = D
    A = np.asfortranarray(A * np.exp(0.3j))
    Xt = np.ones((n, 3), np.complex128)
    return A, Xt


def _growth_of(A):
    """max |u_ij| / max |a_ij| with |z| = |re| + |im| (the solver's measure), numpy LU."""
    import scipy.linalg as sl
    _p, _l, u = sl.lu(A)
    m1 = lambda z: np.abs(z.real) + np.abs(z.imag)
    return float(m1(u).max() / m1(A).max())


def test_pivot_growth_falls_back_to_fp64(ctx):
    """The mixed solve measures the pivot growth of its FP32 factors and, above 10^6,
    factorises A in FP64 instead (the FP32 factors of this matrix carry no correct digit in
    the last column of W)."""
    A, Xt = _growth_matrix()
    B = np.asfortranarray(A @ Xt)
    rho = _growth_of(A)
    assert rho > 1e6
    ctx.set_precision("mixed", max_refine=3, tol=1e-12)
    X = ctx.solve_linear(A, B)
    st = ctx.last_stats
    assert st["fp64_fallback"] == 1 and st["factorizations"] == 2, st
    assert abs(st["pivot_growth"] / rho - 1.0) < 1e-3, (st["pivot_growth"], rho)
    err_np = _rel(np.linalg.solve(A, B), Xt)
    assert _rel(X, Xt) <= max(10 * err_np, 1e-9), (_rel(X, Xt), err_np)
    # the same matrix through the FP64 path reports the same growth, without a fallback
    ctx.set_precision("fp64")
    X = ctx.solve_linear(A, B)
    st = ctx.last_stats
    assert st["fp64_fallback"] == 0 and st["factorizations"] == 1
    assert abs(st["pivot_growth"] / rho - 1.0) < 1e-3
    assert _rel(X, Xt) <= max(10 * err_np, 1e-9)
    ctx.set_precision("mixed", max_refine=3, tol=1e-12)


def test_pivot_growth_limit_is_the_trigger():
    """With the limit raised to 10^12 the same matrix stays on the FP32 factors; a
    well-conditioned matrix reports a growth of order 1 and no fallback."""
    lib = nat.load()
    with api.Context(precision="mixed") as c:
        nat.check(lib.hprmat_b200_dev_set_tuning(c._h, b"growth_limit_exp", 12))
        A, Xt = _growth_matrix()
        c.solve_linear(A, np.asfortranarray(A @ Xt), allow_unconverged=True)
        assert c.last_stats["fp64_fallback"] == 0 and c.last_stats["factorizations"] == 1
        assert c.last_stats["pivot_growth"] > 1e6
        A, B = _diag_dominant(500, 4, 9)
        c.solve_linear(A, B)
        assert c.last_stats["fp64_fallback"] == 0 and 0.5 < c.last_stats["pivot_growth"] < 2.0
        assert lib.hprmat_b200_dev_set_tuning(c._h, b"growth_limit_exp", 31) == nat.ERR_ARG


def test_pivot_growth_error_on_request():
    """opts.growth_error: the same growth matrix makes the mixed solve return
    HPRMAT_B200_PIVOT_GROWTH (with the growth in the stats) instead of factorising in FP64."""
    import ctypes
    lib = nat.load()
    A, Xt = _growth_matrix()
    with api.Context(precision="mixed") as c:
        c.opts.growth_error = 1
        nat.check(lib.hprmat_b200_set_opts(c._h, ctypes.byref(c.opts)))
        with pytest.raises(nat.HprmatError) as e:
            c.solve_linear(A, np.asfortranarray(A @ Xt))
        assert e.value.status == nat.PIVOT_GROWTH
        assert c.last_stats["pivot_growth"] > 1e6 and c.last_stats["fp64_fallback"] == 0
        A2, B2 = _diag_dominant(300, 2, 6)
        X2 = c.solve_linear(A2, B2)
        assert _rel(X2, np.linalg.solve(A2, B2)) <= 1e-12


def test_rmatrix_fp64_fallback_matches_oracle():
    """The R-matrix path's fallback, forced by a growth limit of 10^-30: C(E) factorised in
    FP32, then again in FP64, and U to the refined oracle U within 1e-10 or five times the
    unrefined oracle's own error.  A plain FP64 LU stops at its rounding level: this library's
    lands 8e-11 to 1.1e-10 from the unrefined oracle's U here, depending on the order of its
    roundings (single or paired block steps), the oracle 1.5e-11 from the refined U.  The production C(E) itself has a small
    growth and stays on the mixed path."""
    lib = nat.load()
    w = workloads.production(nch=8)
    ref = _oracle_u(w)
    u_ref = _refined_u(w)
    tol = max(U_TOL, 5 * _rel(ref.cu, u_ref))
    with api.Context(precision="mixed") as c:
        c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        st = c.last_stats
        assert st["fp64_fallback"] == 0 and st["factorizations"] == 1 and st["pivot_growth"] < 1e3, st
        nat.check(lib.hprmat_b200_dev_set_tuning(c._h, b"growth_limit_exp", -30))
        cu, nopen = c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        st = c.last_stats
        assert st["fp64_fallback"] == 1 and st["factorizations"] == 2, st
        assert nopen == ref.nopen
        assert _rel(cu[:nopen, :nopen], u_ref) <= tol, (tol, st)


@pytest.mark.parametrize("kappa", [1e3, 1e8])
def test_condition_estimate_dense(kappa):
    """opts.estimate_condition on the FP64 path: the Hager-Higham estimate of ||A||_1 ||A^-1||_1
    against numpy's exact 1-norm condition number (a lower bound, within a factor 3 here),
    for the exact-kappa Householder matrices and a diagonally dominant one."""
    n = 700
    rng = np.random.default_rng(3)
    v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    v /= np.linalg.norm(v)
    H = np.eye(n) - 2 * np.outer(v, v.conj())
    d = kappa ** (-np.arange(n) / (n - 1))
    A = np.asfortranarray((H * d[None, :]) @ H)
    B = np.asfortranarray(A @ np.ones((n, 2), np.complex128))
    exact = float(np.linalg.cond(A, 1))
    with api.Context(precision="fp64") as c:
        c.solve_linear(A, B)
        assert c.last_stats["cond_estimate"] == 0.0  # off by default
        c.set_estimate_condition(True)
        X = c.solve_linear(A, B)
        est = c.last_stats["cond_estimate"]
        assert exact / 3.0 <= est <= exact * (1 + 1e-6), (est, exact)
        assert abs(est / orc.cond1_estimate(A) - 1.0) < 1e-6  # the oracle's steps, the same estimate
        assert _rel(X, np.linalg.solve(A, B)) <= 1e-12 * max(1.0, kappa / 1e3)
        A2, B2 = _diag_dominant(500, 2, 4)
        c.solve_linear(A2, B2)
        ex2 = float(np.linalg.cond(A2, 1))
        assert ex2 / 3.0 <= c.last_stats["cond_estimate"] <= ex2 * (1 + 1e-6)


def test_condition_estimate_rmatrix_and_fallback():
    """The same estimate of C(E) on the R-matrix FP64 path (against numpy on the oracle's
    assembled C) and after a forced FP64 fallback of the mixed path; none on the mixed path."""
    lib = nat.load()
    w = workloads.small()
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    bnd = orc.boundary_values(w.nch, w.lval, w.qk, w.eta, w.rmax)
    C = orc.assemble(mesh, 1, w.nch, w.lval, w.qk, bnd.xc, w.cpot)
    exact = float(np.linalg.cond(C, 1))
    with api.Context(precision="fp64") as c:
        c.set_estimate_condition(True)
        c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        est = c.last_stats["cond_estimate"]
        assert exact / 3.0 <= est <= exact * (1 + 1e-6), (est, exact)
        assert abs(est / orc.cond1_estimate(C) - 1.0) < 1e-6
        c.set_precision("mixed")
        c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        assert c.last_stats["cond_estimate"] == 0.0
        nat.check(lib.hprmat_b200_dev_set_tuning(c._h, b"growth_limit_exp", -30))
        c.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        assert c.last_stats["fp64_fallback"] == 1
        assert abs(c.last_stats["cond_estimate"] / est - 1.0) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nch,nr", [(5, 37), (3, 51), (1, 600)])
def test_odd_and_long_meshes(ctx, precision, nch, nr):
    """Mesh sizes that are odd, or longer than the assembly's column stride (512): the
    assembly steps the (channel, point) pair of a column instead of dividing, so these check
    its wrap-around against the oracle."""
    w = workloads.production(seed=41 + nr, nch=nch, nr=nr, rmax=20.0, energy=10.0, name=f"mesh{nr}")
    ref = _oracle_u(w)
    # at nr = 600 (one channel) C has kappa_2 = 9.4e9 and the oracle's own unrefined zgesv U is
    # only good to ~8e-10: the reference U here is the oracle's, refined with residuals in
    # extended precision until it no longer changes
    u_ref = _refined_u(w)
    ctx.set_precision(precision)
    cu, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    assert nopen == ref.nopen
    if nopen:
        oracle_err = _rel(ref.cu, u_ref)
        # the refined mixed path reaches the refined U; a plain FP64 LU (here and in the oracle)
        # stops at its rounding level
        tol = U_TOL if precision == "mixed" else max(U_TOL, 5 * oracle_err)
        assert _rel(cu[:nopen, :nopen], u_ref) <= tol, (oracle_err, ctx.last_stats)
    ctx.set_precision("mixed")


@pytest.mark.parametrize("n", [449, 1000, 2117])
def test_fp64_paired_block_steps(ctx, n):
    """The plain FP64 LU runs two 64-column block steps per K = 128 trailing update (the second
    step's interchanges applied to the first step's multipliers through a gathered operand).  On
    general complex matrices (every column pivots; odd step counts and a ragged last panel) the
    paired and the single-step factorisations both solve to FP64 accuracy and agree."""
    rng = np.random.default_rng(n)
    A = np.asfortranarray(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    B = np.asfortranarray(rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3)))
    Xnp = np.linalg.solve(A, B)
    lib = nat.load()
    ctx.set_precision("fp64")
    out = {}
    try:
        for pair in (1, 0):
            nat.check(lib.hprmat_b200_dev_set_tuning(ctx._h, b"f64_pair", pair))
            out[pair] = ctx.solve_linear(A, B)
            assert ctx.last_stats["status"] == nat.OK and ctx.last_stats["info"] == 0
    finally:
        nat.check(lib.hprmat_b200_dev_set_tuning(ctx._h, b"f64_pair", 1))
        ctx.set_precision("mixed")
    for pair in (1, 0):
        assert _rel(out[pair], Xnp) <= 1e-11, pair
    assert _rel(out[1], out[0]) <= 1e-11


@pytest.mark.parametrize("scale", [1e-300, 1e300])
def test_fp64_pivoting_outside_float_range(ctx, scale):
    """FP64 dense solve of a matrix whose entries lie far outside the float range (1e-300 or
    1e300 times O(1) values) with a zero diagonal, so every column needs a row interchange:
    the FP64 panels compare pivot candidates over the whole double range (as zgetrf does),
    so they pivot to the largest entry instead of reporting a false zero pivot."""
    rng = np.random.default_rng(21)
    n, nrhs = 300, 5
    A0 = rng.uniform(0.5, 1.5, (n, n)) + 1j * rng.uniform(-0.5, 0.5, (n, n))
    A0[np.arange(n), np.arange(n)] = 0.0
    A = np.asfortranarray(A0 * scale)
    B = np.asfortranarray(rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)))
    Xnp = np.linalg.solve(A, B)
    ctx.set_precision("fp64")
    X = ctx.solve_linear(A, B)
    assert ctx.last_stats["status"] == nat.OK and ctx.last_stats["info"] == 0
    s = 1.0 / np.abs(Xnp).max()  # norms of 1e300-sized values overflow: compare scaled copies
    assert _rel(X * s, Xnp * s) <= 1e-12
    ctx.set_precision("mixed")


# ---------------------------------------------------------------- failures
def test_singular_matrix_reports_status(ctx):
    n = 300
    A, B = _diag_dominant(n, 2, 11)
    A[:, 17] = 0.0
    for prec in ("fp64", "mixed"):
        ctx.set_precision(prec)
        with pytest.raises(nat.HprmatError) as e:
            ctx.solve_linear(A, B)
        assert e.value.status == nat.SINGULAR
        assert ctx.last_stats["info"] == 18


def test_bounded_wait_reports_timeout_and_context_survives(ctx):
    """The panel barrier's bounded wait, run out on purpose on a counter nothing increments
    (2^14 polls, ~10 ms): the host reads HPRMAT_B200_ERR_TIMEOUT with the site, and the same
    context then solves correctly."""
    lib = nat.load()
    assert lib.hprmat_b200_dev_wait_probe(ctx._h, 1 << 14) == nat.ERR_TIMEOUT
    assert b"site 99" in lib.hprmat_b200_last_error()
    assert lib.hprmat_b200_dev_wait_probe(ctx._h, 100) == nat.ERR_ARG
    w = workloads.small()
    ref = _oracle_u(w)
    ctx.set_precision("mixed")
    cu, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL


def test_refinement_cap_reports_not_converged(ctx):
    """max_refine = 0 with a tolerance the FP32-accurate factors cannot reach."""
    w = workloads.production(nch=20)
    ctx.set_precision("mixed", max_refine=0, tol=1e-13)
    with pytest.raises(nat.HprmatError) as e:
        ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
    assert e.value.status == nat.NOT_CONVERGED
    cu, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot, allow_unconverged=True)
    assert ctx.last_stats["rel_residual"] > 1e-13
    ctx.set_precision("mixed", max_refine=3, tol=1e-13)


def test_bad_arguments(ctx):
    lib = nat.load()
    assert lib.hprmat_b200_solve_linear(ctx._h, None, None, 0, 1, None) == nat.ERR_ARG
    w = workloads.small()
    with pytest.raises(nat.HprmatError) as e:
        ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 2, w.cpot)
    assert e.value.status in (nat.ERR_UNSUPPORTED, nat.ERR_ARG)
