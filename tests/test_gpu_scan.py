"""Batched energy scan (hprmat_b200_rmatrix_scan) against the FP64 oracle, unit by unit.

A small version of the scan workload: J-pi blocks with uneven channel counts on a 60-point
mesh, several energies each (open and closed channels), solved by concurrent worker streams.
Every collision matrix must agree with the oracle's to 1e-10 (relative Frobenius), as for the
single-energy entry point.
"""
import numpy as np
import pytest

from hprmat_b200 import api, workloads
from oracle import rmatrix_oracle as orc

pytestmark = pytest.mark.gpu

U_TOL = 1e-10


def _blocks():
    out = []
    for b, (nch, energies) in enumerate([(4, [2.0, 11.0]), (13, [5.0, 17.5, 29.0]), (24, [8.0, 21.0])]):
        w = workloads.production(seed=500 + b, nch=nch, nr=60, rmax=20.0, energy=1.0, name=f"scan{b}")
        ks = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in energies]
        qk = np.array([k[0] for k in ks])
        eta = np.array([k[1] for k in ks])
        out.append((w, qk, eta))
    return out


@pytest.mark.parametrize("precision,nworkers", [("mixed", 3), ("fp64", 2)])
def test_scan_matches_oracle_per_unit(precision, nworkers):
    blocks = _blocks()
    ctx = api.Context(precision=precision)
    res = ctx.rmatrix_scan([(w.lval, w.cpot, qk, eta) for w, qk, eta in blocks], 20.0, 60, nworkers=nworkers)
    mesh = orc.rmat_ini(60, 1, 20.0)
    for (w, qk, eta), (cu, nopen, status) in zip(blocks, res):
        for e in range(qk.shape[0]):
            ref = orc.rmatrix(w.nch, w.lval, qk[e], eta[e], 20.0, mesh, w.cpot)
            assert status[e] == 0
            assert nopen[e] == ref.nopen
            no = ref.nopen
            err = np.linalg.norm(cu[e, :no, :no] - ref.cu) / np.linalg.norm(ref.cu)
            assert err <= U_TOL, (w.nch, e, err)
    assert ctx.last_scan_seconds > 0.0
    ctx.close()


def test_scan_rejects_inconsistent_blocks():
    w = workloads.small()
    ctx = api.Context()
    with pytest.raises(ValueError):
        ctx.rmatrix_scan([(w.lval, w.cpot, np.zeros((2, 3)), np.zeros((2, 3)))], 10.0, 50)
    ctx.close()


def _dense_scan_blocks():
    """Two blocks with 24 energies each on 1..29 MeV (spacing ~1.2 MeV), unsorted, so that a
    worker walks them in energy order and keeps its factorisation across a run."""
    rng = np.random.default_rng(9)
    out = []
    for b, nch in enumerate([9, 30]):
        w = workloads.production(seed=700 + b, nch=nch, nr=60, rmax=20.0, energy=1.0, name=f"dscan{b}")
        energies = rng.permutation(np.linspace(1.0, 29.0, 24))
        ks = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in energies]
        out.append((w, np.array([k[0] for k in ks]), np.array([k[1] for k in ks])))
    return out


def test_scan_with_factor_reuse_matches_oracle():
    """opts.reuse_factors: the refinement runs on the factors of a nearby energy of the same
    block (C(E) changes only on the diagonal between energies); every unit still agrees with
    the oracle to 1e-10, with fewer factorisations than units."""
    from hprmat_b200 import _native as nat
    lib = nat.load()
    blocks = _dense_scan_blocks()
    ctx = api.Context(precision="mixed", reuse_factors=True)
    lib.hprmat_b200_dev_factorizations(ctx._h, 1)
    res = ctx.rmatrix_scan([(w.lval, w.cpot, qk, eta) for w, qk, eta in blocks], 20.0, 60, nworkers=2,
                           raise_on_unit_error=False)
    nfact = lib.hprmat_b200_dev_factorizations(ctx._h, 1)
    mesh = orc.rmat_ini(60, 1, 20.0)
    nunits = 0
    for (w, qk, eta), (cu, nopen, status) in zip(blocks, res):
        for e in range(qk.shape[0]):
            if status[e] != 0:
                continue  # COULFG cannot evaluate some channels just above threshold
            ref = orc.rmatrix(w.nch, w.lval, qk[e], eta[e], 20.0, mesh, w.cpot)
            no = ref.nopen
            err = np.linalg.norm(cu[e, :no, :no] - ref.cu) / np.linalg.norm(ref.cu)
            assert err <= U_TOL, (w.nch, e, err)
            nunits += 1
    assert nunits >= 40
    assert 0 < nfact < nunits, (nfact, nunits)
    ctx.close()


def test_reuse_across_energies_single_calls():
    """rmatrix with reuse_factors on one context, energies of one block in order and one far jump:
    every result equals the oracle's (the far jump is refactorised if the refinement on the held
    factors does not converge), and a different potential is never solved on held factors."""
    w = workloads.production(seed=3, nch=20, nr=60, rmax=16.0)
    mesh = orc.rmat_ini(60, 1, 16.0)
    ctx = api.Context(precision="mixed", reuse_factors=True)
    facts = []
    for e in [6.0, 6.3, 6.6, 7.0, 25.0]:
        wk = workloads.at_energy(w, e)
        cu, nopen = ctx.rmatrix(w.nch, w.lval, wk.qk, wk.eta, 16.0, 60, 1, w.cpot)
        ref = orc.rmatrix(w.nch, w.lval, wk.qk, wk.eta, 16.0, mesh, w.cpot)
        err = np.linalg.norm(cu[:nopen, :nopen] - ref.cu) / np.linalg.norm(ref.cu)
        assert err <= U_TOL, (e, err, ctx.last_stats)
        facts.append(ctx.last_stats["factorizations"])
    assert facts[0] == 1 and sum(facts[1:4]) == 0, facts
    # a different potential is never solved with the held factors
    w2 = workloads.production(seed=4, nch=20, nr=60, rmax=16.0)
    cu, nopen = ctx.rmatrix(w2.nch, w2.lval, w2.qk, w2.eta, 16.0, 60, 1, w2.cpot)
    assert ctx.last_stats["factorizations"] == 1
    ref = orc.rmatrix(w2.nch, w2.lval, w2.qk, w2.eta, 16.0, mesh, w2.cpot)
    assert np.linalg.norm(cu[:nopen, :nopen] - ref.cu) / np.linalg.norm(ref.cu) <= U_TOL
    ctx.close()


def test_scan_autotune_table_and_parity():
    """hprmat_b200_scan_autotune: one row per distinct order with settings from its candidate
    sets; a scan with the table gives every unit to 1e-10 of the oracle; the table survives a
    get/set round trip, rejects an invalid row, and clears."""
    from hprmat_b200 import _native as nat
    blocks = _blocks()
    args = [(w.lval, w.cpot, qk, eta) for w, qk, eta in blocks]
    ctx = api.Context(precision="mixed")
    table = ctx.scan_autotune(args, 20.0, 60, nworkers=2)
    assert ctx.last_autotune_seconds > 0.0
    assert sorted(r["N"] for r in table) == sorted(w.nch * 60 for w, _q, _e in blocks)
    for r in table:
        assert r["nb"] in (32, 64, 128) and r["panel_cluster"] in (0, 1)
        assert r["panel_rpc_min"] in (16, 32, 64) and r["wave_sb"] in (0, 1, 2)
        assert r["gmres_m"] in (8, 12, 16) and r["tc_grid"] >= 0 and r["ms"] > 0.0
    res = ctx.rmatrix_scan(args, 20.0, 60, nworkers=3)
    mesh = orc.rmat_ini(60, 1, 20.0)
    for (w, qk, eta), (cu, nopen, status) in zip(blocks, res):
        for e in range(qk.shape[0]):
            ref = orc.rmatrix(w.nch, w.lval, qk[e], eta[e], 20.0, mesh, w.cpot)
            assert status[e] == 0 and nopen[e] == ref.nopen
            no = ref.nopen
            assert np.linalg.norm(cu[e, :no, :no] - ref.cu) / np.linalg.norm(ref.cu) <= U_TOL
    # a table forcing 64-column blocks, grid panels, short cycles and a trailing update on 37
    # CTAs for every order still agrees
    forced = [dict(N=w.nch * 60, nb=64, panel_cluster=0, panel_rpc_min=16, wave_sb=1, gmres_m=8, tc_grid=37)
              for w, _q, _e in blocks]
    ctx.set_scan_tune_table(forced)
    assert [{k: r[k] for k in api.Context.TUNE_KEYS} for r in ctx.scan_tune_table()] == forced
    res = ctx.rmatrix_scan(args, 20.0, 60, nworkers=2)
    for (w, qk, eta), (cu, nopen, status) in zip(blocks, res):
        ref = orc.rmatrix(w.nch, w.lval, qk[-1], eta[-1], 20.0, mesh, w.cpot)
        no = ref.nopen
        assert status[-1] == 0
        assert np.linalg.norm(cu[-1, :no, :no] - ref.cu) / np.linalg.norm(ref.cu) <= U_TOL
    bad = dict(forced[0], nb=96)
    with pytest.raises(nat.HprmatError):
        ctx.set_scan_tune_table([bad])
    ctx.set_scan_tune_table([])
    assert ctx.scan_tune_table() == []
    ctx.close()


@pytest.mark.parametrize("blocked", [1, 0])
def test_hessenberg_reduction_is_a_unitary_similarity(blocked):
    """The device Householder reduction, in panels with GEMM updates (blocked) and column by
    column: A = P H P^H with P unitary and H upper Hessenberg, on random complex matrices (one
    order a multiple of the panel width plus two, one not) and on a C(E)-like matrix with a wide
    range of entry sizes."""
    import torch
    from hprmat_b200 import _native as nat
    lib = nat.load()
    ctx = api.Context(precision="fp64")
    nat.check(lib.hprmat_b200_dev_set_tuning(ctx._h, b"hess_blocked", blocked))
    rng = np.random.default_rng(3)
    w = workloads.production(seed=41, nch=5, nr=60, rmax=20.0)
    mesh = orc.rmat_ini(60, 1, 20.0)
    bnd = orc.boundary_values(w.nch, w.lval, w.qk, w.eta, 20.0)
    cases = [rng.standard_normal((300, 300)) + 1j * rng.standard_normal((300, 300)),
             rng.standard_normal((98, 98)) + 1j * rng.standard_normal((98, 98)),
             orc.assemble(mesh, 1, w.nch, w.lval, w.qk, bnd.xc, w.cpot)]
    for A in cases:
        n = A.shape[0]
        lda = n + 2
        buf = np.zeros((n, lda), complex)  # column-major (lda x n)
        buf[:, :n] = A.T
        dA = torch.from_numpy(buf.view(np.float64).copy()).cuda()
        dP = torch.zeros_like(dA)
        nat.check(lib.hprmat_b200_dev_hessenberg(ctx._h, dA.data_ptr(), lda, n, dP.data_ptr()))
        H = dA.cpu().numpy().view(complex).reshape(n, lda)[:, :n].T
        P = dP.cpu().numpy().view(complex).reshape(n, lda)[:, :n].T
        assert np.abs(np.tril(H, -2)).max() == 0.0
        assert np.abs(P.conj().T @ P - np.eye(n)).max() <= 1e-13
        assert np.linalg.norm(P @ H @ P.conj().T - A) <= 1e-14 * np.linalg.norm(A) * n ** 0.5
    ctx.close()


def test_shifted_scan_matches_oracle_per_unit():
    """The shifted (Hessenberg) scan: one reduction per block, O(N^2 nch) per energy plus FP64
    refinement; every unit agrees with the oracle to 1e-10, without sending units to the LU path."""
    from hprmat_b200 import _native as nat
    blocks = _blocks()
    ctx = api.Context(precision="mixed")
    res = ctx.rmatrix_scan([(w.lval, w.cpot, qk, eta) for w, qk, eta in blocks], 20.0, 60, method="shifted")
    mesh = orc.rmat_ini(60, 1, 20.0)
    for (w, qk, eta), (cu, nopen, status) in zip(blocks, res):
        for e in range(qk.shape[0]):
            ref = orc.rmatrix(w.nch, w.lval, qk[e], eta[e], 20.0, mesh, w.cpot)
            assert status[e] == nat.OK
            assert nopen[e] == ref.nopen
            no = ref.nopen
            err = np.linalg.norm(cu[e, :no, :no] - ref.cu) / np.linalg.norm(ref.cu)
            assert err <= U_TOL, (w.nch, e, err)
    ctx.close()


def test_shifted_scan_workers_give_identical_results():
    """Blocks dealt to concurrent worker contexts (hess_workers) go through the same kernels as
    one block at a time; every energy's arithmetic is independent of the batch and the stream it
    runs in, so U, nopen and status are bitwise the same for 1 and 3 workers."""
    from hprmat_b200 import _native as nat
    lib = nat.load()
    blocks = _blocks()
    args = [(w.lval, w.cpot, qk, eta) for w, qk, eta in blocks]
    ctx = api.Context(precision="mixed")
    out = {}
    for nw in (1, 3):
        nat.check(lib.hprmat_b200_dev_set_tuning(ctx._h, b"hess_workers", nw))
        out[nw] = ctx.rmatrix_scan(args, 20.0, 60, method="shifted")
    for (cu1, no1, st1), (cu3, no3, st3) in zip(out[1], out[3]):
        assert np.array_equal(st1, st3) and np.array_equal(no1, no3)
        assert np.array_equal(cu1, cu3)
    assert lib.hprmat_b200_dev_set_tuning(ctx._h, b"hess_workers", 0) == nat.ERR_ARG
    ctx.close()


def test_shifted_scan_on_a_config3_sample():
    """A sample of the energy-scan configuration (blocks of 4..64 channels x 60 points, energies
    in 1-30 MeV): the shifted scan against the oracle on every fourth energy of three blocks,
    and against the LU scan on all of them."""
    from oracle import special_functions as sf
    blocks = workloads.scan_blocks()
    picked = []
    for w, energies in [blocks[i] for i in (0, 5, 9)]:
        ks = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in energies[::16]]
        ks = [k for k in ks if all(sf.coulfg(k[0][c] * w.rmax, k[1][c], float(w.lval[c]))[4] == 0
                                   for c in range(w.nch) if k[0][c] > 0)]
        picked.append((w, np.array([k[0] for k in ks]), np.array([k[1] for k in ks])))
    args = [(w.lval, w.cpot, qk, eta) for w, qk, eta in picked]
    ctx = api.Context(precision="mixed")
    res_s = ctx.rmatrix_scan(args, 20.0, 60, method="shifted")
    res_l = ctx.rmatrix_scan(args, 20.0, 60, nworkers=2)
    mesh = orc.rmat_ini(60, 1, 20.0)
    for (w, qk, eta), (cu, nopen, st), (cl, nl, sl) in zip(picked, res_s, res_l):
        for e in range(qk.shape[0]):
            no = nopen[e]
            assert st[e] == 0 and sl[e] == 0 and nl[e] == no
            assert np.linalg.norm(cu[e, :no, :no] - cl[e, :no, :no]) <= U_TOL * np.linalg.norm(cl[e, :no, :no])
            if e % 4 == 0:
                ref = orc.rmatrix(w.nch, w.lval, qk[e], eta[e], 20.0, mesh, w.cpot)
                assert np.linalg.norm(cu[e, :no, :no] - ref.cu) <= U_TOL * np.linalg.norm(ref.cu), (w.nch, e)
    ctx.close()
