"""The oracle against the reference's golden outputs (CPU).

tests/golden/reference_examples.json holds the printed results of Descouvemont's
examples (rmat_pierre/Ex{1,2,3,4}/output*.txt and the wave functions wf*.txt), extracted by
tests/golden/make_golden.py.  The oracle must reproduce them to the printed 5 significant
digits for every mesh card, including the multi-interval (ns > 1) ones, Ex4's closed channels
(WHIT path), the internal and external wave functions and Ex3's wf_print interpolation.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import rmatrix_oracle as orc
from tests.example_inputs import ex1_setup, ex2_setup, ex3_setup, ex4_setup, ex5_setup
from oracle.special_functions import coulfg, whit

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_examples.json")))


def _printed_close(x, ref, rel=6e-5, abs_=1e-12):
    """Agreement at the printed precision: 5 significant digits (es12.4)."""
    return abs(x - ref) <= rel * abs(ref) + abs_


@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex1"])))
def test_ex1_collision_matrix(card):
    c = GOLD["examples"]["ex1"][card]
    nr, ns, rmax = c["nr"], c["ns"], abs(c["rmax"])
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin = ex1_setup(mesh.zrma)
    for row in c["printed"]["Collision matrix="]:
        lval, qk, eta = kin(row["E"], c["j"])
        u = orc.rmatrix(1, lval, qk, eta, rmax, mesh, cpot).cu[0, 0]
        re, im = row["values"]
        assert _printed_close(u.real, re), (row["E"], u, re)
        # imaginary parts below ~1e-10 are rounding-level; compare against |U| there
        assert abs(u.imag - im) <= 6e-5 * max(abs(im), 1e-14 if abs(im) > 1e-10 else abs(u)), (row["E"], u, im)


@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex2"])))
def test_ex2_phase_shifts(card):
    c = GOLD["examples"]["ex2"][card]
    nr, ns, rmax, j = c["nr"], c["ns"], abs(c["rmax"]), c["j"]
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin = ex2_setup(mesh.zrma, j)
    for row in c["printed"]["phase shift (rad.)="]:
        lval, qk, eta = kin(row["E"])
        cu = orc.rmatrix(2, lval, qk, eta, rmax, mesh, cpot).cu
        d1 = math.atan2(cu[0, 0].imag, cu[0, 0].real) / 2
        d2 = math.atan2(cu[1, 1].imag, cu[1, 1].real) / 2
        for x, ref in zip([d1, d2, abs(cu[0, 1])], row["values"]):
            assert _printed_close(x, ref), (row["E"], x, ref)


@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex4"])))
def test_ex4_amplitudes_closed_channels(card):
    c = GOLD["examples"]["ex4"][card]
    nr, ns, rmax, j = c["nr"], c["ns"], abs(c["rmax"]), c["j"]
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin, nv = ex4_setup(mesh.zrma, j)
    amps = c["printed"]["Amplitude="]
    phs = c["printed"]["phase shift (rad.)="]
    saw_closed = False
    for ra, rp in zip(amps, phs):
        lval, qk, eta = kin(ra["E"])
        saw_closed |= bool((qk < 0).any())
        res = orc.rmatrix(nv, lval, qk, eta, rmax, mesh, cpot)
        col = res.cu[:res.nopen, 0]
        assert len(ra["values"]) == res.nopen
        for x, ref in zip(np.abs(col), ra["values"]):
            assert _printed_close(x, ref, rel=1.2e-4), (ra["E"], x, ref)
        for x, ref in zip(np.arctan2(col.imag, col.real) / 2, rp["values"]):
            assert abs(x - ref) <= 1.2e-4 * max(abs(ref), 1.0), (rp["E"], x, ref)
    assert saw_closed


@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex3"])))
def test_ex3_amplitudes(card):
    c = GOLD["examples"]["ex3"][card]
    nr, ns, rmax, j = c["nr"], c["ns"], abs(c["rmax"]), c["j"]
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin, nv = ex3_setup(mesh.zrma, j)
    for ra, rp in zip(c["printed"]["Amplitude="], c["printed"]["phase shift (rad.)="]):
        lval, qk, eta = kin(ra["E"])
        res = orc.rmatrix(nv, lval, qk, eta, rmax, mesh, cpot)
        col = res.cu[:res.nopen, 0]
        for x, ref in zip(np.abs(col), ra["values"]):
            assert _printed_close(x, ref, rel=1.2e-4), (ra["E"], x, ref)
        for x, ref in zip(np.arctan2(col.imag, col.real) / 2, rp["values"]):
            assert abs(x - ref) <= 1.2e-4 * max(abs(ref), 1.0), (rp["E"], x, ref)


@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex5"])))
def test_ex5_nonlocal_phase_shifts(card):
    """Yamaguchi's non-local potential (full nr x nr block term of rmatrix_hp.F90:283-288)."""
    c = GOLD["examples"]["ex5"][card]
    nr, rmax = c["nr"], abs(c["rmax"])
    mesh = orc.rmat_ini(nr, 1, rmax)
    cpot, cpnl, kin = ex5_setup(mesh.zrma)
    for row in c["printed"]["phase shift (deg.)="]:
        lval, qk, eta = kin(row["E"])
        u = orc.rmatrix(1, lval, qk, eta, rmax, mesh, cpot, cpnl=cpnl).cu[0, 0]
        delta = math.atan2(u.imag, u.real) / 2 * 180 / math.pi
        assert _printed_close(delta, row["values"][0]), (row["E"], delta, row["values"])
        assert _printed_close(abs(u), row["values"][1]), (row["E"], abs(u))


def wf_case(name):
    """(mesh, rmax, cpot, kin, nch, blocks, cpnl) of the wave-function card of example ``name``
    (cpnl: the non-local potential of Ex5, else None)."""
    wf = GOLD["wavefunctions"][name]
    c = GOLD["examples"][name][wf["card"]]
    nr, ns, rmax = c["nr"], c["ns"], abs(c["rmax"])
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpnl = None
    if name == "ex1":
        cpot, k1 = ex1_setup(mesh.zrma)
        kin, nv = (lambda e: k1(e, c["j"])), 1
    elif name == "ex5":
        cpot, cpnl, kin = ex5_setup(mesh.zrma)
        nv = 1
    elif name == "ex2":
        cpot, kin = ex2_setup(mesh.zrma, c["j"])
        nv = 2
    else:
        cpot, kin, nv = (ex3_setup if name == "ex3" else ex4_setup)(mesh.zrma, c["j"])
    return mesh, rmax, cpot, kin, nv, wf["blocks"], cpnl


def _close_in_channel(got, ref, rel=6e-5, floor=1e-3):
    """Printed-precision agreement per channel column, with an absolute floor at `floor` times
    the column's largest value (deep under the barrier the printed values are ~1e-26)."""
    scale = np.abs(ref).max(axis=0, keepdims=True)
    return np.abs(got - ref) <= rel * (np.abs(ref) + floor * scale)


@pytest.mark.parametrize("name", sorted(GOLD["wavefunctions"]))
def test_wave_functions_internal_and_external(name):
    """Internal wave functions at the mesh points (C^-1 of the surface amplitudes) and the
    external Coulomb/Whittaker forms at r = zrma(nr ns) + 0.2 i, as the drivers print them
    (rmat_pierre/Ex*/example*.f, wave_functions.txt)."""
    mesh, rmax, cpot, kin, nv, blocks, cpnl = wf_case(name)
    for b in blocks:
        lval, qk, eta = kin(b["E"])
        cu, no, cf = orc.rmatrix_wf(nv, lval, qk, eta, rmax, mesh, cpot, [1], cpnl=cpnl)
        ref = np.array(b["internal"])
        np.testing.assert_allclose(ref[:, 0], mesh.zrma, atol=6e-4)
        refc = ref[:, 1::2] + 1j * ref[:, 2::2]
        assert _close_in_channel(cf[:, :, 0], refc).all(), (name, b["E"])
        ext = []
        for row in b["external"]:
            r = mesh.zrma[-1] + 0.2 * round((row[0] - mesh.zrma[-1]) / 0.2)
            nop, nclo, vals = 0, no, []
            for iv in range(nv):
                l = int(lval[iv])
                if qk[iv] > 0:
                    fc, gc, _, _, _ = coulfg(qk[iv] * r, eta[iv], float(l))
                    nop += 1
                    co = complex(gc, fc) * math.sqrt(qk[0] / qk[iv])
                    vals.append(-cu[nop - 1, 0] * co + (np.conj(co) if iv == 0 else 0))
                else:
                    nclo += 1
                    f, _, _ = whit(eta[iv], r, -qk[iv], -qk[iv] ** 2, l, 0)
                    vals.append(cu[nclo - 1, 0] * f[l])
            ext.append(vals)
        ref = np.array(b["external"])
        assert _close_in_channel(np.array(ext), ref[:, 1::2] + 1j * ref[:, 2::2]).all(), (name, b["E"])


def test_ex3_wf_print_fixed_step():
    """wf_print on r = 2, 4, ..., 20 fm (Ex3, rmax = 14): the spline inside, Coulomb outside.
    Descouvemont's wf_print passes an unset yp2 as the spline's last-point condition
    (rmat_pierre/rmatrix.f:339,350); it evaluated to 0 there, which only the point r = rmax,
    beyond the last mesh point, sees.  HPRMAT sets yp2 = 1e30 (natural, src/rmatrix_hp.F90:693-694)."""
    c = GOLD["examples"]["ex3"][3]
    nr, ns, rmax = c["nr"], c["ns"], abs(c["rmax"])
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin, nv = ex3_setup(mesh.zrma, c["j"])
    for b in GOLD["fixed_step"]["ex3"]:
        lval, qk, eta = kin(b["E"])
        cu, no, cf = orc.rmatrix_wf(nv, lval, qk, eta, rmax, mesh, cpot, [1])
        for iv, rows in enumerate(b["channels"]):
            ref = np.array(rows)
            np.testing.assert_allclose(ref[:, 0], c["h"] * np.arange(1, c["npoin"] + 1))
            out = orc.wf_print(nv, lval, qk, eta, rmax, mesh, cu, no, cf, iv + 1, 1, c["npoin"], c["h"], ypn=0.0)
            refc = ref[:, 1] + 1j * ref[:, 2]
            assert _close_in_channel(out[:, None], refc[:, None]).all(), (b["E"], iv)
            natural = orc.wf_print(nv, lval, qk, eta, rmax, mesh, cu, no, cf, iv + 1, 1, c["npoin"], c["h"])
            inside = ref[:, 0] < mesh.zrma[-1]
            np.testing.assert_allclose(natural[inside], out[inside], rtol=0, atol=1e-3 * np.abs(out).max())


def test_mixed_type2_matches_dense_on_small_problem():
    """The oracle's Type 2 restatement (CGETRF + refinement) agrees with Type 1 on Ex2."""
    c = GOLD["examples"]["ex2"][0]
    mesh = orc.rmat_ini(c["nr"], 1, abs(c["rmax"]))
    cpot, kin = ex2_setup(mesh.zrma, c["j"])
    lval, qk, eta = kin(24.0)
    u1 = orc.rmatrix(2, lval, qk, eta, abs(c["rmax"]), mesh, cpot).cu
    u2 = orc.rmatrix(2, lval, qk, eta, abs(c["rmax"]), mesh, cpot, solver="mixed").cu
    assert np.linalg.norm(u1 - u2) / np.linalg.norm(u1) < 1e-9


def test_legzo_matches_numpy_gauss_legendre():
    for n in (2, 7, 50, 200):
        x, w = orc.legzo(n)
        xr, wr = np.polynomial.legendre.leggauss(n)
        assert np.allclose(x, (np.sort(xr) + 1) / 2, rtol=0, atol=1e-14)
        assert np.allclose(w, wr[np.argsort(xr)] / 2, rtol=1e-9, atol=0)


def test_oracle_condition_estimate_against_exact():
    """The oracle's Hager-Higham estimate (the checker of opts.estimate_condition) is a lower
    bound of numpy's exact 1-norm condition number, within a factor 3, on exact-kappa
    Householder matrices and the small workload's C(E)."""
    from hprmat_b200 import workloads
    n = 300
    rng = np.random.default_rng(3)
    v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    v /= np.linalg.norm(v)
    H = np.eye(n) - 2 * np.outer(v, v.conj())
    cases = []
    for kappa in (1e3, 1e8):
        d = kappa ** (-np.arange(n) / (n - 1))
        cases.append((H * d[None, :]) @ H)
    w = workloads.small()
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    bnd = orc.boundary_values(w.nch, w.lval, w.qk, w.eta, w.rmax)
    cases.append(orc.assemble(mesh, 1, w.nch, w.lval, w.qk, bnd.xc, w.cpot))
    for A in cases:
        exact = float(np.linalg.cond(A, 1))
        est = orc.cond1_estimate(A)
        assert exact / 3.0 <= est <= exact * (1 + 1e-6), (est, exact)
