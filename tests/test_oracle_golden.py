"""The oracle against the reference's golden outputs (CPU).

tests/golden/reference_examples.json holds the printed results of Descouvemont's
examples (rmat_pierre/Ex{1,2,4}/output*.txt), extracted by tests/golden/make_golden.py.
The oracle must reproduce them to the printed 5 significant digits for every mesh card,
including the multi-interval (ns > 1) ones and Ex4's closed channels (WHIT path).
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import rmatrix_oracle as orc
from tests.example_inputs import ex1_setup, ex2_setup, ex4_setup

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
