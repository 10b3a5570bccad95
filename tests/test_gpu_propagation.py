"""Multi-interval R-matrix propagation (ns > 1) on the device against the oracle.

Every mesh card of the reference's golden examples (rmat_pierre/Ex{1,2,4}/output*.txt via
tests/golden/reference_examples.json: ns = 1 to 5, Ex4 with closed channels) goes through the
C ABI at both precisions: U agrees with the oracle's FP64 propagation to 1e-10 relative
(Frobenius) and reproduces the printed values.  A production-generator problem with three
intervals checks the propagated path at N = 1200 per interval.
"""
import json
import math
import os

import numpy as np
import pytest

from hprmat_b200 import api, workloads
from oracle import rmatrix_oracle as orc
from tests.example_inputs import ex1_setup, ex2_setup, ex4_setup

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_examples.json")))
U_TOL = 1e-10


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _printed_close(x, ref, rel=6e-5, abs_=1e-12):
    return abs(x - ref) <= rel * abs(ref) + abs_


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(precision="mixed")
    yield c
    c.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex1"])))
def test_ex1_cards(ctx, precision, card):
    c = GOLD["examples"]["ex1"][card]
    nr, ns, rmax = c["nr"], c["ns"], abs(c["rmax"])
    ctx.set_precision(precision)
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin = ex1_setup(mesh.zrma)
    for row in c["printed"]["Collision matrix="]:
        lval, qk, eta = kin(row["E"], c["j"])
        cu, nopen = ctx.rmatrix(1, lval, qk, eta, rmax, nr, ns, cpot)
        ref = orc.rmatrix(1, lval, qk, eta, rmax, mesh, cpot).cu[0, 0]
        u = cu[0, 0]
        assert abs(u - ref) <= U_TOL * abs(ref), (row["E"], u, ref, ctx.last_stats)
        assert _printed_close(u.real, row["values"][0]), (row["E"], u, row["values"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex2"])))
def test_ex2_cards(ctx, precision, card):
    c = GOLD["examples"]["ex2"][card]
    nr, ns, rmax, j = c["nr"], c["ns"], abs(c["rmax"]), c["j"]
    ctx.set_precision(precision)
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin = ex2_setup(mesh.zrma, j)
    for row in c["printed"]["phase shift (rad.)="]:
        lval, qk, eta = kin(row["E"])
        cu, nopen = ctx.rmatrix(2, lval, qk, eta, rmax, nr, ns, cpot)
        ref = orc.rmatrix(2, lval, qk, eta, rmax, mesh, cpot).cu
        assert _rel(cu[:2, :2], ref) <= U_TOL, (row["E"], ctx.last_stats)
        d1 = math.atan2(cu[0, 0].imag, cu[0, 0].real) / 2
        d2 = math.atan2(cu[1, 1].imag, cu[1, 1].real) / 2
        for x, r in zip([d1, d2, abs(cu[0, 1])], row["values"]):
            assert _printed_close(x, r), (row["E"], x, r)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex4"])))
def test_ex4_cards_closed_channels(ctx, precision, card):
    c = GOLD["examples"]["ex4"][card]
    nr, ns, rmax, j = c["nr"], c["ns"], abs(c["rmax"]), c["j"]
    ctx.set_precision(precision)
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin, nv = ex4_setup(mesh.zrma, j)
    for ra in c["printed"]["Amplitude="]:
        lval, qk, eta = kin(ra["E"])
        cu, nopen = ctx.rmatrix(nv, lval, qk, eta, rmax, nr, ns, cpot)
        ref = orc.rmatrix(nv, lval, qk, eta, rmax, mesh, cpot)
        assert nopen == ref.nopen
        assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL, (ra["E"], ctx.last_stats)
        for x, r in zip(np.abs(cu[:nopen, 0]), ra["values"]):
            assert _printed_close(x, r, rel=1.2e-4), (ra["E"], x, r)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_production_generator_three_intervals(ctx, precision):
    """20 channels x 60 points per interval, three intervals on [0, 18 fm]: open and closed
    channels, Coulomb, complex couplings; the propagated U against the oracle."""
    nr, ns, rmax, nch = 60, 3, 18.0, 20
    mesh = orc.rmat_ini(nr, ns, rmax)
    w = workloads.with_intervals(workloads.production(nch=nch, nr=nr, rmax=rmax), ns)
    np.testing.assert_allclose(np.sort(mesh.zrma), mesh.zrma)
    ctx.set_precision(precision)
    cu, nopen = ctx.rmatrix(nch, w.lval, w.qk, w.eta, rmax, nr, ns, w.cpot)
    ref = orc.rmatrix(nch, w.lval, w.qk, w.eta, rmax, mesh, w.cpot)
    assert nopen == ref.nopen and 0 < nopen < nch
    assert _rel(cu[:nopen, :nopen], ref.cu) <= U_TOL, ctx.last_stats
    st = ctx.last_stats
    assert st["nrhs"] == 2 * nch
