"""Non-local potentials on the device (rmatrix with ncp2 > 0, src/rmatrix_hp.F90:283-288).

The assembly adds sqrt(w_i w_j) a cpnl(i nr + j, c, c') to every channel block; the FP64
refinement then multiplies by a dense copy of C(E).  Checked against the oracle to 1e-10 and
against the golden phase shifts of Yamaguchi's potential (rmat_pierre/Ex5/output5.txt) at both
precisions, and on a coupled-channel problem with non-local couplings.
"""
import math

import numpy as np
import pytest

from hprmat_b200 import api, workloads
from oracle import rmatrix_oracle as orc
from tests.example_inputs import ex5_setup
from tests.test_oracle_golden import GOLD, _printed_close

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(precision="mixed")
    yield c
    c.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("card", range(len(GOLD["examples"]["ex5"])))
def test_ex5_yamaguchi(ctx, precision, card):
    c = GOLD["examples"]["ex5"][card]
    nr, rmax = c["nr"], abs(c["rmax"])
    ctx.set_precision(precision)
    mesh = orc.rmat_ini(nr, 1, rmax)
    cpot, cpnl, kin = ex5_setup(mesh.zrma)
    for row in c["printed"]["phase shift (deg.)="]:
        lval, qk, eta = kin(row["E"])
        cu, nopen = ctx.rmatrix(1, lval, qk, eta, rmax, nr, 1, cpot, cpnl=cpnl)
        ref = orc.rmatrix(1, lval, qk, eta, rmax, mesh, cpot, cpnl=cpnl).cu[0, 0]
        u = cu[0, 0]
        assert abs(u - ref) <= TOL * abs(ref), (row["E"], u, ref, ctx.last_stats)
        delta = math.atan2(u.imag, u.real) / 2 * 180 / math.pi
        assert _printed_close(delta, row["values"][0]), (row["E"], delta, row["values"])


def _nonlocal_couplings(nch, nr, zrma, seed=5):
    """Separable Gaussian non-local couplings with complex strengths, symmetric in (c, c')."""
    rng = np.random.default_rng(seed)
    s = rng.uniform(-2.0, 2.0, (nch, nch)) + 1j * rng.uniform(-0.3, 0.0, (nch, nch))
    s = np.triu(s) + np.triu(s, 1).T
    r = np.asarray(zrma)
    g = np.exp(-((r[:, None] - 1.5) ** 2 + (r[None, :] - 1.5) ** 2) / 2.0)
    cpnl = np.zeros((nr * nr, nch, nch), dtype=np.complex128, order="F")
    for a in range(nch):
        for b in range(nch):
            cpnl[:, a, b] = (s[a, b] * g).reshape(-1)
    return cpnl


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_coupled_channels_with_nonlocal_couplings(ctx, precision):
    """12 channels x 60 points (N = 720), open and closed channels, Coulomb, local and
    non-local couplings; U and the wave functions of two entrance channels."""
    nr, rmax, nch = 60, 12.0, 12
    w = workloads.production(nch=nch, nr=nr, rmax=rmax)
    mesh = orc.rmat_ini(nr, 1, rmax)
    cpnl = _nonlocal_couplings(nch, nr, mesh.zrma)
    ctx.set_precision(precision)
    cu, nopen = ctx.rmatrix(nch, w.lval, w.qk, w.eta, rmax, nr, 1, w.cpot, cpnl=cpnl)
    ref = orc.rmatrix(nch, w.lval, w.qk, w.eta, rmax, mesh, w.cpot, cpnl=cpnl)
    assert nopen == ref.nopen and 0 < nopen < nch
    assert _rel(cu[:nopen, :nopen], ref.cu) <= TOL, ctx.last_stats
    # the non-local term matters
    assert _rel(orc.rmatrix(nch, w.lval, w.qk, w.eta, rmax, mesh, w.cpot).cu, ref.cu) > 1e-3
    cu2, nopen2, cf = ctx.rmatrix_wf(nch, w.lval, w.qk, w.eta, rmax, nr, 1, w.cpot, [1, 2], cpnl=cpnl)
    _, _, cf_ref = orc.rmatrix_wf(nch, w.lval, w.qk, w.eta, rmax, mesh, w.cpot, [1, 2], u=cu2, cpnl=cpnl)
    assert _rel(cf, cf_ref) <= TOL


def test_nonlocal_requires_one_interval(ctx):
    mesh = orc.rmat_ini(10, 2, 8.0)
    cpot, cpnl, kin = ex5_setup(mesh.zrma[:10])
    cpot = np.zeros((20, 1, 1), dtype=np.complex128, order="F")
    lval, qk, eta = kin(1.0)
    with pytest.raises(api.HprmatError):
        ctx.rmatrix(1, lval, qk, eta, 8.0, 10, 2, cpot, cpnl=cpnl)
