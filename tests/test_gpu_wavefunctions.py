"""Wave functions on the device (rmatrix with twf) against the oracle and the golden files.

The device builds the internal wave functions from the per-interval solutions of the R-matrix
step (C^-1 of the propagated surface amplitudes).  Every example card that writes wave
functions (rmat_pierre/Ex{1,2,3,4,5}/wf*.txt, ns = 1 to 5, Ex4 with closed channels, Ex5 with
Yamaguchi's non-local potential) is checked
at both precisions: U against the oracle to 1e-10; cf and the closed-channel amplitudes
against the oracle's reconstruction from the device's U to 1e-10 (relative, per entrance
channel) -- where |U| ~ 1 under a barrier (Ex1: |cop| ~ 1e7) the small components of the
wave function follow the last bits of U, which no two FP64 solvers share; cf against the
printed values; and wf_print on the device result against Ex3's printed fixed-step values.
"""
import json
import os

import numpy as np
import pytest

from hprmat_b200 import api, workloads
from oracle import rmatrix_oracle as orc
from tests.test_oracle_golden import GOLD, _close_in_channel, wf_case

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
@pytest.mark.parametrize("name", sorted(GOLD["wavefunctions"]))
def test_wave_functions_against_oracle_and_golden(ctx, precision, name):
    mesh, rmax, cpot, kin, nv, blocks, cpnl = wf_case(name)
    ctx.set_precision(precision)
    for b in blocks:
        lval, qk, eta = kin(b["E"])
        cu, nopen, cf = ctx.rmatrix_wf(nv, lval, qk, eta, rmax, mesh.nr, mesh.ns, cpot, [1], cpnl=cpnl)
        u_ref = orc.rmatrix(nv, lval, qk, eta, rmax, mesh, cpot, cpnl=cpnl).cu
        assert _rel(cu[:nopen, :nopen], u_ref) <= TOL, (name, b["E"], ctx.last_stats)
        cu_ref, no_ref, cf_ref = orc.rmatrix_wf(nv, lval, qk, eta, rmax, mesh, cpot, [1], u=cu, cpnl=cpnl)
        assert nopen == no_ref
        assert _rel(cf[:, :, 0], cf_ref[:, :, 0]) <= TOL, (name, b["E"], ctx.last_stats)
        assert _rel(cu[:nv, 0], cu_ref[:, 0]) <= TOL, (name, b["E"])
        ref = np.array(b["internal"])
        assert _close_in_channel(cf[:, :, 0], ref[:, 1::2] + 1j * ref[:, 2::2]).all(), (name, b["E"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_several_entrance_channels_three_intervals(ctx, precision):
    """20 channels x 60 points per interval, three intervals, open and closed channels: wave
    functions for three entrance channels and the closed-channel amplitudes."""
    nr, ns, rmax, nch = 60, 3, 18.0, 20
    mesh = orc.rmat_ini(nr, ns, rmax)
    w = workloads.with_intervals(workloads.production(nch=nch, nr=nr, rmax=rmax), ns)
    ctx.set_precision(precision)
    nvc = [1, 2, 4]
    cu, nopen, cf = ctx.rmatrix_wf(nch, w.lval, w.qk, w.eta, rmax, nr, ns, w.cpot, nvc)
    u_ref = orc.rmatrix(nch, w.lval, w.qk, w.eta, rmax, mesh, w.cpot).cu
    assert _rel(cu[:nopen, :nopen], u_ref) <= TOL
    cu_ref, no_ref, cf_ref = orc.rmatrix_wf(nch, w.lval, w.qk, w.eta, rmax, mesh, w.cpot, nvc, u=cu)
    assert nopen == no_ref and 0 < nopen < nch
    for ic in range(len(nvc)):
        assert _rel(cf[:, :, ic], cf_ref[:, :, ic]) <= TOL, (ic, ctx.last_stats)
    assert _rel(cu[:nch, :len(nvc)], cu_ref[:, :len(nvc)]) <= TOL
    assert np.abs(cu[nopen:, :len(nvc)]).max() > 0  # closed-channel amplitudes written


def test_single_interval_wave_function(ctx):
    """ns = 1 (the production mode): the wave function from the one solve."""
    w = workloads.production(nch=12, nr=80, rmax=16.0)
    mesh = orc.rmat_ini(80, 1, 16.0)
    ctx.set_precision("mixed")
    cu, nopen, cf = ctx.rmatrix_wf(12, w.lval, w.qk, w.eta, 16.0, 80, 1, w.cpot, [1, 2])
    cu_ref, no_ref, cf_ref = orc.rmatrix_wf(12, w.lval, w.qk, w.eta, 16.0, mesh, w.cpot, [1, 2], u=cu)
    assert _rel(cf, cf_ref) <= TOL
    u_only, _ = ctx.rmatrix(12, w.lval, w.qk, w.eta, 16.0, 80, 1, w.cpot)
    assert _rel(cu[:nopen, :nopen], u_only[:nopen, :nopen]) <= TOL


def test_ex3_wf_print_on_device_result(ctx):
    """wf_print of the device wave function reproduces Ex3's printed fixed-step values at every
    point except r = rmax: there Descouvemont's spline end condition (an unset yp2) differs from
    HPRMAT's natural one, and the device result is compared with the oracle's natural spline."""
    c = GOLD["examples"]["ex3"][3]
    nr, ns, rmax = c["nr"], c["ns"], abs(c["rmax"])
    mesh, _, cpot, kin, nv, _, _ = wf_case("ex3")
    ctx.set_precision("mixed")
    for b in GOLD["fixed_step"]["ex3"]:
        lval, qk, eta = kin(b["E"])
        cu, nopen, cf = ctx.rmatrix_wf(nv, lval, qk, eta, rmax, nr, ns, cpot, [1])
        cu_ref, no_ref, cf_ref = orc.rmatrix_wf(nv, lval, qk, eta, rmax, mesh, cpot, [1], u=cu)
        got_all, ref_all = [], []
        for iv, rows in enumerate(b["channels"]):
            got = api.wf_print(lval, qk, eta, rmax, nr, ns, cu, nopen, cf, mesh.zrma, iv + 1, 1, c["npoin"], c["h"])
            ref = np.array(rows)
            r = ref[:, 0]
            keep = np.abs(r - rmax) > 1e-9
            refc = ref[:, 1] + 1j * ref[:, 2]
            assert _close_in_channel(got[keep, None], refc[keep, None]).all(), (b["E"], iv)
            got_all.append(got)
            ref_all.append(orc.wf_print(nv, lval, qk, eta, rmax, mesh, cu_ref, no_ref, cf_ref, iv + 1, 1, c["npoin"],
                                        c["h"]))
        # the same measure as cf: relative over all channels of the entrance channel
        assert _rel(np.array(got_all), np.array(ref_all)) <= TOL


def test_bad_entrance_channel(ctx):
    mesh, rmax, cpot, kin, nv, blocks, _ = wf_case("ex4")
    lval, qk, eta = kin(blocks[0]["E"])
    nopen = int((qk > 0).sum())
    with pytest.raises(api.HprmatError):
        ctx.rmatrix_wf(nv, lval, qk, eta, rmax, mesh.nr, mesh.ns, cpot, [nopen + 1])
