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
