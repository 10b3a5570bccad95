"""The FP64 reference adjoint (oracle) against central finite differences of the oracle's
own collision matrix, and the differentiable torch potential against the NumPy generator.
CPU only: these pin the adjoint formulas that the device adjoint is checked against."""
import numpy as np
import torch

from hprmat_b200 import workloads
from hprmat_b200.autograd import potential_matrix
from oracle import rmatrix_oracle as orc


def _loss(w, mesh, cpot, target):
    res = orc.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, cpot)
    return float(np.sum(np.abs(res.cu - target) ** 2)), res.cu


def test_oracle_adjoint_matches_central_differences():
    w = workloads.small()
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    rng = np.random.default_rng(7)
    target = orc.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot * 1.01).cu
    L0, u = _loss(w, mesh, w.cpot, target)
    u2, grad = orc.rmatrix_adjoint(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot, 2 * (u - target))
    assert np.allclose(u2, u)
    h = 1e-6
    for _ in range(4):  # random complex directions over all mesh points and channel pairs
        d = rng.standard_normal(w.cpot.shape) + 1j * rng.standard_normal(w.cpot.shape)
        lp, _ = _loss(w, mesh, w.cpot + h * d, target)
        lm, _ = _loss(w, mesh, w.cpot - h * d, target)
        fd = (lp - lm) / (2 * h)
        ad = float(np.real(np.sum(np.conj(grad) * d)))
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-300), (fd, ad)


def test_torch_potential_matches_numpy_generator():
    w = workloads.production(nch=6, nr=30)
    r = torch.from_numpy(workloads.lagrange_radii(w.nr, w.rmax))
    p = torch.tensor(w.params.as_array(), dtype=torch.float64)
    cp = potential_matrix(r, torch.from_numpy(w.coupling), p, w.hm, w.params.z1z2)
    assert np.allclose(cp.numpy(), w.cpot, rtol=1e-14, atol=1e-14)
