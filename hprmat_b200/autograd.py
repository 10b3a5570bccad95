"""Differentiable collision matrix for PyTorch.

``collision_matrix(cpot, ...)`` returns U (nopen x nopen, complex128) from the potential at
the Lagrange mesh points, cpot[i, c, c'] = V_cc'(r_i) / (hbar^2/2mu), as a
``torch.autograd.Function``: the forward is the refined device solve; the backward is the
adjoint -- from the forward's kept solution for a symmetric potential, else a solve with C^T on
FP64 LU factors (``hprmat_b200_rmatrix_adjoint``).  Gradients with
respect to potential parameters follow from building ``cpot`` with differentiable torch
operations (``potential_matrix`` mirrors the synthetic potentials of
``hprmat_b200.workloads``).  The reference has no derivatives; this is the adjoint row of the
hot path.
"""
from __future__ import annotations

import numpy as np
import torch

from . import workloads

__all__ = ["CollisionMatrix", "collision_matrix", "potential_matrix"]


class CollisionMatrix(torch.autograd.Function):
    """Forward: the refined device solve.  For a symmetric potential (C(E) complex symmetric)
    the forward keeps its solution X = C^-1 Q on the device and the backward forms the gradient
    from it without another solve (``Context.rmatrix_x`` / ``adjoint_from_x``); otherwise the
    backward runs ``rmatrix_adjoint`` (FP64 forward and a solve with C^T)."""

    @staticmethod
    def forward(fctx, cpot, solver, lval, qk, eta, rmax, nr):
        c_np = np.asfortranarray(cpot.detach().cpu().numpy().astype(np.complex128))
        nch = c_np.shape[1]
        symmetric = bool(np.array_equal(c_np[:nr], c_np[:nr].transpose(0, 2, 1)))
        x = None
        if symmetric:
            cu, nopen, x = solver.rmatrix_x(nch, lval, qk, eta, rmax, nr, c_np)
        else:
            cu, nopen = solver.rmatrix(nch, lval, qk, eta, rmax, nr, 1, c_np)
        fctx.save_for_backward(cpot.detach())
        fctx.args = (solver, lval, qk, eta, rmax, nr, nopen, x, cu)
        return torch.from_numpy(np.ascontiguousarray(cu[:nopen, :nopen])).to(cpot.device)

    @staticmethod
    def backward(fctx, grad_u):
        (cpot,) = fctx.saved_tensors
        solver, lval, qk, eta, rmax, nr, nopen, x, cu = fctx.args
        c_np = np.asfortranarray(cpot.cpu().numpy().astype(np.complex128))
        nch = c_np.shape[1]
        gu = grad_u.detach().cpu().numpy()
        if x is not None:
            grad = solver.adjoint_from_x(nch, lval, qk, eta, rmax, nr, c_np, cu, x, gu)
        else:
            _, _, grad = solver.rmatrix_adjoint(nch, lval, qk, eta, rmax, nr, c_np, gu)
        return torch.from_numpy(np.ascontiguousarray(grad)).to(cpot.device), None, None, None, None, None, None


def collision_matrix(cpot: torch.Tensor, solver, lval, qk, eta, rmax: float, nr: int) -> torch.Tensor:
    """U (nopen x nopen) from cpot (nr, nch, nch) complex128; differentiable in cpot."""
    return CollisionMatrix.apply(cpot, solver, lval, qk, eta, rmax, nr)


def potential_matrix(r: torch.Tensor, coupling: torch.Tensor, params: torch.Tensor, hm: float,
                     z1z2: float) -> torch.Tensor:
    """cpot(r_i, c, c') / hm for the Woods-Saxon + Coulomb diagonal and Gaussian couplings of
    ``workloads.potential_matrix``, differentiable in params = (V0, W0, R, a, coupling scale,
    Coulomb radius)."""
    v0, w0, rws, aws, cscale, rc = params.unbind(0)
    ws = torch.complex(v0, w0) / (1.0 + torch.exp((r - rws) / aws))
    if z1z2 != 0.0:
        ze = z1z2 * workloads.E2
        vc = torch.where(r <= rc, ze * (3.0 - (r / rc) ** 2) / (2.0 * rc), ze / r)
    else:
        vc = torch.zeros_like(r)
    g = torch.exp(-(r / 2.0) ** 2)
    nch = coupling.shape[0]
    cp = (cscale * coupling)[None, :, :] * g[:, None, None]
    eye = torch.eye(nch, dtype=torch.bool)
    cp = torch.where(eye[None, :, :], (ws + vc).to(cp.dtype)[:, None, None], cp)
    return cp / hm
