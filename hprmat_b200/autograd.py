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

__all__ = ["CollisionMatrix", "CollisionMatrices", "collision_matrix", "collision_matrices", "potential_matrix"]


def _symmetric(cpot: torch.Tensor, nr: int) -> bool:
    """cpot(i, c, c') == cpot(i, c', c) at the mesh points (compared where cpot lives)."""
    return bool(torch.equal(cpot[:nr], cpot[:nr].transpose(1, 2)))


def _device_path(cpot: torch.Tensor, solver) -> bool:
    """A CUDA potential on the solver's device: the solve and the gradient stay on the device."""
    return cpot.is_cuda and cpot.device.index == solver.device


class CollisionMatrix(torch.autograd.Function):
    """Forward: the refined device solve.  For a symmetric potential (C(E) complex symmetric)
    the forward keeps its solution X = C^-1 Q on the device and the backward forms the gradient
    from it without another solve (``Context.rmatrix_x`` / ``adjoint_from_x``); a potential that
    is a CUDA tensor on the solver's device is handed to the library by its device address
    (``rmatrix_x_device`` / ``adjoint_from_x_device``: only O(nch^2) values cross to the host).
    Otherwise the backward runs ``rmatrix_adjoint`` (FP64 forward and a solve with C^T)."""

    @staticmethod
    def forward(fctx, cpot, solver, lval, qk, eta, rmax, nr):
        cpot = cpot.detach().to(torch.complex128)
        symmetric = _symmetric(cpot, nr)
        nch = cpot.shape[1]
        x = None
        on_dev = symmetric and _device_path(cpot, solver)
        if on_dev:
            cu, nopen, x = solver.rmatrix_x_device(nch, lval, qk, eta, rmax, nr, cpot)
            u = cu[:nopen, :nopen].contiguous()
        else:
            c_np = np.asfortranarray(cpot.cpu().numpy())
            if symmetric:
                cu, nopen, x = solver.rmatrix_x(nch, lval, qk, eta, rmax, nr, c_np)
            else:
                cu, nopen = solver.rmatrix(nch, lval, qk, eta, rmax, nr, 1, c_np)
            u = torch.from_numpy(np.ascontiguousarray(cu[:nopen, :nopen])).to(cpot.device)
        fctx.save_for_backward(cpot)
        fctx.args = (solver, lval, qk, eta, rmax, nr, nopen, x, cu, on_dev)
        return u

    @staticmethod
    def backward(fctx, grad_u):
        (cpot,) = fctx.saved_tensors
        solver, lval, qk, eta, rmax, nr, nopen, x, cu, on_dev = fctx.args
        nch = cpot.shape[1]
        if on_dev:
            grad = solver.adjoint_from_x_device(nch, lval, qk, eta, rmax, nr, cpot, cu, x, grad_u)
            return grad, None, None, None, None, None, None
        c_np = np.asfortranarray(cpot.cpu().numpy())
        gu = grad_u.detach().cpu().numpy()
        if x is not None:
            grad = solver.adjoint_from_x(nch, lval, qk, eta, rmax, nr, c_np, cu, x, gu)
        else:
            _, _, grad = solver.rmatrix_adjoint(nch, lval, qk, eta, rmax, nr, c_np, gu)
        return torch.from_numpy(np.ascontiguousarray(grad)).to(cpot.device), None, None, None, None, None, None


def collision_matrix(cpot: torch.Tensor, solver, lval, qk, eta, rmax: float, nr: int) -> torch.Tensor:
    """U (nopen x nopen) from cpot (nr, nch, nch) complex128; differentiable in cpot."""
    return CollisionMatrix.apply(cpot, solver, lval, qk, eta, rmax, nr)


def _round_robin(pool, n, fn):
    """fn(context, i) for i < n, energy i on context i % len(pool); each context's energies in
    order on one host thread (a context is used by one thread at a time), results in order."""
    from concurrent.futures import ThreadPoolExecutor
    out = [None] * n

    def run(w):
        for i in range(w, n, len(pool)):
            out[i] = fn(pool[w], i)

    nw = min(len(pool), n)
    if nw <= 1:
        run(0) if n else None
        return out
    with ThreadPoolExecutor(nw) as ex:
        for f in [ex.submit(run, w) for w in range(nw)]:
            f.result()
    return out


class CollisionMatrices(torch.autograd.Function):
    """U at several energies of one channel block, differentiable in the potential.  The
    forward solves run concurrently on a pool of contexts (one host thread and one CUDA stream
    each), so that the small solves of different energies overlap on the GPU.  Symmetric
    potential: each forward keeps its solution X on the device and the backward forms the
    energy's gradient from it (no second solve); otherwise the backward runs
    ``rmatrix_adjoint`` per energy.  The gradient is the sum over the energies."""

    @staticmethod
    def forward(fctx, cpot, pool, lval, kin, rmax, nr):
        cpot = cpot.detach().to(torch.complex128)
        nch = cpot.shape[1]
        symmetric = _symmetric(cpot, nr)
        on_dev = symmetric and all(_device_path(cpot, ctx) for ctx in pool)
        c_np = None if on_dev else np.asfortranarray(cpot.cpu().numpy())

        def fwd(ctx, i):
            qk, eta = kin[i]
            if on_dev:
                return ctx.rmatrix_x_device(nch, lval, qk, eta, rmax, nr, cpot)
            if symmetric:
                return ctx.rmatrix_x(nch, lval, qk, eta, rmax, nr, c_np)
            cu, nopen = ctx.rmatrix(nch, lval, qk, eta, rmax, nr, 1, c_np)
            return cu, nopen, None

        res = _round_robin(pool, len(kin), fwd)
        fctx.save_for_backward(cpot)
        fctx.args = (pool, lval, kin, rmax, nr, res, symmetric, on_dev)
        if on_dev:
            return tuple(cu[:no, :no].contiguous() for cu, no, _ in res)
        return tuple(torch.from_numpy(np.ascontiguousarray(cu[:no, :no])).to(cpot.device) for cu, no, _ in res)

    @staticmethod
    def backward(fctx, *grads):
        (cpot,) = fctx.saved_tensors
        pool, lval, kin, rmax, nr, res, symmetric, on_dev = fctx.args
        nch = cpot.shape[1]
        c_np = None if on_dev else np.asfortranarray(cpot.cpu().numpy())

        def bwd(ctx, i):
            qk, eta = kin[i]
            cu, _, x = res[i]
            if on_dev:
                return ctx.adjoint_from_x_device(nch, lval, qk, eta, rmax, nr, cpot, cu, x, grads[i])
            gu = grads[i].detach().cpu().numpy()
            if symmetric:
                return ctx.adjoint_from_x(nch, lval, qk, eta, rmax, nr, c_np, cu, x, gu)
            return ctx.rmatrix_adjoint(nch, lval, qk, eta, rmax, nr, c_np, gu)[2]

        parts = _round_robin(pool, len(kin), bwd)
        if on_dev:
            return torch.stack(parts).sum(0), None, None, None, None, None
        total = np.zeros_like(c_np)
        for g in parts:
            total += g
        return torch.from_numpy(np.ascontiguousarray(total)).to(cpot.device), None, None, None, None, None


def collision_matrices(cpot: torch.Tensor, pool, lval, kin, rmax: float, nr: int):
    """U (nopen_E x nopen_E) for every (qk, eta) in ``kin``, from cpot (nr, nch, nch); ``pool``:
    a list of ``api.Context`` (the forward solves of different energies run concurrently, one
    per context).  Differentiable in cpot."""
    return CollisionMatrices.apply(cpot, list(pool), lval, list(kin), rmax, nr)


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
    eye = torch.eye(nch, dtype=torch.bool, device=coupling.device)
    cp = torch.where(eye[None, :, :], (ws + vc).to(cp.dtype)[:, None, None], cp)
    return cp / hm
