"""Device adjoint (hprmat_b200_rmatrix_adjoint) and the torch autograd wrapper.

* The gradient with respect to the potential at every mesh point agrees with the FP64 oracle
  adjoint (dense LAPACK solve with C^T) to 1e-8 relative (Frobenius).
* Gradients of sum |U - U_target|^2 over several energies with respect to the six potential
  parameters, through torch.autograd, agree with central finite differences (step 1e-6) of the
  device forward to 1e-6 relative.
"""
import numpy as np
import pytest
import torch

from hprmat_b200 import api, workloads
from hprmat_b200.autograd import collision_matrix, potential_matrix
from oracle import rmatrix_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["small", "production20"])
def test_adjoint_matches_oracle_gradient(name):
    w = workloads.small() if name == "small" else workloads.production(nch=20, nr=60, rmax=15.0)
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    target = orc.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot * 1.02).cu
    u_ref, _ = orc.rmatrix_adjoint(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot, np.zeros_like(target))
    gu = 2 * (u_ref - target)
    _, g_ref = orc.rmatrix_adjoint(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot, gu)
    ctx = api.Context(precision="mixed")
    cu, nopen, g = ctx.rmatrix_adjoint(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, w.cpot, gu)
    assert nopen == u_ref.shape[0]
    assert np.linalg.norm(cu[:nopen, :nopen] - u_ref) <= 1e-10 * np.linalg.norm(u_ref)
    err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert err <= 1e-8, err
    ctx.close()


def test_adjoint_nonsymmetric_potential_uses_transposed_solve():
    """A potential with cpot(c, c') != cpot(c', c): C(E) is not symmetric, the device solves with
    C^T on its FP64 factors; the gradient agrees with the oracle's dense C^T solve."""
    w = workloads.production(nch=10, nr=50, rmax=14.0)
    cpot = np.array(w.cpot, order="F")
    rng = np.random.default_rng(11)
    tri = np.triu(rng.uniform(-0.05, 0.05, (w.nch, w.nch)), 1)
    cpot += (tri * np.exp(-(workloads.lagrange_radii(w.nr, w.rmax) / 3.0) ** 2)[:, None, None]) / w.hm
    assert not np.allclose(cpot, cpot.transpose(0, 2, 1))
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    u_ref = orc.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, cpot).cu
    gu = np.conj(u_ref) * 0.3 + 0.1
    _, g_ref = orc.rmatrix_adjoint(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, cpot, gu)
    ctx = api.Context(precision="mixed")
    cu, nopen, g = ctx.rmatrix_adjoint(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, cpot, gu)
    assert np.linalg.norm(cu[:nopen, :nopen] - u_ref) <= 1e-10 * np.linalg.norm(u_ref)
    assert ctx.last_stats["factorizations"] == 1
    err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert err <= 1e-8, err
    ctx.close()


def test_adjoint_with_factor_reuse_over_energies():
    """reuse_factors on: the symmetric-potential adjoint at consecutive energies keeps one
    factorisation; every gradient still matches the oracle."""
    w = workloads.production(nch=16, nr=60, rmax=15.0)
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    ctx = api.Context(precision="mixed", reuse_factors=True)
    facts = 0
    for e in (8.0, 8.4, 8.8, 9.2):
        wk = workloads.at_energy(w, e)
        u_ref = orc.rmatrix(w.nch, w.lval, wk.qk, wk.eta, w.rmax, mesh, w.cpot).cu
        gu = 2 * (u_ref - np.eye(u_ref.shape[0]))
        _, g_ref = orc.rmatrix_adjoint(w.nch, w.lval, wk.qk, wk.eta, w.rmax, mesh, w.cpot, gu)
        cu, nopen, g = ctx.rmatrix_adjoint(w.nch, w.lval, wk.qk, wk.eta, w.rmax, w.nr, w.cpot, gu)
        facts += ctx.last_stats["factorizations"]
        assert np.linalg.norm(cu[:nopen, :nopen] - u_ref) <= 1e-10 * np.linalg.norm(u_ref)
        assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) <= 1e-8
    assert facts < 4, facts
    ctx.close()


def test_parameter_gradients_match_central_differences():
    w = workloads.production(nch=12, nr=60, rmax=15.0)
    energies = [6.0, 12.0, 19.0]
    r = torch.from_numpy(workloads.lagrange_radii(w.nr, w.rmax))
    coup = torch.from_numpy(w.coupling)
    p0 = torch.tensor(w.params.as_array(), dtype=torch.float64)
    ptarget = p0 * torch.tensor([1.02, 0.97, 1.01, 1.03, 0.95, 1.04], dtype=torch.float64)
    ctx = api.Context(precision="mixed")
    kin = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in energies]

    def loss(p, with_grad):
        cp = potential_matrix(r, coup, p, w.hm, w.params.z1z2)
        tgt = potential_matrix(r, coup, ptarget, w.hm, w.params.z1z2).detach().numpy()
        tot = 0.0
        for qk, eta in kin:
            u_t = ctx.rmatrix(w.nch, w.lval, qk, eta, w.rmax, w.nr, 1, np.asfortranarray(tgt))[0]
            u = collision_matrix(cp, ctx, w.lval, qk, eta, w.rmax, w.nr)
            no = u.shape[0]
            tot = tot + torch.sum(torch.abs(u - torch.from_numpy(u_t[:no, :no])) ** 2)
        return tot

    p = p0.clone().requires_grad_(True)
    L = loss(p, True)
    L.backward()
    g = p.grad.numpy()
    h = 1e-6
    for k in range(6):
        e = torch.zeros(6, dtype=torch.float64)
        e[k] = h * max(1.0, abs(float(p0[k])))
        fd = (float(loss(p0 + e, False)) - float(loss(p0 - e, False))) / (2 * float(e[k]))
        assert abs(fd - g[k]) <= 1e-6 * max(abs(fd), 1e-12) + 1e-9, (k, fd, g[k])
    ctx.close()


def test_adjoint_from_kept_forward_solution():
    """rmatrix_x keeps X = C^-1 Q on the device; adjoint_from_x forms the gradient from it with no
    further solve and matches rmatrix_adjoint and the oracle."""
    w = workloads.production(nch=14, nr=60, rmax=15.0)
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    u_ref = orc.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot).cu
    gu = 2 * (u_ref - 0.5 * np.eye(u_ref.shape[0]))
    _, g_ref = orc.rmatrix_adjoint(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot, gu)
    ctx = api.Context(precision="mixed")
    cu, nopen, x = ctx.rmatrix_x(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, w.cpot)
    assert x.is_cuda and tuple(x.shape) == (w.nch * w.nr, w.nch)
    assert np.linalg.norm(cu[:nopen, :nopen] - u_ref) <= 1e-10 * np.linalg.norm(u_ref)
    g = ctx.adjoint_from_x(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, w.cpot, cu, x, gu)
    assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) <= 1e-8
    _, _, g2 = ctx.rmatrix_adjoint(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, w.cpot, gu)
    assert np.linalg.norm(g - g2) / np.linalg.norm(g2) <= 1e-10
    bad = np.array(w.cpot, order="F")
    bad[:, 0, 1] += 1e-3
    with pytest.raises(api.HprmatError):
        ctx.adjoint_from_x(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, bad, cu, x, gu)
    ctx.close()


def test_batched_collision_matrices_match_per_energy():
    """collision_matrices over a pool of 3 contexts (concurrent solves) gives the same U and the
    same parameter gradient as collision_matrix energy by energy."""
    from hprmat_b200.autograd import collision_matrices
    w = workloads.production(nch=10, nr=50, rmax=15.0)
    energies = [5.0, 7.5, 10.0, 12.5, 15.0]
    kin = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in energies]
    r = torch.from_numpy(workloads.lagrange_radii(w.nr, w.rmax))
    coup = torch.from_numpy(w.coupling)
    p0 = torch.tensor(w.params.as_array(), dtype=torch.float64)
    pool = [api.Context(precision="mixed") for _ in range(3)]
    ctx = api.Context(precision="mixed")

    p = p0.clone().requires_grad_(True)
    us = collision_matrices(potential_matrix(r, coup, p, w.hm, w.params.z1z2), pool, w.lval, kin, w.rmax, w.nr)
    L1 = sum(torch.sum(torch.abs(u) ** 2 * (1 + k)) for k, u in enumerate(us))
    L1.backward()
    g1 = p.grad.clone()

    q = p0.clone().requires_grad_(True)
    cp = potential_matrix(r, coup, q, w.hm, w.params.z1z2)
    us2 = [collision_matrix(cp, ctx, w.lval, qk, eta, w.rmax, w.nr) for qk, eta in kin]
    L2 = sum(torch.sum(torch.abs(u) ** 2 * (1 + k)) for k, u in enumerate(us2))
    L2.backward()
    for a, b in zip(us, us2):
        a, b = a.detach(), b.detach()
        assert torch.allclose(a, b, rtol=0, atol=1e-12 * float(b.abs().max()))
    assert torch.allclose(g1, q.grad, rtol=1e-10, atol=1e-12 * float(q.grad.abs().max()))
    for c in pool + [ctx]:
        c.close()


def _config4():
    """The adjoint configuration: 32 channels x 100 points (N = 3200), three of its 64 energies
    (one low, one middle, one high; COULFG evaluates every open channel at all three)."""
    from oracle import special_functions as sf
    w, energies = workloads.adjoint_case()
    picked = []
    for e in (energies[3], energies[31], energies[60]):
        qk, eta = workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2)
        assert all(sf.coulfg(qk[c] * w.rmax, eta[c], float(w.lval[c]))[4] == 0 for c in range(w.nch) if qk[c] > 0)
        picked.append((qk, eta))
    return w, picked


def test_config4_mesh_gradient_matches_oracle_adjoint():
    """N = 3200: the device gradient with respect to the potential at every mesh point, for
    L = sum |U - U_target|^2 (target from perturbed parameters), against the FP64 oracle adjoint
    (dense LAPACK solves) to 1e-8, with the potential handed over as a CUDA tensor (the
    device-resident forward and backward of the autograd function)."""
    w, kin = _config4()
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    tgt = w.cpot * 1.01
    ctx = api.Context(precision="mixed")
    cp_dev = torch.from_numpy(np.ascontiguousarray(w.cpot)).cuda()
    for qk, eta in kin[:2]:
        u_ref = orc.rmatrix(w.nch, w.lval, qk, eta, w.rmax, mesh, w.cpot).cu
        u_tgt = orc.rmatrix(w.nch, w.lval, qk, eta, w.rmax, mesh, tgt).cu
        gu = 2 * (u_ref - u_tgt)
        _, g_ref = orc.rmatrix_adjoint(w.nch, w.lval, qk, eta, w.rmax, mesh, w.cpot, gu)
        cp = cp_dev.clone().requires_grad_(True)
        u = collision_matrix(cp, ctx, w.lval, qk, eta, w.rmax, w.nr)
        assert u.is_cuda
        L = torch.sum(torch.abs(u - torch.from_numpy(u_tgt).cuda()) ** 2)
        L.backward()
        assert np.linalg.norm(u.detach().cpu().numpy() - u_ref) <= 1e-10 * np.linalg.norm(u_ref)
        assert cp.grad.is_cuda
        # torch's gradient of a real loss with respect to a complex tensor follows dL = Re sum
        # conj(grad) dcpot, the convention of the library and of the oracle adjoint
        g = cp.grad.cpu().numpy()
        err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
        assert err <= 1e-8, err
    ctx.close()


def test_config4_parameter_gradients_match_central_differences():
    """N = 3200, three energies: the gradient of L = sum_E sum |U - U_target|^2 with respect to
    the six potential parameters (V0, W0, R, a, coupling scale, Coulomb radius), through
    torch.autograd on CUDA tensors, against central differences (step 1e-6 relative) of the
    device forward to 1e-6.  The differences' forward solves run to tighter tolerances so that
    the solver's rounding noise in U stays far below the difference quotient."""
    w, kin = _config4()
    dev = torch.device("cuda", 0)
    r = torch.from_numpy(workloads.lagrange_radii(w.nr, w.rmax)).to(dev)
    coup = torch.from_numpy(w.coupling).to(dev)
    p0 = torch.tensor(w.params.as_array(), dtype=torch.float64, device=dev)
    ptarget = p0 * torch.tensor([1.02, 0.97, 1.01, 1.03, 0.95, 1.04], dtype=torch.float64, device=dev)
    ctx = api.Context(precision="mixed", max_refine=8)
    tgt = potential_matrix(r, coup, ptarget, w.hm, w.params.z1z2)
    targets = [collision_matrix(tgt, ctx, w.lval, qk, eta, w.rmax, w.nr).detach() for qk, eta in kin]

    def loss(p):
        cp = potential_matrix(r, coup, p, w.hm, w.params.z1z2)
        tot = 0.0
        for (qk, eta), ut in zip(kin, targets):
            u = collision_matrix(cp, ctx, w.lval, qk, eta, w.rmax, w.nr)
            tot = tot + torch.sum(torch.abs(u - ut) ** 2)
        return tot

    p = p0.clone().requires_grad_(True)
    loss(p).backward()
    g = p.grad.cpu().numpy()
    ctx.set_precision("mixed", max_refine=8, tol=1e-14, surface_tol=1e-13)
    for k in range(6):
        e = torch.zeros(6, dtype=torch.float64, device=dev)
        e[k] = 1e-6 * max(1.0, abs(float(p0[k])))
        with torch.no_grad():
            fd = (float(loss(p0 + e)) - float(loss(p0 - e))) / (2 * float(e[k]))
        assert abs(fd - g[k]) <= 1e-6 * abs(fd) + 1e-12, (k, fd, g[k])
    ctx.close()


def test_device_and_host_potentials_give_the_same_gradient():
    """collision_matrix with the potential as a CUDA tensor (device entry points, nothing of the
    potential's size crosses to the host) and as a CPU tensor (host entry points): the same U
    and the same mesh-point gradient."""
    w = workloads.production(nch=12, nr=60, rmax=15.0)
    ctx = api.Context(precision="mixed")
    out = []
    for device in ("cpu", "cuda"):
        cp = torch.from_numpy(np.ascontiguousarray(w.cpot)).to(device).requires_grad_(True)
        u = collision_matrix(cp, ctx, w.lval, w.qk, w.eta, w.rmax, w.nr)
        assert u.device.type == device
        L = torch.sum(torch.abs(u) ** 2 * torch.arange(1, u.shape[1] + 1, device=device))
        L.backward()
        assert cp.grad.device.type == device
        out.append((u.detach().cpu().numpy(), cp.grad.cpu().numpy()))
    (u0, g0), (u1, g1) = out
    assert np.linalg.norm(u1 - u0) <= 1e-12 * np.linalg.norm(u0)
    assert np.linalg.norm(g1 - g0) <= 1e-10 * np.linalg.norm(g0)
    ctx.close()
