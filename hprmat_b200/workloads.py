"""Seeded synthetic coupled-channel inputs of the sizes the solver is measured on.

Each generator returns the arguments of ``rmatrix`` (src/rmatrix_hp.F90:175-176) for one
(J, pi, E): channel angular momenta ``lval``, signed wave numbers ``qk`` (negative for
closed channels), Sommerfeld parameters ``eta`` and the coupling potentials ``cpot`` in
fm^-2 (V / (hbar^2/2mu)) at the Lagrange mesh points, Fortran layout (ncp1, nch, nch).

Conventions follow the reference's example drivers: hbar^2/2mu = 20.736/mu MeV fm^2
(examples/Ex1/example1_hp.f90:55); k = sqrt(|E - threshold| / hm), negative when closed;
eta = Z1 Z2 e^2 / (2 hm |k|) with e^2 = 1.44 MeV fm; a uniformly charged sphere for the
Coulomb term (examples/Ex4/example4_hp.f90:94-95).

Workloads (all seeded, deterministic):
  * ``small``      -- 8 channels x 50 points on [0, 10 fm] (N = 400), E = 5 MeV, l = 0..7,
                      all channels open, no Coulomb.
  * ``production`` -- 128 channels x 200 points on [0, 20 fm] (N = 25600), E = 10 MeV,
                      complex couplings, thresholds U(0, 20) MeV (open and closed channels),
                      Coulomb Z1 Z2 = 6 with a 3 fm charge radius.
  * ``sweep``      -- the production generator at nch in {20, 50, 80, 128, 256}, with the
                      thresholds of closed channels moved to 40 MeV.
  * ``scan``       -- 12 J-pi blocks with nch ~ U{4..64} x 60 points, 256 energies each.
  * ``adjoint``    -- 32 channels x 100 points (N = 3200) at 64 energies.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

E2 = 1.44          # e^2 in MeV fm
HBAR2_2MU = 20.736  # hbar^2 / (2 * 1 amu) in MeV fm^2


@dataclass
class PotentialParams:
    """Parameters of the synthetic potential (the differentiable ones come first)."""
    v0: float = -50.0      # Woods-Saxon real depth (MeV)
    w0: float = -10.0      # Woods-Saxon imaginary depth (MeV)
    rws: float = 3.0       # Woods-Saxon radius (fm)
    aws: float = 0.6       # Woods-Saxon diffuseness (fm)
    cscale: float = 1.0    # scale of the Gaussian couplings
    rc: float = 3.0        # Coulomb charge radius (fm)
    z1z2: float = 0.0      # Z1 * Z2

    def as_array(self):
        return np.array([self.v0, self.w0, self.rws, self.aws, self.cscale, self.rc])


@dataclass
class Workload:
    name: str
    nch: int
    nr: int
    ns: int
    rmax: float
    energy: float
    hm: float
    lval: np.ndarray
    thresholds: np.ndarray
    coupling: np.ndarray       # (nch, nch) complex couplings c_ij (MeV), symmetric
    params: PotentialParams
    cpot: np.ndarray = field(default=None, repr=False)   # (nr, nch, nch) complex, Fortran
    qk: np.ndarray = None
    eta: np.ndarray = None

    @property
    def n(self):
        return self.nch * self.nr


def lagrange_radii(nr: int, rmax: float) -> np.ndarray:
    """Mesh abscissas r_i = a x_i with x_i the Gauss-Legendre nodes on (0, 1)."""
    x, _ = np.polynomial.legendre.leggauss(nr)
    return np.sort((x + 1.0) / 2.0) * rmax


def potential_matrix(r: np.ndarray, nch: int, coupling: np.ndarray, p: PotentialParams,
                     hm: float) -> np.ndarray:
    """cpot(r_i, c, c') / hm for the diagonal Woods-Saxon + Coulomb and Gaussian couplings."""
    ws = complex(p.v0, p.w0) / (1.0 + np.exp((r - p.rws) / p.aws))
    if p.z1z2 != 0.0:
        ze = p.z1z2 * E2
        vc = np.where(r <= p.rc, ze * (3.0 - (r / p.rc) ** 2) / (2.0 * p.rc), ze / np.maximum(r, 1e-300))
    else:
        vc = np.zeros_like(r)
    g = np.exp(-(r / 2.0) ** 2)
    cpot = np.empty((r.shape[0], nch, nch), dtype=np.complex128, order="F")
    cpot[:] = (p.cscale * coupling)[None, :, :] * g[:, None, None]
    diag = ws + vc
    for c in range(nch):
        cpot[:, c, c] = diag
    return cpot / hm


def channel_kinematics(energy: float, thresholds: np.ndarray, hm: float, z1z2: float):
    """Signed k (negative = closed) and eta per channel, as in examples/Ex4/example4_hp.f90:118-129."""
    e2 = energy - thresholds
    k = np.sqrt(np.abs(e2) / hm)
    eta = (z1z2 * E2 / (2.0 * hm)) / k if z1z2 != 0.0 else np.zeros_like(k)
    qk = np.where(e2 < 0, -k, k)
    return qk, eta


def _finish(w: Workload) -> Workload:
    r = lagrange_radii(w.nr, w.rmax)
    w.cpot = potential_matrix(r, w.nch, w.coupling, w.params, w.hm)
    w.qk, w.eta = channel_kinematics(w.energy, w.thresholds, w.hm, w.params.z1z2)
    return w


def _sym(rng, nch, complex_part: bool):
    re = rng.uniform(-5.0, 5.0, size=(nch, nch))
    c = re.astype(np.complex128)
    if complex_part:
        c = c + 1j * rng.uniform(-1.0, 0.0, size=(nch, nch))
    c = np.triu(c, 1)
    return c + c.T


def small(seed: int = 0) -> Workload:
    """8 channels x 50 points (N = 400), E = 5 MeV, all channels open."""
    rng = np.random.default_rng(seed)
    nch, nr = 8, 50
    coupling = _sym(rng, nch, complex_part=False)
    thr = rng.uniform(0.0, 3.0, size=nch)
    return _finish(Workload("small", nch, nr, 1, 10.0, 5.0, HBAR2_2MU,
                            np.arange(nch, dtype=np.int32), thr, coupling, PotentialParams()))


def production(seed: int = 1, nch: int = 128, nr: int = 200, rmax: float = 20.0,
               energy: float = 10.0, closed_threshold: float | None = None,
               name: str = "production") -> Workload:
    """128 channels x 200 points (N = 25600) at E = 10 MeV with open and closed channels."""
    rng = np.random.default_rng(seed)
    coupling = _sym(rng, nch, complex_part=True)
    thr = rng.uniform(0.0, 20.0, size=nch)
    thr[0] = 0.0  # the entrance channel is open
    if closed_threshold is not None:
        thr = np.where(thr > energy, closed_threshold, thr)
    lval = (np.arange(nch) % 10).astype(np.int32)
    params = PotentialParams(z1z2=6.0, rc=3.0)
    return _finish(Workload(name, nch, nr, 1, rmax, energy, HBAR2_2MU, lval, thr, coupling,
                            params))


SWEEP_NCH = (20, 50, 80, 128, 256)


def sweep(nch: int, seed: int = 2) -> Workload:
    """Production generator at N = 200 nch with closed-channel thresholds at 40 MeV."""
    return production(seed=seed, nch=nch, closed_threshold=40.0, name=f"sweep{nch}")


def with_intervals(w: Workload, ns: int) -> Workload:
    """The same potential on ns intervals of w.nr points each over [0, w.rmax] (R-matrix
    propagation, src/rmatrix_hp.F90:153-157 for the mesh): cpot has w.nr * ns rows."""
    rmax0 = w.rmax / ns
    x = lagrange_radii(w.nr, 1.0)
    r = np.concatenate([(s + x) * rmax0 for s in range(ns)])
    out = Workload(w.name, w.nch, w.nr, ns, w.rmax, w.energy, w.hm, w.lval, w.thresholds,
                   w.coupling, w.params)
    out.cpot = potential_matrix(r, w.nch, w.coupling, w.params, w.hm)
    out.qk, out.eta = w.qk, w.eta
    return out


def at_energy(w: Workload, energy: float) -> Workload:
    """The same potential at another energy (only k and eta change)."""
    out = Workload(w.name, w.nch, w.nr, w.ns, w.rmax, energy, w.hm, w.lval, w.thresholds,
                   w.coupling, w.params, w.cpot)
    out.qk, out.eta = channel_kinematics(energy, w.thresholds, w.hm, w.params.z1z2)
    return out


def scan_blocks(seed: int = 3, nblocks: int = 12, nenergies: int = 256, nr: int = 60,
                rmax: float = 20.0):
    """J-pi blocks of the batched energy scan: list of (Workload at E[0], energies)."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(nblocks):
        nch = int(rng.integers(4, 65))
        w = production(seed=seed * 1000 + b, nch=nch, nr=nr, rmax=rmax, energy=1.0,
                       name=f"scan{b}")
        energies = np.sort(rng.uniform(1.0, 30.0, size=nenergies))
        out.append((w, energies))
    return out


def adjoint_case(seed: int = 4, nch: int = 32, nr: int = 100, nenergies: int = 64):
    """32 channels x 100 points, 64 energies in 5-25 MeV."""
    w = production(seed=seed, nch=nch, nr=nr, rmax=20.0, energy=10.0, name="adjoint")
    energies = np.linspace(5.0, 25.0, nenergies)
    return w, energies
