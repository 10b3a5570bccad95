"""Inputs of the reference's example drivers, restated for the tests.

The potentials and kinematics follow examples/Ex1/example1_hp.f90:53-88,102-105
(alpha + 208Pb), examples/Ex2/example2_hp.f90:32-73,86-88 (Reid NN, T=1) and
examples/Ex4/example4_hp.f90:37-133 (12C + alpha, coupled channels with closed ones) and
rmat_pierre/Ex3/example3.f:1-98 (16O + 44Ca, the same rotational-model couplings).
The mesh-dependent arrays are evaluated at the abscissas `zrma` the caller passes in.
"""
from __future__ import annotations

import math

import numpy as np


def ex1_setup(zrma):
    a1, a2, z1, z2 = 208, 4, 82, 2
    rmu = a1 * a2 / (a1 + a2)
    ze = z1 * z2 * 1.44
    hm = 20.736 / rmu
    eta0 = ze / (2 * hm)
    an = 0.5803
    rn = 1.1132 * (a1 ** (1.0 / 3) + a2 ** (1.0 / 3))
    cpot = np.zeros((len(zrma), 1, 1), dtype=np.complex128, order="F")
    for i, r in enumerate(zrma):
        xx = 1 + math.exp((r - rn) / an)
        cvn = -complex(100, 10) / xx
        cpot[i, 0, 0] = (cvn + ze / r) / hm

    def kin(e, l):
        qk = math.sqrt(e / hm)
        return np.array([l], np.int32), np.array([qk]), np.array([eta0 / qk])

    return cpot, kin


def ex2_setup(zrma, j):
    hm = 20.736 / 0.5
    cpot = np.zeros((len(zrma), 2, 2), dtype=np.complex128, order="F")
    for i, r in enumerate(zrma):
        xx = r * 0.7
        zz = math.exp(-xx)
        vcen = (-10.463 * zz + 105.468 * zz ** 2 - 3187.8 * zz ** 4 + 9924.3 * zz ** 6) / xx
        vtens = (-10.463 * ((1 + 3 / xx + 3 / xx ** 2) * zz - (12 / xx + 3 / xx ** 2) * zz ** 4) / xx
                 + 351.77 * zz ** 4 / xx - 1673.5 * zz ** 6 / xx)
        vls = 708.91 * zz ** 4 / xx - 2713.1 * zz ** 6 / xx
        cpot[i, 0, 0] = vcen - 2 * (j - 1) * vtens / (2 * j + 1) + (j - 1) * vls
        cpot[i, 0, 1] = 6 * vtens * math.sqrt(j * (j + 1.0)) / (2 * j + 1)
        cpot[i, 1, 0] = cpot[i, 0, 1]
        cpot[i, 1, 1] = vcen - 2 * (j + 2) * vtens / (2 * j + 1) - (j + 2) * vls
    cpot /= hm

    def kin(e):
        qk = math.sqrt(e / hm)
        return np.array([j - 1, j + 1], np.int32), np.array([qk, qk]), np.zeros(2)

    return cpot, kin


def _deformed_setup(zrma, j, a1, a2, z1, z2, ispi, th, v0, w0, r0, an, lam, ben, bec):
    """Coupled channels of a deformed Woods-Saxon + Coulomb potential (the drivers'
    rotational-model couplings with 3j/6j coefficients)."""
    from sympy.physics.wigner import wigner_3j, wigner_6j
    ncha = len(ispi)
    pi4 = 4 * math.acos(-1.0)
    rn = r0 * (a1 ** (1.0 / 3) + a2 ** (1.0 / 3))
    rv = r0 * a1 ** (1.0 / 3)
    rmu = a1 * a2 / (a1 + a2)
    ze = z1 * z2 * 1.44
    hm = 20.736 / rmu
    eta0 = ze / (2 * hm)
    chans = [(n, ispi[n], l) for n in range(ncha) for l in range(abs(j - ispi[n]), j + ispi[n] + 1, 2)]
    nv = len(chans)
    xfac = np.zeros((nv, nv))
    for a, (n, ii, l) in enumerate(chans):
        for b, (n2, ii2, l2) in enumerate(chans):
            fac = (2 * l + 1) * (2 * l2 + 1) * (2 * ii + 1) * (2 * ii2 + 1) * (2 * lam + 1)
            t1 = float(wigner_3j(ii2, lam, ii, 0, 0, 0))
            t2 = float(wigner_3j(l, lam, l2, 0, 0, 0))
            s6 = float(wigner_6j(ii, l, j, l2, ii2, lam))
            xfac[a, b] = t1 * t2 * s6 * math.sqrt(fac / pi4)
            if (abs(l - l2) // 2) % 2 == 1:
                xfac[a, b] = -xfac[a, b]
    if (j + lam) % 2 == 1:
        xfac = -xfac
    cpot = np.zeros((len(zrma), nv, nv), dtype=np.complex128, order="F")
    for i, r in enumerate(zrma):
        xx1 = math.exp((r - rn) / an)
        xx = 1 + xx1
        cvn = -complex(v0, w0) / xx
        vc = (3 - (r / rn) ** 2) / 2 / rn if r <= rn else 1 / r
        for iv in range(nv):
            cpot[i, iv, iv] = cvn + ze * vc
        cvn = -complex(v0, w0) * ben * rv * xx1 / (an * xx ** 2)
        vc = r ** lam / rn ** (lam + lam + 1) if r <= rn else 1 / r ** (lam + 1)
        vc = 3 * ze * vc * bec * rv ** lam / (2 * lam + 1)
        cpot[i] += xfac * (cvn + vc)
    cpot /= hm

    def kin(e):
        lval, qk, eta = [], [], []
        for (n, ii, l) in chans:
            e2 = e - th[n]
            k = math.sqrt(abs(e2) / hm)
            lval.append(l)
            eta.append(eta0 / k)
            qk.append(-k if e2 < 0 else k)
        return np.array(lval, np.int32), np.array(qk), np.array(eta)

    return cpot, kin, nv


def ex3_setup(zrma, j):
    """16O + 44Ca (rmat_pierre/Ex3/example3.f:1-98): two states of 44Ca, 4 channels at J = 30."""
    return _deformed_setup(zrma, j, 44, 16, 20, 8, [0, 2], [0.0, 1.156], 110, 20, 1.2, 0.5, 2, 0.40, 0.0)


def ex4_setup(zrma, j):
    """12C + alpha (examples/Ex4/example4_hp.f90:37-133): three states of 12C, closed channels."""
    return _deformed_setup(zrma, j, 12, 4, 6, 2, [0, 2, 4], [0.0, 4.44, 14.08], 110, 20, 1.2, 0.5, 2, 0.58, 0)


def ex5_setup(zrma):
    """Yamaguchi's separable non-local potential (rmat_pierre/Ex5/example5.f:12-41), one s-wave
    channel, no Coulomb: cpot = 0 and cpnl((i-1) nr + j) = -2 beta (alpha + beta)^2
    exp(-beta (r_i + r_j)) in fm^-2 (hbar^2/2mu = 41.472 MeV fm^2)."""
    hm, al, be = 41.472, 0.2316053, 1.3918324
    nr = len(zrma)
    r = np.asarray(zrma)
    cpot = np.zeros((nr, 1, 1), dtype=np.complex128, order="F")
    cpnl = np.zeros((nr * nr, 1, 1), dtype=np.complex128, order="F")
    cpnl[:, 0, 0] = (-2 * be * (al + be) ** 2 * np.exp(-be * (r[:, None] + r[None, :]))).reshape(-1)

    def kin(e):
        qk = math.sqrt(e / hm)
        return np.array([0], np.int32), np.array([qk]), np.array([0.0])

    return cpot, cpnl, kin
