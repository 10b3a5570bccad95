"""Oracle (test infrastructure only): CPU restatement of HPRMAT's boundary functions.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may use
this module, and only as the checker.  The product computes the same quantities in
``hprmat_b200/csrc/coulomb.cuh``.

Restated algorithms (reference paths are relative to the HPRMAT project root):

* ``coulfg``  -- ``src/special_functions.f:1-275`` (Barnett's COULFG, Steed's method,
  CPC 27 (1982) 147), restricted to the form the R-matrix path calls it with:
  ``MODE1=1, KFN=0, XLMIN=XLMAX`` (``src/rmatrix_hp.F90:232``), so ``LXTRA=0`` and no
  recurrence in lambda is needed.
* ``jwkb``    -- ``src/special_functions.f:277-306``.
* ``whit``    -- ``src/special_functions.f:309-416`` (I.J. Thompson's Whittaker function:
  asymptotic series at a far point plus Numerov integration inwards).

The Fortran source writes several literals in default (single) precision, e.g.
``10.0/12.0`` and ``0.15`` in WHIT.  Those constants are reproduced here exactly as the
Fortran compiler forms them (single-precision value widened to double), because they set
WHIT's result at the 1e-8 level and therefore the closed-channel Bloch term of C(E).
"""
from __future__ import annotations

import math

import numpy as np


def _f32(x: float) -> float:
    """Value of a default-precision Fortran REAL literal after widening to REAL*8."""
    return float(np.float32(x))


# Single-precision literals of WHIT (src/special_functions.f:354-376).
_W_10_12 = float(np.float32(10.0) / np.float32(12.0))
_W_1_6 = float(np.float32(1.0) / np.float32(6.0))
_W_1_12 = float(np.float32(1.0) / np.float32(12.0))
_W_1_60 = float(np.float32(1.0) / np.float32(60.0))
_W_0_15 = _f32(0.15)


def jwkb(xx: float, eta1: float, xl: float):
    """JWKB approximation to F and G (src/special_functions.f:277-306).

    Returns (fjwkb, gjwkb, iexp).  If the turning-point test fails the Fortran routine
    returns without touching its outputs; that case yields ``None`` here.
    """
    zero, half, one, six, ten = 0.0, 0.5, 1.0, 6.0, 10.0
    rl35 = 35.0
    aloge = math.log(ten)
    x = xx
    eta = eta1
    gh2 = x * (eta + eta - x)
    xll1 = max(xl * xl + xl, 0.0)
    if gh2 + xll1 <= zero:
        return None
    hll = xll1 + six / rl35
    hl = math.sqrt(hll)
    sl = eta / hl + hl / x
    rl2 = one + eta * eta / hll
    gh = math.sqrt(gh2 + hll) / x
    phi = x * gh - half * (hl * math.log((gh + sl) ** 2 / rl2) - math.log(gh))
    if eta != zero:
        phi = phi - eta * math.atan2(x * gh, x - eta)
    phi10 = -phi * aloge
    iexp = int(phi10)
    if iexp > 70:
        gjwkb = ten ** (phi10 - iexp)
    else:
        gjwkb = math.exp(-phi)
        iexp = 0
    fjwkb = half / (gh * gjwkb)
    return fjwkb, gjwkb, iexp


def coulfg(xx: float, eta1: float, xl: float):
    """F_l, G_l, F'_l, G'_l at a single integer-spaced lambda (src/special_functions.f:1-275).

    Returns ``(fc, gc, fcp, gcp, ifail)``; derivatives are with respect to ``xx``.
    """
    zero, one, two, ten2, abort = 0.0, 1.0, 2.0, 100.0, 2.0e4
    half, tm30 = 0.5, 1.0e-30
    accur = 1.0e-16
    eta = eta1
    gjwkb = zero
    etane0 = eta != zero
    acc = accur * 10.0
    acc4 = acc * ten2 * ten2
    acch = math.sqrt(acc)
    if xx <= acch:
        return 0.0, 0.0, 0.0, 0.0, -1
    x = xx
    xlm = xl
    if xlm <= -one:
        return 0.0, 0.0, 0.0, 0.0, -2
    e2mm1 = eta * eta + xlm * xlm + xlm
    xlturn = x * (x - two * eta) < xlm * xlm + xlm
    xll = xlm  # LXTRA = 0 (XLMIN = XLMAX)

    # CF1 = F'/F at lambda = xll (src/special_functions.f:88-115)
    xi = one / x
    fcl = one
    pk = xll + one
    px = pk + abort
    f = eta / pk + pk * xi
    if abs(f) < tm30:
        f = tm30
    d = zero
    c = f
    while True:
        pk1 = pk + one
        ek = eta / pk
        rk2 = one + ek * ek
        tk = (pk + pk1) * (xi + ek / pk1)
        d = tk - rk2 * d
        c = tk - rk2 / c
        if abs(c) < tm30:
            c = tm30
        if abs(d) < tm30:
            d = tm30
        d = one / d
        df = d * c
        f = f * df
        if d < zero:
            fcl = -fcl
        pk = pk1
        if pk > px:
            return 0.0, 0.0, 0.0, 0.0, -3
        if abs(df - one) < acc:
            break

    # CF2 = p + i q (src/special_functions.f:153-196)
    iexp = 1
    if xlturn:
        r = jwkb(x, eta, max(xlm, zero))
        if r is not None:
            fjwkb, gjwkb, iexp = r
        else:
            fjwkb = 0.0
    use_jwkb = iexp > 1 or gjwkb > one / (acch * ten2)
    if not use_jwkb:
        xlturn = False
        ta = two * abort
        pk = zero
        wi = eta + eta
        p = zero
        q = one - eta * xi
        ar = -e2mm1
        ai = eta
        br = two * (x - eta)
        bi = two
        dr = br / (br * br + bi * bi)
        di = -bi / (br * br + bi * bi)
        dp = -xi * (ar * di + ai * dr)
        dq = xi * (ar * dr - ai * di)
        while True:
            p = p + dp
            q = q + dq
            pk = pk + two
            ar = ar + pk
            ai = ai + wi
            bi = bi + two
            d = ar * dr - ai * di + br
            di = ai * dr + ar * di + bi
            c = one / (d * d + di * di)
            dr = c * d
            di = -c * di
            a = br * dr - bi * di - one
            b = bi * dr + br * di
            c = dp * a - dq * b
            dq = dp * b + dq * a
            dp = c
            if pk > ta:
                return 0.0, 0.0, 0.0, 0.0, -4
            if abs(dp) + abs(dq) < (abs(p) + abs(q)) * acc:
                break
        gam = (f - p) / q
        if q <= acc4 * abs(p):
            return 0.0, 0.0, 0.0, 0.0, -5
        w = one / math.sqrt((f - p) * gam + q)
    else:
        # src/special_functions.f:198-201
        w = fjwkb
        gam = gjwkb * w
        p = f
        q = one

    # Normalisation for KFN = 0 (src/special_functions.f:205-221)
    alpha = zero
    beta = one
    fcm = math.copysign(w, fcl) * beta
    if not xlturn:
        gcl = fcm * gam
    else:
        gcl = gjwkb * beta
    gpl = gcl * (p - q / gam) - alpha * gcl
    fcp = fcm * (f - alpha)
    return fcm, gcl, fcp, gpl, 0


def whit(heta: float, r: float, xk: float, e: float, ll: int, ie: int = 0):
    """Whittaker function W and k*dW/d(kr) for l = 0..ll (src/special_functions.f:309-416).

    Returns ``(f, fd, ie)`` with ``f[l]``, ``fd[l]`` for l = 0..ll; ``fd`` already carries
    the factor ``xk`` applied at the end of the Fortran routine (``FD(M)=AK*FD(M)``).
    """
    fpmax = 1.0e290
    L = ll + 1
    ee = -1.0
    ak = xk
    eta = heta
    rho = ak * r
    s = [0.0] * 8  # 1-based S(1..7)
    t = [0.0] * 4  # 1-based T(1..3)
    is_ = 7
    pje = 30.0 * rho + 1.0
    h = float(max(int(pje), 4))
    h = rho / h
    rhoa = 10.0 * (eta + 1.0)
    if rhoa - rho <= 0:
        ifeql = 1
        rhoa = rho
    else:
        ifeql = 0
    pje = rhoa / h + 0.5
    rhoa = h * int(pje)
    if ifeql <= 0:
        if rhoa - rho - 1.5 * h < 0:
            rhoa = rho + 2.0 * h
    assert ee <= 0
    f = [0.0] * (L + 1)
    fd = [0.0] * (L + 1)
    while True:
        # label 55: asymptotic series at rhoa
        c = 1.0 / rhoa
        a = 1.0
        b = 1.0 - c * eta
        f[1] = a
        fd[1] = b
        for m in range(1, 27):
            d = 0.5 * (eta + float(m - 1)) * (eta + float(m)) * c / float(m)
            a = -a * d
            b = -b * d - a * c
            f[1] = f[1] + a
            fd[1] = fd[1] + b
        a = -eta * math.log(2.0 * rhoa) - rhoa
        fpminl = -math.log(fpmax)
        if ie == 0 and a < fpminl:
            ie = int(fpminl - a)
        a = math.exp(a + ie)
        f[1] = a * f[1]
        fd[1] = a * fd[1] * (-1.0 - 2 * eta / rhoa)
        if ifeql > 0:
            break  # label 61
        s[is_] = f[1]
        if is_ == 7:
            is_ = 6
            rhoa = rhoa + h
            continue
        # label 27: Numerov integration inwards
        a = 2.0 - _W_10_12 * h * h * ee
        b = _W_1_6 * h * eta
        c = 1.0 + _W_1_12 * h * h * ee
        m1 = int(rhoa / h - 0.5)
        m2 = int(rho / h - 1.5)
        t[2] = b / float(m1 + 1)
        t[3] = b / float(m1)
        js = m1
        for _ in range(m2, m1 + 1):
            for i in range(1, 7):
                s[i] = s[i + 1]
            t[1] = t[2]
            t[2] = t[3]
            t[3] = b / float(js - 1)
            s[7] = ((a + 10.0 * t[2]) * s[6] - (c - t[1]) * s[5]) / (c - t[3])
            js = js - 1
            if abs(s[7]) > fpmax:
                for i in range(2, 8):
                    s[i] = s[i] / fpmax
        t[1] = s[4]
        t[2] = (_W_1_60 * (s[1] - s[7]) + _W_0_15 * (s[6] - s[2]) + 0.75 * (s[3] - s[5])) / h
        f[1] = t[1]
        fd[1] = t[2]
        break
    # label 61: upward recurrence in l
    c = 1.0 / rho
    for m in range(1, L):
        a = eta / float(m)
        b = a + c * float(m)
        f[m + 1] = (b * f[m] - fd[m]) / (a + 1.0)
        fd[m + 1] = (a - 1.0) * f[m] - b * f[m + 1]
    for m in range(1, L + 1):
        fd[m] = ak * fd[m]
    return f[1:], fd[1:], ie
