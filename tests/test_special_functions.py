"""Boundary functions: the oracle's COULFG/WHIT restatement against mpmath (CPU)."""
import math

import mpmath as mp
import pytest

from oracle.special_functions import coulfg, whit

mp.mp.dps = 30


@pytest.mark.parametrize("x,eta,l", [(5.0, 0.0, 0), (19.2, 0.0, 3), (27.5, 1.7, 4), (40.0, 0.3, 9),
                                     (12.0, 0.9, 2), (25.0, 2.5, 0)])
def test_coulfg_oscillating_region(x, eta, l):
    f, g, fp, gp, ifail = coulfg(x, eta, float(l))
    assert ifail == 0
    F = float(mp.coulombf(l, eta, x))
    G = float(mp.coulombg(l, eta, x))
    Fp = float(mp.diff(lambda t: mp.coulombf(l, eta, t), x))
    Gp = float(mp.diff(lambda t: mp.coulombg(l, eta, t), x))
    for a, b in [(f, F), (g, G), (fp, Fp), (gp, Gp)]:
        assert abs(a - b) <= 1e-12 * max(1.0, abs(b)), (a, b)
    # Wronskian F'G - FG' = 1
    assert abs(fp * g - f * gp - 1.0) < 1e-12


def test_coulfg_jwkb_branch_is_the_reference_approximation():
    """Deep under the barrier COULFG switches to the JWKB estimates of F and G
    (src/special_functions.f:153-154, 198-201): they agree with the exact functions only to
    about a percent there, exactly as in the reference (Ex1's 10-20 MeV points use it)."""
    x, eta, l = 19.2, 16.2, 20
    f, g, fp, gp, ifail = coulfg(x, eta, float(l))
    F = float(mp.coulombf(l, eta, x))
    G = float(mp.coulombg(l, eta, x))
    assert ifail == 0
    assert abs(f - F) <= 0.02 * abs(F)
    assert abs(g - G) <= 0.02 * abs(G)


@pytest.mark.parametrize("eta,r,k,l", [(0.0, 10.0, 0.5, 0), (0.4, 20.0, 0.8, 3), (1.3, 14.0, 0.6, 5),
                                       (0.0, 8.0, 1.2, 2)])
def test_whittaker(eta, r, k, l):
    f, fd, ie = whit(eta, r, k, -k * k, l, 0)
    W = mp.whitw(-eta, l + 0.5, 2 * k * r)
    Wd = mp.diff(lambda t: mp.whitw(-eta, l + 0.5, 2 * k * t), r)
    scale = math.exp(ie)
    # WHIT is an asymptotic series (26 terms) plus Numerov steps with single-precision
    # constants and an upward recurrence in l: accurate to ~1e-3 relative at these points
    # (the reference method's own accuracy; the oracle and the product share it).
    assert abs(f[l] - float(W) * scale) <= 1e-3 * abs(float(W) * scale)
    assert abs(fd[l] - float(Wd) * scale) <= 1e-3 * abs(float(Wd) * scale)
    # the log-derivative a W'/W that enters C(E) is what matters
    assert abs(fd[l] / f[l] - float(Wd / W)) <= 1e-3 * abs(float(Wd / W))
