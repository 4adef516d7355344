"""CPU checks of the Coriolis oracle (oracle/sph_coriolis.py).

- The restated Gaunt integral gs equals the integral over [-1, 1] of three
  Schmidt-normalised associated Legendre functions (Gauss-Legendre quadrature).
- The closed forms the device tables use for the rotation's couplings (degree
  1, order 0) equal the restated leadki / leadli for every (l, m) up to 40.
- The spectral curl of the Coriolis term equals the grid route: the CPU
  transform oracle forms -c z x u on the grid (z is the poloidal l = 1, m = 0
  field S = r^2/2, the reference's rotation spectrum), transforms it back,
  and its curl is taken spectrally; with S_u = b r + c r^2, T_u = e r + f r^2
  every radial profile involved is a quadratic, so the 3-point central
  difference on three radii is exact.
"""
from math import factorial

import numpy as np
import pytest

from kemorin_mhd_b200.config import PROD_CROSS, SphConfig, rj_order
from oracle.sph_coriolis import gs, leadki, leadli, rot_coriolis


def _schmidt(l, m, x):
    from scipy.special import lpmv
    v = lpmv(m, l, x) * (-1) ** m          # no Condon-Shortley phase
    if m > 0:
        v = v * np.sqrt(2.0 * factorial(l - m) / factorial(l + m))
    return v


@pytest.mark.parametrize("m1,l1,m2,l2,m3,l3", [(0, 1, 0, 2, 0, 3), (1, 2, 0, 1, 1, 3), (2, 5, 0, 1, 2, 4),
                                               (3, 7, 1, 2, 2, 5), (2, 4, 1, 3, 1, 3), (5, 9, 2, 6, 3, 5),
                                               (0, 1, 0, 10, 0, 11), (7, 20, 0, 1, 7, 21)])
def test_gaunt_equals_quadrature(m1, l1, m2, l2, m3, l3):
    x, w = np.polynomial.legendre.leggauss(120)
    ref = np.sum(w * _schmidt(l1, m1, x) * _schmidt(l2, m2, x) * _schmidt(l3, m3, x))
    assert abs(gs(m1, l1, m2, l2, m3, l3) - ref) <= 1e-13 * max(1.0, abs(ref))


def test_coriolis_closed_forms_equal_restated_integrals():
    for l in range(1, 41):
        for m in range(-l, l + 1):
            if l >= 2 and abs(m) <= l - 1:
                c1 = 4.0 * np.sqrt(l * l - m * m) / ((2 * l - 1) * (2 * l + 1))
                assert abs(leadki(1, 0, l - 1, m, l, m) - c1) <= 1e-15 * c1
            c2 = 4.0 * np.sqrt((l + 1) ** 2 - m * m) / ((2 * l + 1) * (2 * l + 3))
            assert abs(leadki(1, 0, l + 1, m, l, m) - c2) <= 1e-15 * c2
            ce = -4.0 * m / (2 * l + 1)
            assert abs(leadli(1, 0, l, -m, l, m) - ce) <= 1e-15 * max(abs(ce), 1.0)


def _quadratic_velocity(L, r, seed):
    """Velocity and vorticity spectra (S, dS/dr, T) on the radii r for
    S_u = b r + c r^2, T_u = e r + f r^2 per mode (l = 0 zero)."""
    l, m = rj_order(L)
    J = len(l)
    rng = np.random.default_rng(seed)
    b, c, e, f = (rng.standard_normal(J) * (l > 0) for _ in range(4))
    g3 = l * (l + 1.0)
    R = r[:, None]
    vS, vdS, vT = b * R + c * R * R, b + 2 * c * R, e * R + f * R * R
    wS, wdS, wT = vT, e + 2 * f * R, -2 * c + g3 * (b / R + c)
    return l, m, [x.reshape(-1) for x in (vS, vdS, vT)], [x.reshape(-1) for x in (wS, wdS, wT)]


@pytest.mark.parametrize("L", [7, 15])
def test_spectral_coriolis_curl_equals_grid_route(L):
    from oracle.oracle import Oracle
    coef = 1.7
    r0, h = 1.1, 0.05
    r = np.array([r0 - h, r0, r0 + h])
    cfg = SphConfig(L, 3 * (L + 1) // 2, 3 * (L + 1), 3, nvb=2, nsb=0, nvf=1, nsf=0,
                    products=((PROD_CROSS, 0, 1, -coef),))
    l, m, velo, vort = _quadratic_velocity(L, r, seed=L)
    J = len(l)
    j10 = int(np.flatnonzero((l == 1) & (m == 0))[0])
    d = np.zeros((J * 3, 6), order="F")
    for k in range(3):
        d[k * J + j10, 0] = 0.5 * r[k] ** 2     # z as a poloidal field
        d[k * J + j10, 1] = r[k]
    for q in range(3):
        d[:, 3 + q] = velo[q]
    frc = Oracle(cfg, nthreads=4, radius=r).cycle(d)        # -c z x u: (S_f, dS_f/dr, T_f)
    Sf, dSf, Tf = (frc[:, q].reshape(3, J) for q in range(3))
    pol_grid = Tf[1]
    tor_grid = -(dSf[2] - dSf[0]) / (2 * h) + l * (l + 1.0) * Sf[1] / r0 ** 2
    pol, tor = (x.reshape(3, J)[1] for x in rot_coriolis(r, L, l, m, velo, vort, coef))
    scale = max(np.abs(pol_grid).max(), np.abs(tor_grid).max())
    # the grid route accumulates the two transforms' rounding (about 1.5e-12 here);
    # a wrong coupling, coefficient or sign shows as an O(1) difference
    assert np.abs(pol - pol_grid).max() <= 1e-11 * scale
    assert np.abs(tor - tor_grid).max() <= 1e-11 * scale
