"""CPU checks of the pole-transform oracle (oracle/sph_pole.py): the Schmidt
values at the poles against scipy, and the sign conventions by the uniform
fields x, y, z (poloidal l = 1 fields with S = r^2 / 2, dS/dr = r: orders
+1, -1 and 0), which are (1, 0, 0), (0, 1, 0), (0, 0, 1) at both poles."""
from math import factorial

import numpy as np
import pytest

from kemorin_mhd_b200.config import rj_order
from oracle.sph_pole import b_trans_pole, pole_values


def _schmidt(l, m, x):
    from scipy.special import lpmv
    v = lpmv(m, l, x) * (-1) ** m
    if m > 0:
        v = v * np.sqrt(2.0 * factorial(l - m) / factorial(l + m))
    return v


@pytest.mark.parametrize("l", [1, 2, 3, 7, 12])
def test_pole_values_against_scipy(l):
    pn, ps, dpn, dps = pole_values(l)
    assert pn == _schmidt(l, 0, 1.0) and abs(ps - _schmidt(l, 0, -1.0)) < 1e-15
    h = 1e-5          # one-sided differences of P_l^1(cos theta) at theta = 0 and pi
    fn = (_schmidt(l, 1, np.cos(h)) - 0.0) / h
    fs = (0.0 - _schmidt(l, 1, np.cos(np.pi - h))) / h
    assert abs(fn - dpn) < 1e-6 * l * l and abs(fs - dps) < 1e-6 * l * l


def test_uniform_fields_at_the_poles():
    L, nr = 5, 3
    r = np.array([0.6, 1.0, 1.4])
    l, m = rj_order(L)
    J = len(l)
    d = np.zeros((J * nr, 10))
    for v, mm in enumerate((1, -1, 0)):        # x, y, z
        j = int(np.flatnonzero((l == 1) & (m == mm))[0])
        for k in range(nr):
            d[k * J + j, 3 * v] = 0.5 * r[k] ** 2
            d[k * J + j, 3 * v + 1] = r[k]
    j20 = int(np.flatnonzero((l == 2) & (m == 0))[0])
    d[j20::J, 9] = 1.0                          # scalar P_2^0: 1 at both poles
    v = b_trans_pole(r, L, l, m, d, 3, 1)
    expect = np.concatenate([np.eye(3).reshape(-1), [1.0]])
    for row in range(2 * nr):
        assert np.abs(v[row] - expect).max() < 1e-14, (row, v[row])


def test_center_oracle_uniform_z_and_scalars_untouched():
    """Centre node (b_trans_center): the uniform field z (S(1,0) = r^2 / 2)
    gives (0, 0, 1); orders -1 / +1 feed components 1 / 2 with the factor -2
    as schmidt_b_trans_center_vect assigns them; scalar entries keep v_in."""
    from oracle.sph_pole import b_trans_center
    L, nr = 4, 3
    radius = np.array([0.2, 0.6, 1.0])
    l, m = rj_order(L)
    J = len(l)
    d = np.zeros((J * nr, 4))
    jz = int(np.flatnonzero((l == 1) & (m == 0))[0])
    for k in range(nr):
        d[k * J + jz, 0] = radius[k] ** 2 / 2
    v = b_trans_center(radius, l, m, d, 1, 1, v_in=[9.0, 9.0, 9.0, 7.5])
    assert np.allclose(v, [0.0, 0.0, 1.0, 7.5], rtol=0, atol=1e-15)
    jm, jp = (int(np.flatnonzero((l == 1) & (m == s))[0]) for s in (-1, 1))
    d2 = np.zeros_like(d)
    d2[jm, 0], d2[jp, 0] = 0.02, -0.04
    v2 = b_trans_center(radius, l, m, d2, 1, 1)
    assert np.allclose(v2[:3], [-2 * 0.02 / 0.04, 2 * 0.04 / 0.04, 0.0], rtol=1e-15, atol=0)
