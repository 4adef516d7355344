"""Pins the CPU FP64 oracle (a restatement of the reference's CPU path).

The reference stores no golden vectors for this path and cannot be compiled
here (Fortran 90, no Fortran compiler), so the oracle is pinned by scipy's
independent Gauss nodes / associated Legendre functions and by invariants.
"""
import ctypes

import numpy as np
import pytest
import scipy.special as sp

from oracle import oracle as om
from kemorin_mhd_b200.config import (SphConfig, rj_order, PROD_SCALAR, PROD_CROSS,
                                     PROD_VEC_SCALAR, PROD_DOT)
from kemorin_mhd_b200.synthetic import make_d_rj

CFG = SphConfig(31, 48, 96, 9)


def _refine(o):
    om.lib().oracle_refine_weights.argtypes = [ctypes.c_void_p]
    om.lib().oracle_refine_weights(o._h)


@pytest.fixture(scope="module")
def orc():
    return om.Oracle(CFG, nthreads=4)


def test_gauss_nodes_match_scipy(orc):
    t = orc.tables()
    x, w = sp.roots_legendre(CFG.nth)
    # reference order: first node x ~ -1 (colatitude ~ pi)
    assert np.abs(np.cos(t["colat"]) - x).max() < 1e-15
    # gauss_integration.f90:111-116 forms the weight from P'_n at the previous
    # Newton iterate, so the reference's weights carry ~1e-13 absolute error.
    assert np.abs(t["weight"] - w).max() < 1e-11
    assert abs(t["weight"].sum() - 2.0) < 1e-11


@pytest.mark.parametrize("n", [2, 3, 7, 48, 96])
def test_gauss_exactness_refined(n):
    o = om.Oracle(SphConfig(3, n, 8, 2), nthreads=1)
    _refine(o)
    t = o.tables()
    x = np.cos(t["colat"])
    for k in range(0, 2 * n):
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs((t["weight"] * x ** k).sum() - exact) < 5e-15 * max(1, n)


def test_schmidt_matches_scipy(orc):
    t = orc.tables()
    x = np.cos(t["colat"])
    for j in range(orc.J):
        l, m = int(t["l"][j]), abs(int(t["m"][j]))
        ref = sp.lpmv(m, l, x) * (-1) ** m
        if m > 0:
            ref = ref * np.sqrt(2.0 * sp.factorial(l - m) / sp.factorial(l + m))
        assert np.abs(ref - t["P"][j]).max() < 2e-14, (l, m)


def test_dpdtheta_matches_recurrence(orc):
    t = orc.tables()
    th = t["colat"]
    x = np.cos(th)
    for j in range(orc.J):
        l, m = int(t["l"][j]), abs(int(t["m"][j]))
        if l == 0:
            continue
        # (x^2-1) dP_l^m/dx = l x P_l^m - (l+m) P_{l-1}^m ; dP/dtheta = -sin(theta) dP/dx
        Pl = sp.lpmv(m, l, x)
        Pl1 = sp.lpmv(m, l - 1, x) if l - 1 >= m else 0.0 * x
        dPdx = (l * x * Pl - (l + m) * Pl1) / (x * x - 1.0)
        ref = -np.sin(th) * dPdx * (-1) ** m
        if m > 0:
            ref = ref * np.sqrt(2.0 * sp.factorial(l - m) / sp.factorial(l + m))
        assert np.abs(ref - t["dP"][j]).max() < 1e-13 * max(1.0, np.abs(ref).max()), (l, m)


def test_schmidt_orthogonality_refined():
    o = om.Oracle(CFG, nthreads=2)
    _refine(o)
    t = o.tables()
    for m in range(0, CFG.ltr + 1, 5):
        idx = [j for j in range(o.J) if t["m"][j] == m]
        P = t["P"][idx]
        G = (P * t["weight"][None, :]) @ P.T
        ls = t["l"][idx]
        norm = (2.0 if m == 0 else 4.0) / (2 * ls + 1)
        assert np.abs(G - np.diag(norm)).max() < 1e-14


def test_roundtrip_refined_weights():
    o = om.Oracle(CFG, nthreads=4)
    _refine(o)
    d = make_d_rj(CFG, seed=7)
    back = o.f_trans(o.b_trans(d))
    for c in range(CFG.ncb):
        assert np.abs(back[:, c] - d[:, c]).max() <= 1e-13 * np.abs(d[:, c]).max()


def test_roundtrip_reference_weights(orc):
    # the reference's weight error (~1e-12 relative) bounds its own round trip
    d = make_d_rj(CFG, seed=7)
    back = orc.f_trans(orc.b_trans(d))
    for c in range(CFG.ncb):
        assert np.abs(back[:, c] - d[:, c]).max() <= 1e-10 * np.abs(d[:, c]).max()


def _grid(o, f, c):
    cfg = o.cfg
    return f[:, c].reshape(cfg.nph, cfg.nth, cfg.nr)


@pytest.mark.parametrize("lm,fn", [
    ((1, 0), lambda T, P: np.cos(T)),
    ((1, 1), lambda T, P: np.sin(T) * np.cos(P)),
    ((1, -1), lambda T, P: np.sin(T) * np.sin(P)),
    ((2, 2), lambda T, P: np.sqrt(3) / 2 * np.sin(T) ** 2 * np.cos(2 * P)),
    ((3, -2), lambda T, P: np.sqrt(15) / 2 * np.cos(T) * np.sin(T) ** 2 * np.sin(2 * P)),
])
def test_analytic_scalar_modes(orc, lm, fn):
    l, m = rj_order(CFG.ltr)
    J = CFG.J
    d = np.zeros((J * CFG.nr, CFG.ncb), order="F")
    j = np.where((l == lm[0]) & (m == lm[1]))[0][0]
    d[j + J * np.arange(CFG.nr), 9] = 1.0
    g = _grid(orc, orc.b_trans(d), 9)
    t = orc.tables()
    T, P = np.meshgrid(t["colat"], 2 * np.pi * np.arange(CFG.nph) / CFG.nph)
    for k in range(CFG.nr):
        assert np.abs(g[:, :, k] - fn(T, P)).max() < 1e-14


def test_analytic_vector_mode(orc):
    l, m = rj_order(CFG.ltr)
    J = CFG.J
    d = np.zeros((J * CFG.nr, CFG.ncb), order="F")
    j = np.where((l == 1) & (m == 1))[0][0]
    kk = J * np.arange(CFG.nr)
    d[j + kk, 0], d[j + kk, 1], d[j + kk, 2] = 1.0, 0.5, 0.25
    f = orc.b_trans(d)
    t = orc.tables()
    T, P = np.meshgrid(t["colat"], 2 * np.pi * np.arange(CFG.nph) / CFG.nph)
    r = CFG.radius()
    for k in range(CFG.nr):
        ur, ut, up = (_grid(orc, f, c)[:, :, k] for c in range(3))
        # S Y with Y = sin(theta) cos(phi): u_r = 2 S Y / r^2,
        # u_theta = dS/r dY/dtheta + T/(r sin) dY/dphi, u_phi = dS/(r sin) dY/dphi - T/r dY/dtheta
        assert np.abs(ur - 2 * np.sin(T) * np.cos(P) / r[k] ** 2).max() < 1e-13
        assert np.abs(ut - (0.5 * np.cos(T) * np.cos(P) - 0.25 * np.sin(P)) / r[k]).max() < 1e-13
        assert np.abs(up - (-0.5 * np.sin(P) - 0.25 * np.cos(T) * np.cos(P)) / r[k]).max() < 1e-13


def test_scalar_product_spectrum():
    # T = P_1^0 = cos(theta): T^2 = 1/3 + (2/3) P_2^0
    cfg = SphConfig(8, 12, 24, 3, nvb=0, nsb=1, nvf=0, nsf=1,
                    products=((PROD_SCALAR, 0, 0, 1.0),))
    o = om.Oracle(cfg, nthreads=1)
    _refine(o)
    l, m = rj_order(cfg.ltr)
    J = cfg.J
    d = np.zeros((J * cfg.nr, 1), order="F")
    j1 = np.where((l == 1) & (m == 0))[0][0]
    d[j1 + J * np.arange(cfg.nr), 0] = 1.0
    out = o.cycle(d)
    exp = np.zeros(J)
    exp[np.where((l == 0) & (m == 0))[0][0]] = 1.0 / 3.0
    exp[np.where((l == 2) & (m == 0))[0][0]] = 2.0 / 3.0
    for k in range(cfg.nr):
        assert np.abs(out[J * k:J * (k + 1), 0] - exp).max() < 1e-14


def test_cycle_products_layout():
    # cycle == f_trans(products(b_trans)) evaluated with numpy products
    cfg = SphConfig(15, 24, 48, 4)
    o = om.Oracle(cfg, nthreads=2)
    d = make_d_rj(cfg, seed=3)
    f = o.b_trans(d)
    u, w, b, T = f[:, 0:3], f[:, 3:6], f[:, 6:9], f[:, 9]
    frc = np.zeros((f.shape[0], 10), order="F")
    frc[:, 0:3] = np.cross(w, u)
    frc[:, 3:6] = np.cross(u, b)
    frc[:, 6:9] = u * T[:, None]
    frc[:, 9] = (u * w).sum(1)
    ref = o.f_trans(frc)
    out = o.cycle(d)
    assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max()
