"""CPU oracle (test infrastructure only) of the curl of the Coriolis term in
spectral space, as the reference evaluates it from the backward transform's
velocity and vorticity spectra before the forward transform returns.

Restates, in exact rational arithmetic where the reference counts primes:
- gs_prime (CORE_src/spherical_harmonics/normgi_by_primes.f90:86-196): the
  Schmidt-normalised Gaunt integral
      gs = (-1)^(s-l2-m3) 2 sqrt(2)^(#nonzero m) sqrt(GSI) GI sum_t (-1)^t TI(t),
      s = (l1+l2+l3)/2,
      GI = (2s-2l3)! s! / ((s-l1)! (s-l2)! (s-l3)! (2s+1)!),
      GSI = (l1-m1)! (l2+m2)! (l3+m3)! (l3-m3)! / ((l1+m1)! (l2-m2)!),
      TI(t) = (l1+m1+t)! (l2+l3-m1-t)! / ((l1-m1-t)! (l2-l3+m1+t)! (l3-m3-t)! t!),
      t from max(l3-l2-m1, -l1-m1, 0) to min(l1-m1, l3-m3, l2+l3-m1)
  (the reference multiplies sqrt(p^e) over prime powers in floating point;
  here the square root is taken once of the exact rational, so values agree
  to rounding);
- leadki / leadli / normki / normli (cal_gaunt_itgs.f90), setei / leades
  (normei.f90): the Adams-Gaunt and Elsasser integrals;
- cal_gaunt_coriolis_rlm and interact_rot_coriolis_rlm
  (MHD_src/sph_MHD/interact_coriolis_rlm.f90): the coupled modes (l-1, m),
  (l+1, m), (l, -m) of each mode and the sw / tw coefficients;
- g_sph_rlm columns 3, 4, 5, 17 (spherical_harmonics.f90:91-140 with the l = 0
  override of g(j,3) = 1/2 in copy_sph_normalization_2_rlm,
  schmidt_poly_on_rtm_grid.f90:89-113);
- the rotation spectrum of a unit z rotation, (r^2/2, r, 1)
  (set_rotation_spectr, t_poloidal_rotation.f90);
- sum_rot_coriolis_rlm_10 (MHD_src/sph_MHD/sum_coriolis_terms_rlm.f90:94-189).

Parity unpinned against the reference's own outputs (no Fortran compiler in
this image); the Gaunt integrals are pinned by their defining integrals
evaluated by Gauss-Legendre quadrature in the tests.
"""
from fractions import Fraction
from math import factorial, isqrt

import numpy as np


def _f(n):
    return factorial(n)


def _signed_sqrt_of(sign, q, bits=160):
    """sign * sqrt(q) for a non-negative Fraction q, correctly rounded to well
    beyond double precision."""
    if q == 0:
        return 0.0
    num = q.numerator << (2 * bits)
    root = isqrt(num // q.denominator)
    return sign * (root / (1 << bits))


def gs(m1, l1, m2, l2, m3, l3):
    """Schmidt-normalised Gaunt integral (gs_prime), exact up to the last rounding."""
    s = (l1 + l2 + l3) // 2
    gi = Fraction(_f(2 * s - 2 * l3) * _f(s), _f(s - l1) * _f(s - l2) * _f(s - l3) * _f(2 * s + 1))
    gsi = Fraction(_f(l1 - m1) * _f(l2 + m2) * _f(l3 + m3) * _f(l3 - m3), _f(l1 + m1) * _f(l2 - m2))
    tmax = min(l1 - m1, l3 - m3, l2 + l3 - m1)
    tmin = -min(l2 - l3 + m1, l1 + m1, 0)
    tsum = Fraction(0)
    for t in range(tmin, tmax + 1):
        ti = Fraction(_f(l1 + m1 + t) * _f(l2 + l3 - m1 - t),
                      _f(l1 - m1 - t) * _f(l2 - l3 + m1 + t) * _f(l3 - m3 - t) * _f(t))
        tsum += (-1) ** t * ti
    x = 2 * gi * tsum * (-1) ** ((s - l2 - m3) % 2)
    nz = (m1 != 0) + (m2 != 0) + (m3 != 0)
    q = x * x * gsi * 2 ** nz
    return _signed_sqrt_of(1 if x >= 0 else -1, q)


def _normki(g, m1, m2, m3):
    if m1 * m2 * m3 > 0:
        return -g * 0.5 if (m2 < 0 and m3 < 0) else g * 0.5
    if m2 == 0 and m1 * m3 > 0:
        return g
    if m3 == 0 and m2 * m1 > 0:
        return g
    if m3 == 0 and m2 == 0 and m1 == 0:
        return 2.0 * g
    return 0.0


def _normli(e, m1, m2, m3, mm1):
    if m1 * m2 * m3 < 0:
        return e * 0.5 if (m3 > 0 and m2 > 0) else -e * 0.5
    if m2 == 0 and m1 * m3 < 0:
        return -float(int(m1 / mm1)) * e
    if m3 == 0 and m2 * m1 < 0:
        return -float(int(m1 / mm1)) * e
    return 0.0


def _triangle(l1, l2, l3):
    return l1 + l2 >= l3 and l2 + l3 >= l1 and l3 + l1 >= l2


def _m_match(m1, m2, m3):
    return 0 in (m1 + m2 + m3, m1 + m2 - m3, m1 - m2 + m3, -m1 + m2 + m3)


def leadki(l1, m1, l2, m2, l3, m3):
    """Adams-Gaunt integral K (cal_gaunt_itgs.f90, leadki)."""
    if not _triangle(l1, l2, l3) or (l1 + l2 + l3) % 2 != 0 or not _m_match(m1, m2, m3):
        return 0.0
    a1, a2, a3 = abs(m1), abs(m2), abs(m3)
    if a1 == a2 + a3:
        return _normki(gs(a1, l1, a2, l2, a3, l3), m1, m2, m3)
    if a2 == a1 + a3:
        return _normki(gs(a2, l2, a1, l1, a3, l3), m2, m1, m3)
    if a3 == a2 + a1:
        return _normki(gs(a3, l3, a2, l2, a1, l1), m3, m2, m1)
    return 0.0


def _leades(m2, l2, m3, l3, gg):
    a1 = float((l2 + m2) * (l3 - m3))
    a2 = float((l3 + m3) * (l2 - m2))
    a3 = float((l2 + m2 - 1) * (l3 + m3 + 1))
    a4 = float((l3 + m3 - 1) * (l2 + m2 + 1))
    a5 = float((l2 - m2) * (l3 - m3))
    if m2 - 1 == 0:
        a3 *= 2.0
    if m3 == 0:
        a3 *= 0.5
        a4 *= 0.5
    if m2 == 0:
        a3 *= 0.5
        a4 *= 0.5
    if m3 - 1 == 0:
        a4 *= 2.0
    sq = np.sqrt
    return -(sq(a1) * (sq(a3) * gg[0] + sq(a5) * gg[1]) - sq(a2) * (sq(a4) * gg[2] + sq(a5) * gg[3])) * 0.5


def setei(l1, m1, l2, m2, l3, m3):
    """Elsasser integral with m1 = m2 + m3 (normei.f90, setei)."""
    if l2 == l3 and m2 == m3:
        return 0.0
    gg = [0.0] * 4
    if (m3 + 1) > l3 or abs(m2 - 1) > (l2 - 1):
        gg[0] = 0.0
    elif m2 == 0:
        gg[0] = -gs(m3 + 1, l3, 1, l2 - 1, m1, l1)
    else:
        gg[0] = gs(m1, l1, m2 - 1, l2 - 1, m3 + 1, l3)
    gg[1] = 0.0 if m2 > l2 - 1 else gs(m1, l1, m2, l2 - 1, m3, l3)
    if (m2 + 1) > l2 or abs(m3 - 1) > (l3 - 1):
        gg[2] = 0.0
    elif m3 == 0:
        gg[2] = -gs(m2 + 1, l2, 1, l3 - 1, m1, l1)
    else:
        gg[2] = gs(m1, l1, m2 + 1, l2, m3 - 1, l3 - 1)
    gg[3] = 0.0 if m3 > l3 - 1 else gs(m1, l1, m2, l2, m3, l3 - 1)
    return _leades(m2, l2, m3, l3, gg)


def leadli(l1, m1, l2, m2, l3, m3):
    """Elsasser integral L (cal_gaunt_itgs.f90, leadli)."""
    if not _triangle(l1, l2, l3) or (l1 + l2 + l3) % 2 != 1 or not _m_match(m1, m2, m3):
        return 0.0
    a1, a2, a3 = abs(m1), abs(m2), abs(m3)
    if a1 == a2 + a3:
        return _normli(setei(l1, a1, l2, a2, l3, a3), m1, m2, m3, a1)
    if a2 == a1 + a3:
        return -_normli(setei(l2, a2, l1, a1, l3, a3), m2, m1, m3, a2)
    if a3 == a2 + a1:
        return -_normli(setei(l3, a3, l2, a2, l1, a1), m3, m2, m1, a3)
    return 0.0


def g_rlm(l, m):
    """g_sph_rlm(j, 3), (j, 4), (j, 5), (j, 17) of mode (l, m)."""
    if l == 0 and m == 0:
        return 0.5, 0.0, 2.0, 0.0
    return float(l * (l + 1)), float((l - 1) * l), float((l + 1) * (l + 2)), float(2 * l + 1) / float(4 * l * (l + 1))


def gaunt_coriolis(L, l_of_j, m_of_j):
    """cal_gaunt_coriolis_rlm: per mode j the coupled mode indices (jgi1, jgi2,
    jei) -- (l-1, m), (l+1, m), (l, -m), or j itself where that mode does not
    exist -- and the integrals gi1, gi2, ei."""
    idx = {(int(l), int(m)): j for j, (l, m) in enumerate(zip(l_of_j, m_of_j))}
    J = len(l_of_j)
    jg = np.zeros((J, 3), dtype=np.int64)
    gi = np.zeros((J, 3))
    for j in range(J):
        l3, m3 = int(l_of_j[j]), int(m_of_j[j])
        k1 = k2 = (l3, m3)
        g1 = g2 = e1 = 0.0
        l2 = l3 - 1
        if 1 <= l2 <= L and abs(m3) <= l2:
            g1, k1 = leadki(1, 0, l2, m3, l3, m3), (l2, m3)
        l2 = l3 + 1
        if 1 <= l2 <= L and abs(m3) <= l2:
            g2, k2 = leadki(1, 0, l2, m3, l3, m3), (l2, m3)
        ke = (0, 0)
        if l3 >= 1:
            e1, ke = leadli(1, 0, l3, -m3, l3, m3), (l3, -m3)
        if l3 * (l3 + 1) + m3 == 0:
            k1 = k2 = ke = (0, 0)
            g2 = e1 = 0.0
        jg[j] = idx[k1], idx[k2], idx[ke]
        gi[j] = g1, g2, e1
    return jg, gi


def interact_rot(l_of_j, m_of_j, gi):
    """interact_rot_coriolis_rlm: sw(2,3,j) and tw(2,4,j) (0-based here)."""
    J = len(l_of_j)
    sw = np.zeros((J, 2, 3))
    tw = np.zeros((J, 2, 4))
    for j in range(J):
        g3, g4, g5, g17 = g_rlm(int(l_of_j[j]), int(m_of_j[j]))
        g1, g2, e1 = gi[j]
        sw[j, 0, 0] = (2.0 - g4 - g3) * g1 * g17
        sw[j, 1, 0] = (2.0 - g5 - g3) * g2 * g17
        sw[j, 0, 1] = g4 * (2.0 - g4 + g3) * g1 * g17 * 0.5
        sw[j, 1, 1] = g5 * (2.0 - g5 + g3) * g2 * g17 * 0.5
        sw[j, 0, 2] = 2.0 * e1 * g17
        tw[j, 0, 2] = -(g3 * (2.0 + g4 - g3) + 2.0 * (-2.0 + g4 + g3)) * g1 * g17 * 0.5
        tw[j, 1, 2] = -(g3 * (2.0 + g5 - g3) + 2.0 * (-2.0 + g5 + g3)) * g2 * g17 * 0.5
        tw[j, 0, 3] = -(-2.0 + g4 + g3) * g1 * g17
        tw[j, 1, 3] = -(-2.0 + g5 + g3) * g2 * g17
        tw[j, 0, 0] = -2.0 * e1 * g17
        tw[j, 0, 1] = -g3 * e1 * g17
    return sw, tw


def rot_coriolis(radius, L, l_of_j, m_of_j, velo, vort, coef_cor):
    """Curl of the Coriolis term (pol, tor), each J*Nr with j fastest, from the
    velocity and vorticity spectra velo = (S, dS/dr, T), vort = (S, dS/dr, T),
    as sum_rot_coriolis_rlm_10 with a unit z rotation."""
    r = np.asarray(radius, dtype=np.float64)
    nr, J = len(r), len(l_of_j)
    jg, gi = gaunt_coriolis(L, l_of_j, m_of_j)
    sw, tw = interact_rot(l_of_j, m_of_j, gi)
    vS, vdS, vT = (np.asarray(x).reshape(nr, J) for x in velo)
    wS, wdS, wT = (np.asarray(x).reshape(nr, J) for x in vort)
    g3 = np.array([g_rlm(int(l), int(m))[0] for l, m in zip(l_of_j, m_of_j)])
    k1, k2, ke = jg[:, 0], jg[:, 1], jg[:, 2]
    pol = np.zeros((nr, J))
    tor = np.zeros((nr, J))
    for k in range(nr):
        ar = 1.0 / r[k]
        w0, w1, w2 = 0.5 * 1.0 * r[k] ** 2, 1.0 * r[k], 1.0
        dvp1, dvp2 = vdS[k, k1], vdS[k, k2]
        wp_l1 = wS[k, ke]
        vp1, vp2 = vS[k, k1], vS[k, k2]
        d2vp_l1 = ar * ar * g3 * vS[k, ke] - wT[k, ke]
        vp_l1 = vS[k, ke]
        wp1, wp2 = wS[k, k1], wS[k, k2]
        dwp1 = wdS[k, k1] - 2.0 * ar * wS[k, k1]
        dwp2 = wdS[k, k2] - 2.0 * ar * wS[k, k2]
        p = (sw[:, 0, 0] * w0 * dvp1 + sw[:, 1, 0] * w0 * dvp2 + sw[:, 0, 2] * w0 * wp_l1
             + sw[:, 0, 1] * w1 * vp1 + sw[:, 1, 1] * w1 * vp2)
        t = (tw[:, 0, 0] * w0 * d2vp_l1 - tw[:, 0, 1] * w2 * vp_l1 + tw[:, 0, 2] * w1 * wp1
             + tw[:, 1, 2] * w1 * wp2 + tw[:, 0, 3] * w0 * dwp1 + tw[:, 1, 3] * w0 * dwp2)
        pol[k] = -coef_cor * p * ar * ar
        tor[k] = -coef_cor * t * ar * ar
    return pol.reshape(-1), tor.reshape(-1)
