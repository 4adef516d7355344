"""CPU oracle (test infrastructure only) of the backward transform at the
poles, for grids with pole points: schmidt_b_trans_pole_vect and
schmidt_b_trans_pole_scalar (PARALLEL_src/SPH_SHELL_src/schmidt_b_trans_at_pole.f90:88-289),
driven by pole_backward_transforms (pole_sph_transform.f90:107-162).

Per radius k, rows k (north pole) and nr + k (south pole) of v_pole
(2 nr x ncomp), summed over l in the reference's loop order:
- scalar: sum_l s(l, 0) P_l^0(+-1);
- vector component 3 (z): +-sum_l S(l, 0) P_l^0(+-1) g3(l), times 1/r^2;
- components 1, 2 (x, y) from the orders -1 ("1s") and +1 ("1c"):
    north  x += T(l,-1) dP,  y += dS(l,-1) dP;   x += dS(l,1) dP,  y -= T(l,1) dP
    south  x += T(l,-1) dP', y -= dS(l,-1) dP';  x -= dS(l,1) dP', y -= T(l,1) dP'
  times 1/r;
with the Schmidt values at the poles (set_lagender_pole_rlm,
CORE_src/SPH_SPECTR_src/schmidt_poly_on_rtm_grid.f90:201-266, evaluated there
by the recurrence at theta = 0 and pi) in closed form: P_l^0(1) = 1,
P_l^0(-1) = (-1)^l, dP_l^1/dtheta = sqrt(l(l+1)/2) at the north pole and
(-1)^l sqrt(l(l+1)/2) at the south pole (dP_l^1/dtheta = (sqrt(2l(l+1)) P_l^0
- sqrt((l-1)(l+2)) P_l^2) / 2 with P_l^2 = 0 at the poles); g3 = g_sph_rlm(j,3)
= l(l+1), 1/2 at l = 0.

The centre node of a full-sphere grid (b_trans_center) follows
schmidt_b_trans_center_vect / _scalar (schmidt_b_trans_at_center.f90:45-119):
from the innermost radius r_1, vector components (1, 2, 3) =
(-2 S(1,-1), -2 S(1,+1), 2 S(1,0)) / r_1^2 -- the pairing of the code, whose
header comment names the opposite one -- and scalar entries unchanged.

Parity unpinned against the reference's own outputs (no Fortran compiler in
this image); the tests pin the sign conventions by the uniform fields x, y, z
(poloidal l = 1 fields with S = r^2/2) and the pole values by quadrature.
"""
import numpy as np


def pole_values(l):
    """(P north, P south, dP/dtheta north, dP/dtheta south) of degree l for m = 0 / 1."""
    l = np.asarray(l, dtype=np.float64)
    sgn = np.where(np.asarray(l, dtype=np.int64) % 2 == 1, -1.0, 1.0)
    dp = np.sqrt(0.5 * l * (l + 1.0))
    return np.ones_like(l), sgn, dp, sgn * dp


def b_trans_pole(radius, L, l_of_j, m_of_j, d_rj, nvb, nsb):
    """v_pole (2 nr x (3 nvb + nsb)) from d_rj (J*nr x ncomp, vectors (S, dS/dr, T) first)."""
    r = np.asarray(radius, dtype=np.float64)
    nr, J = len(r), len(l_of_j)
    idx = {(int(a), int(b)): j for j, (a, b) in enumerate(zip(l_of_j, m_of_j))}
    ncomp = 3 * nvb + nsb
    dr = np.asarray(d_rj, dtype=np.float64)
    v = np.zeros((2 * nr, ncomp))
    for k in range(nr):
        ar = 1.0 / r[k]
        row = lambda c, l, m: dr[k * J + idx[(l, m)], c]  # noqa: E731
        for nd in range(nvb):
            cS, cD, cT = 3 * nd, 3 * nd + 1, 3 * nd + 2
            zn = zs = xn = yn = xs = ys = 0.0
            for l in range(0, L + 1):
                pn, ps, _, _ = pole_values(l)
                g3 = 0.5 if l == 0 else float(l * (l + 1))
                zn = zn + row(cS, l, 0) * pn * g3
                zs = zs - row(cS, l, 0) * ps * g3
            for l in range(1, L + 1):
                _, _, dpn, dps = pole_values(l)
                xn = xn + row(cT, l, -1) * dpn
                yn = yn + row(cD, l, -1) * dpn
                xs = xs + row(cT, l, -1) * dps
                ys = ys - row(cD, l, -1) * dps
            for l in range(1, L + 1):
                _, _, dpn, dps = pole_values(l)
                xn = xn + row(cD, l, 1) * dpn
                yn = yn - row(cT, l, 1) * dpn
                xs = xs - row(cD, l, 1) * dps
                ys = ys - row(cT, l, 1) * dps
            v[k, cS:cS + 3] = xn * ar, yn * ar, zn * ar * ar
            v[nr + k, cS:cS + 3] = xs * ar, ys * ar, zs * ar * ar
        for q in range(nsb):
            c = 3 * nvb + q
            sn = ss = 0.0
            for l in range(0, L + 1):
                pn, ps, _, _ = pole_values(l)
                sn = sn + row(c, l, 0) * pn
                ss = ss + row(c, l, 0) * ps
            v[k, c], v[nr + k, c] = sn, ss
    return v


def b_trans_center(radius, l_of_j, m_of_j, d_rj, nvb, nsb, v_in=None):
    """The centre node's components (3 nvb + nsb) from the innermost radius of
    d_rj (J*nr x ncomp); scalar entries are copied from v_in (zeros if None)."""
    r1 = float(np.asarray(radius, dtype=np.float64)[0])
    idx = {(int(a), int(b)): j for j, (a, b) in enumerate(zip(l_of_j, m_of_j))}
    dr = np.asarray(d_rj, dtype=np.float64)
    v = np.zeros(3 * nvb + nsb) if v_in is None else np.array(v_in, dtype=np.float64)
    for nd in range(nvb):
        c = 3 * nd
        v[c] = -2.0 * dr[idx[(1, -1)], c] * (1.0 / r1) * (1.0 / r1)
        v[c + 1] = -2.0 * dr[idx[(1, 1)], c] * (1.0 / r1) * (1.0 / r1)
        v[c + 2] = 2.0 * dr[idx[(1, 0)], c] * (1.0 / r1) * (1.0 / r1)
    return v
