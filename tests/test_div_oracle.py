"""CPU checks of the divergence oracle (oracle/sph_div.py): the 3x3 cofactor
inverse, and the radial FDM of the reference being exact for quadratic
radial profiles (interior three-point rows and the fixed-field one-sided
boundary rows), so the divergence of an exactly differentiated quadratic
vanishes and that of S = r^2 with dS/dr = 0 is 2 g3 / r."""
import numpy as np

from kemorin_mhd_b200.config import SphConfig, rj_order
from oracle.sph_div import div_flux, fdm_coefs, inverse33


def test_inverse33_matches_numpy():
    rng = np.random.default_rng(3)
    for _ in range(20):
        a = rng.standard_normal((3, 3)) + 3 * np.eye(3)
        assert np.abs(inverse33(a) - np.linalg.inv(a)).max() < 1e-13


def test_fdm_exact_for_quadratics():
    r = SphConfig(15, 24, 48, 17).radius()
    d1, icb, cmb = fdm_coefs(r)
    for f, df in ((lambda x: 1.0 + 0 * x, lambda x: 0 * x), (lambda x: x, lambda x: 1 + 0 * x),
                  (lambda x: x * x, lambda x: 2 * x)):
        v = f(r)
        for k in range(1, len(r) - 1):
            assert abs(d1[k] @ v[k - 1:k + 2] - df(r[k])) < 1e-11
        assert abs(icb @ v[0:3] - df(r[0])) < 1e-11
        assert abs(cmb @ v[::-1][0:3] - df(r[-1])) < 1e-11


def test_divergence_of_quadratic_profiles():
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    rng = np.random.default_rng(4)
    a, b, c = (rng.standard_normal(cfg.J) for _ in range(3))
    S = np.outer(np.ones_like(r), a) + np.outer(r, b) + np.outer(r * r, c)
    dS = np.outer(np.ones_like(r), b) + np.outer(2 * r, c)
    out = div_flux(r, l, S.reshape(-1), dS.reshape(-1), fix_in=S[0], fix_out=S[-1])
    assert np.abs(out).max() < 1e-9 * np.abs(S).max() * (cfg.ltr + 1) ** 2
    # S = r^2, dS/dr column zero: div = 2 r max(l(l+1), 1/2) / r^2
    S2 = np.outer(r * r, np.ones(cfg.J))
    out2 = div_flux(r, l, S2.reshape(-1), np.zeros(S2.size), fix_in=S2[0], fix_out=S2[-1]).reshape(len(r), -1)
    g3 = np.maximum(np.where(l == 0, 0.5, l * (l + 1.0)), 0.5)
    assert np.abs(out2 - 2.0 * np.outer(1.0 / r, g3)).max() < 1e-10 * g3.max()


def test_rot_uxb_oracle_on_quadratic_profiles():
    """pol = T, dpol/dr = dT/dr, tor = -d(dS/dr)/dr + g3 S / r^2 exactly for
    quadratic radial profiles in the interior; insulating boundary rows."""
    from oracle.sph_div import rot_uxb
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    rng = np.random.default_rng(5)
    a, b, c, e = (rng.standard_normal(cfg.J) for _ in range(4))
    one = np.ones_like(r)
    S = np.outer(one, a) + np.outer(r, b)
    dS = np.outer(one, b) + np.outer(r * r, c)         # d(dS)/dr = 2 c r
    T = np.outer(r * r, e)                              # dT/dr = 2 e r
    pol, dpol, tor = (x.reshape(len(r), -1) for x in rot_uxb(r, l, S.reshape(-1), dS.reshape(-1), T.reshape(-1)))
    g3 = l * (l + 1.0)
    assert np.array_equal(pol, T)
    inner = slice(1, len(r) - 1)
    assert np.abs(dpol[inner] - np.outer(2 * r, e)[inner]).max() < 1e-10
    tor_ref = -np.outer(2 * r, c) + np.outer(1 / r ** 2, g3) * S
    assert np.abs(tor[inner] - tor_ref[inner]).max() < 1e-9 * np.abs(tor_ref).max()
    assert np.allclose(dpol[0], (l + 1.0) / r[0] * T[0]) and np.allclose(dpol[-1], -l / r[-1] * T[-1])
    assert not tor[0].any() and not tor[-1].any()


def _rot_force_case(bc, S, T):
    from oracle.sph_div import rot_force
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    dS = np.zeros_like(S)
    out = rot_force(r, l, S.reshape(-1), dS.reshape(-1), T.reshape(-1), bc, bc)
    g3 = l * (l + 1.0)
    return r, g3, [x.reshape(len(r), -1) for x in out]


def test_rot_force_non_slip_rows_exact_for_quadratics():
    """Non-slip rows assume dS/dr = 0 on the boundary: d2S/dr2 = 2 for
    S = (r - r_b)^2; the one-sided dT/dr is exact for T = r^2."""
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    ones = np.ones(cfg.J)
    T = np.outer(r * r, ones)
    for b in (0, -1):
        S = np.outer((r - r[b]) ** 2, ones)
        _, g3, (pol, dpol, tor) = _rot_force_case("non_slip", S, T)
        assert np.array_equal(pol, T)
        assert np.abs(dpol[b] - 2 * r[b]).max() < 1e-10
        assert np.abs(tor[b] + 2.0).max() < 1e-9


def test_rot_force_free_slip_rows_exact():
    """Free-slip rows: d2S/dr2 exact for S = a r + c r^2 (S extrapolates to 0
    at r = 0), dT/dr = 2 T / r on the boundary (T = r^2 exact)."""
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    ones = np.ones(cfg.J)
    S = np.outer(0.3 * r + 1.7 * r * r, ones)
    T = np.outer(r * r, ones)
    _, g3, (pol, dpol, tor) = _rot_force_case("free_slip", S, T)
    for b in (0, -1):
        assert np.abs(dpol[b] - 2 * r[b]).max() < 1e-10
        ref = -(2 * 1.7 - g3 / r[b] ** 2 * S[b])
        assert np.abs(tor[b] - ref).max() < 1e-9 * np.abs(ref).max()


def test_rot_force_interior_equals_rot_uxb():
    from oracle.sph_div import rot_force, rot_uxb
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    rng = np.random.default_rng(9)
    S, dS, T = (rng.standard_normal(cfg.J * cfg.nr) for _ in range(3))
    a = [x.reshape(cfg.nr, -1)[1:-1] for x in rot_force(r, l, S, dS, T)]
    b = [x.reshape(cfg.nr, -1)[1:-1] for x in rot_uxb(r, l, S, dS, T)]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_div_force_uses_boundary_values():
    from oracle.sph_div import div_force
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    rng = np.random.default_rng(10)
    a, b, c = (rng.standard_normal(cfg.J) for _ in range(3))
    S = np.outer(np.ones_like(r), a) + np.outer(r, b) + np.outer(r * r, c)
    dS = np.outer(np.ones_like(r), b) + np.outer(2 * r, c)
    out = div_force(r, l, S.reshape(-1), dS.reshape(-1))
    assert np.abs(out).max() < 1e-9 * np.abs(S).max() * (cfg.ltr + 1) ** 2


def test_curl_rows_use_zero_g3_at_degree_zero():
    """The curl's g3 is g_sph_rj(j,3) = l(l+1) with no l = 0 override (0 there),
    while the divergence takes max(g3, 1/2): the interior l = 0 toroidal row is
    -d(dS)/dr (the force curl's boundary rows still see S through d2S/dr2)."""
    from oracle.sph_div import rot_force, rot_uxb
    cfg = SphConfig(7, 12, 24, 6)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    j0 = int(np.flatnonzero(l == 0)[0])
    rng = np.random.default_rng(12)
    S, dS, T = (rng.standard_normal(cfg.J * cfg.nr) for _ in range(3))
    S2 = S.reshape(cfg.nr, -1).copy()
    S2[:, j0] += 100.0                                   # the l = 0 S must not matter
    for f in (rot_uxb, rot_force):
        a = f(r, l, S, dS, T)[2].reshape(cfg.nr, -1)
        b = f(r, l, S2.reshape(-1), dS, T)[2].reshape(cfg.nr, -1)
        assert np.array_equal(a[1:-1, j0], b[1:-1, j0])


def test_fixed_flux_rows_take_the_flux():
    """A fixed-flux side gives div = (flux - dS/dr) max(g3, 1/2) / r^2 there,
    whatever S is; the other rows are those of the fixed-field divergence."""
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    rng = np.random.default_rng(14)
    S, dS = rng.standard_normal(cfg.J * cfg.nr), rng.standard_normal(cfg.J * cfg.nr)
    fi, fo = rng.standard_normal(cfg.J), rng.standard_normal(cfg.J)
    a = div_flux(r, l, S, dS, fi, fo, "flux", "flux").reshape(cfg.nr, -1)
    b = div_flux(r, l, S, dS, fi, fo).reshape(cfg.nr, -1)
    g3 = np.maximum(np.where(l == 0, 0.5, l * (l + 1.0)), 0.5)
    d = dS.reshape(cfg.nr, -1)
    assert np.array_equal(a[1:-1], b[1:-1])
    assert np.array_equal(a[0], (fi - d[0]) * g3 * (1.0 / r[0]) ** 2)
    assert np.array_equal(a[-1], (fo - d[-1]) * g3 * (1.0 / r[-1]) ** 2)


def test_pseudo_vacuum_rows():
    from oracle.sph_div import rot_uxb
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    rng = np.random.default_rng(15)
    S, dS, T = (rng.standard_normal(cfg.J * cfg.nr) for _ in range(3))
    pol, dpol, tor = (x.reshape(cfg.nr, -1) for x in rot_uxb(r, l, S, dS, T, "pseudo_vacuum", "pseudo_vacuum"))
    assert np.array_equal(pol, T.reshape(cfg.nr, -1))
    for k in (0, -1):
        assert not dpol[k].any() and not tor[k].any()


def test_vorticity_and_current_exact_cases():
    """Interior: tor = -d2S/dr2 + l(l+1) S / r^2 exactly for quadratic S; an
    insulating outer row is exact for a quadratic S with the potential field's
    slope dS/dr = -l S / r there (inner: (l + 1) S / r)."""
    from oracle.sph_div import current, vorticity
    cfg = SphConfig(15, 24, 48, 9)
    r = cfg.radius()
    l, _ = rj_order(cfg.ltr)
    lf = l.astype(np.float64)
    g3 = lf * (lf + 1.0)
    rng = np.random.default_rng(16)
    a, b, c = (rng.standard_normal(cfg.J) for _ in range(3))
    S = np.outer(np.ones_like(r), a) + np.outer(r, b) + np.outer(r * r, c)
    T = np.zeros_like(S)
    for f in (vorticity, current):
        tor = f(r, l, S.reshape(-1), np.zeros(S.size), T.reshape(-1))[2].reshape(cfg.nr, -1)
        ref = -2.0 * c + g3 * S / r[:, None] ** 2
        assert np.abs(tor[1:-1] - ref[1:-1]).max() < 1e-9 * np.abs(ref).max()
    for side in (0, -1):
        rb = r[side]
        slope = (lf + 1.0) / rb if side == 0 else -lf / rb
        S2 = np.outer(np.ones_like(r), a) + np.outer(r - rb, slope * a) + np.outer((r - rb) ** 2, c)
        tor = current(r, l, S2.reshape(-1), np.zeros(S2.size), T.reshape(-1))[2].reshape(cfg.nr, -1)
        ref = -(2.0 * c - g3 * S2[side] / rb ** 2)
        assert np.abs(tor[side] - ref).max() < 1e-8 * np.abs(ref).max()
