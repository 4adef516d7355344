"""FP64 tier parity: CUDA path (through the C-ABI) vs the CPU FP64 oracle.

Tolerance: max-norm relative error per field <= 1e-13 (the plain FP64 cycle
must reproduce the reference CPU transform to 1e-13).
"""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, rj_order, PROD_SCALAR
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.oracle import Oracle
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

TOL = 1e-13

CFGS = [
    SphConfig(31, 48, 96, 33, name="L31"),
    SphConfig(47, 73, 144, 6, name="L47_odd_nth"),          # odd N_theta: equator row
    SphConfig(16, 26, 40, 5, nvb=1, nsb=2, nvf=1, nsf=1,     # nph = 40 = 8*5
              products=((1, 0, 1, 0.5), (3, 0, 1, 2.0)), name="L16_mixed"),
    SphConfig(63, 96, 3072, 3, name="L63_wide_nph3072"),    # line too wide for shared memory: pair by pair
]


@pytest.fixture(scope="module", params=CFGS, ids=lambda c: c.name)
def pair(request):
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = request.param
    return cfg, SphTransform(cfg), Oracle(cfg, nthreads=8)


@pytest.mark.gpu
def test_tables_match_oracle(pair):
    cfg, tr, orc = pair
    t = orc.tables()
    l, m = t["l"], t["m"]
    for mm in sorted({0, 1, 2, cfg.ltr // 2, cfg.ltr}):
        colat, w, P, dP = tr.tables(mm)
        assert np.abs(colat - t["colat"]).max() < 1e-15
        assert np.abs(w - t["weight"]).max() <= 1e-15 * np.abs(t["weight"]).max() * 4
        idx = [j for j in range(len(l)) if m[j] == mm]
        Pref = t["P"][idx][:, :cfg.nh]
        dPref = t["dP"][idx][:, :cfg.nh]
        # FMA contraction and sqrt rounding differ between the device and host
        # recurrences, and the difference grows with the number of recurrence
        # steps (~ (L+1) ulps); dP mixes two recurrences and cancels.
        tolP, toldP = 4e-16 * (cfg.ltr + 1), 3e-15 * (cfg.ltr + 1)
        assert np.abs(P - Pref).max() <= tolP * max(1.0, np.abs(Pref).max())
        assert np.abs(dP - dPref).max() <= toldP * max(1.0, np.abs(dPref).max())


@pytest.mark.gpu
def test_b_trans_matches_oracle(pair):
    import torch
    cfg, tr, orc = pair
    d = make_d_rj(cfg, seed=11)
    ref = orc.b_trans(d)
    fld = torch.empty((cfg.ncb, cfg.nr * cfg.nth * cfg.nph), dtype=torch.float64, device="cuda")
    tr.sph_b_trans(to_dev_fortran(d), fld)
    err = col_relerr(from_dev_fortran(fld), ref)
    assert err.max() <= TOL, err


@pytest.mark.gpu
def test_f_trans_matches_oracle(pair):
    import torch
    cfg, tr, orc = pair
    rng = np.random.default_rng(5)
    nnod = cfg.nr * cfg.nth * cfg.nph
    frc = np.asfortranarray(rng.standard_normal((nnod, cfg.ncf)))
    ref = orc.f_trans(frc)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.sph_f_trans(to_dev_fortran(frc), out)
    err = col_relerr(from_dev_fortran(out), ref)
    assert err.max() <= TOL, err


@pytest.mark.gpu
def test_cycle_matches_oracle(pair):
    import torch
    cfg, tr, orc = pair
    d = make_d_rj(cfg, seed=3)
    ref = orc.cycle(d)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    err = col_relerr(from_dev_fortran(out), ref)
    assert err.max() <= TOL, err


@pytest.mark.gpu
def test_cycle_host_pointers(pair):
    cfg, tr, orc = pair
    d = make_d_rj(cfg, seed=4)
    ref = orc.cycle(d)
    out = np.zeros((cfg.J * cfg.nr, cfg.ncf), order="F")
    tr.nonlinear_cycle(d, out)
    assert col_relerr(out, ref).max() <= TOL


@pytest.mark.gpu
def test_custom_rj_order_and_wide_ld():
    """d_rj with a permuted j order and extra columns (ld > J*Nr, cols not contiguous)."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(15, 24, 48, 4, nvb=1, nsb=1, nvf=1, nsf=0,
                    products=((1, 0, 0, 1.0),))
    l, m = rj_order(cfg.ltr)
    perm = np.random.default_rng(0).permutation(cfg.J)
    idx = np.stack([l[perm], m[perm]], 1).reshape(-1)
    tr = SphTransform(cfg, idx_rj_lm=idx)
    orc = Oracle(cfg, nthreads=2)
    d = make_d_rj(cfg, seed=9)
    ref = orc.cycle(d)
    n = cfg.J * cfg.nr
    ld = n + 7
    # permuted input: row j' of block k holds mode perm[j']
    big = np.zeros((ld, 8), order="F")
    for k in range(cfg.nr):
        big[k * cfg.J:(k + 1) * cfg.J, 2:5] = d[k * cfg.J + perm, 0:3]
        big[k * cfg.J:(k + 1) * cfg.J, 6] = d[k * cfg.J + perm, 3]
    out = np.zeros((ld, 5), order="F")
    tr.nonlinear_cycle(big, out, cols_b=[2, 6], cols_f=[1], ld_in=ld, ld_out=ld)
    got = np.zeros((n, 3))
    for k in range(cfg.nr):
        got[k * cfg.J + perm] = out[k * cfg.J:(k + 1) * cfg.J, 1:4]
    assert col_relerr(got, ref[:, 0:3]).max() <= TOL


@pytest.mark.gpu
def test_scalar_product_single_mode():
    """T = P_1^0 -> T^2 = 1/3 + 2/3 P_2^0 through the full GPU cycle."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(8, 12, 24, 3, nvb=0, nsb=1, nvf=0, nsf=1, products=((PROD_SCALAR, 0, 0, 1.0),))
    tr = SphTransform(cfg)
    l, m = rj_order(cfg.ltr)
    J = cfg.J
    d = np.zeros((J * cfg.nr, 1), order="F")
    d[np.where((l == 1) & (m == 0))[0][0] + J * np.arange(cfg.nr), 0] = 1.0
    out = np.zeros_like(d)
    tr.nonlinear_cycle(d, out)
    exp = np.zeros(J)
    exp[np.where((l == 0) & (m == 0))[0][0]] = 1.0 / 3.0
    exp[np.where((l == 2) & (m == 0))[0][0]] = 2.0 / 3.0
    # the reference's Gauss weights carry ~1e-12 relative error (P'_n taken at
    # the previous Newton iterate, gauss_integration.f90:111-116), hence 1e-11
    for k in range(cfg.nr):
        assert np.abs(out[J * k:J * (k + 1), 0] - exp).max() < 1e-11


# Grid/field shapes that select each variant of the fused FFT + products kernel:
# N = 3 (L + 1) (zero band of the spectrum pruned) or a wider grid, the standard
# MHD product list or a generic one, and the other compiled field counts.
# (Nr >= 3: with two radii the synthetic spectra vanish at both ends of the
# shell and the relative error of the degenerate output columns is noise.)
FFT_CFGS = [
    SphConfig(31, 48, 192, 5, name="L31_nph192"),                      # N > 3(L+1): no pruning
    SphConfig(31, 48, 96, 4, products=((0, 0, 1, 0.5), (0, 2, 0, 2.0), (1, 1, 0, -1.0), (2, 2, 2, 1.5)),
              name="L31_generic_products"),                            # generic product code
    SphConfig(63, 96, 192, 3, nvb=2, nsb=1, nvf=2, nsf=1,
              products=((0, 1, 0, 1.0), (1, 0, 0, 1.0), (2, 0, 1, 1.0)), name="L63_2v1s"),
    SphConfig(255, 384, 768, 3, nvb=1, nsb=1, nvf=1, nsf=0, products=((1, 0, 0, 1.0),), name="L255_1v1s"),
    SphConfig(511, 768, 1536, 3, name="L511_Nr3"),                     # the benchmark's angular grid
]


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", FFT_CFGS, ids=lambda c: c.name)
def test_cycle_fft_variants(cfg):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    tr = SphTransform(cfg)
    orc = Oracle(cfg, nthreads=8)
    d = make_d_rj(cfg, seed=13)
    ref = orc.cycle(d)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    err = col_relerr(from_dev_fortran(out), ref)
    assert err.max() <= TOL, err
