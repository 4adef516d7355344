"""FP64 tier with P_l^m generated inside the Legendre kernels (on-the-fly P).

With KMHD_FLAG_P_ON_THE_FLY the handle stores no P / dP tables: the DMMA
kernels run the fixed-order Schmidt recurrence (orders m - 1, m, m + 1 for
dP) in generator warps, from per-order coefficients, start values and seeds
every 64 degrees.  The generated values are the stored tables' up to rounding
(sin^m is carried through the recurrence instead of multiplied in at every
degree), so the tier keeps the FP64 tolerance against the oracle: max-norm
relative error per field <= 1e-13.
"""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.oracle import Oracle
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

TOL = 1e-13

CFGS = [
    SphConfig(31, 48, 96, 9, name="L31"),
    SphConfig(47, 73, 144, 6, name="L47_odd_nth"),
    SphConfig(16, 26, 40, 5, nvb=1, nsb=2, nvf=1, nsf=1,
              products=((1, 0, 1, 0.5), (3, 0, 1, 2.0)), name="L16_mixed"),
    SphConfig(127, 192, 384, 5, name="L127"),
]


def table_tol(L):
    """Bounds on |P_otf - P_ref| (relative to max |P|, |dP|): the fixed-order
    recurrence is marginally stable near the poles, where a rounding error of
    step l grows linearly over the later steps, so two recurrences with
    different rounding (sin^m carried through the recurrence here, multiplied
    in at every degree by the stored tables and the oracle) drift apart like
    (L+1)^2 ulps; measured 1.05e-13 at L=127, m=0."""
    return 1.6e-17 * (L + 1) ** 2, 3.2e-17 * (L + 1) ** 2


@pytest.fixture(scope="module", params=CFGS, ids=lambda c: c.name)
def pair(request):
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = request.param
    return cfg, SphTransform(cfg, p_on_the_fly=True), Oracle(cfg, nthreads=8)


@pytest.mark.gpu
def test_otf_tables_match_oracle(pair):
    cfg, tr, orc = pair
    t = orc.tables()
    l, m = t["l"], t["m"]
    for mm in sorted({0, 1, 2, 3, cfg.ltr // 2, cfg.ltr - 1, cfg.ltr}):
        _, _, P, dP = tr.tables(mm)
        idx = [j for j in range(len(l)) if m[j] == mm]
        Pref = t["P"][idx][:, :cfg.nh]
        dPref = t["dP"][idx][:, :cfg.nh]
        tolP, toldP = table_tol(cfg.ltr)
        assert np.abs(P - Pref).max() <= tolP * max(1.0, np.abs(Pref).max()), mm
        assert np.abs(dP - dPref).max() <= toldP * max(1.0, np.abs(dPref).max()), mm


@pytest.mark.gpu
def test_otf_b_trans_matches_oracle(pair):
    import torch
    cfg, tr, orc = pair
    d = make_d_rj(cfg, seed=41)
    ref = orc.b_trans(d)
    fld = torch.empty((cfg.ncb, cfg.nr * cfg.nth * cfg.nph), dtype=torch.float64, device="cuda")
    tr.sph_b_trans(to_dev_fortran(d), fld)
    assert col_relerr(from_dev_fortran(fld), ref).max() <= TOL


@pytest.mark.gpu
def test_otf_f_trans_matches_oracle(pair):
    import torch
    cfg, tr, orc = pair
    rng = np.random.default_rng(42)
    frc = np.asfortranarray(rng.standard_normal((cfg.nr * cfg.nth * cfg.nph, cfg.ncf)))
    ref = orc.f_trans(frc)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.sph_f_trans(to_dev_fortran(frc), out)
    assert col_relerr(from_dev_fortran(out), ref).max() <= TOL


@pytest.mark.gpu
def test_otf_cycle_matches_oracle(pair):
    import torch
    cfg, tr, orc = pair
    d = make_d_rj(cfg, seed=43)
    ref = orc.cycle(d)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    assert col_relerr(from_dev_fortran(out), ref).max() <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [SphConfig(511, 768, 1536, 3, name="L511_Nr3"),
                                 SphConfig(1023, 1536, 3072, 3, name="L1023_Nr3")],
                         ids=lambda c: c.name)
def test_otf_vs_stored_tables_large_L(cfg):
    """At the benchmark grids (the CPU oracle needs minutes there): on-the-fly
    against the stored-table FP64 tier on the same input, and the generated P
    of the highest orders (longest start-value products) against the stored."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    d = to_dev_fortran(make_d_rj(cfg, seed=44))
    outs, tabs = [], []
    for otf in (False, True):
        tr = SphTransform(cfg, p_on_the_fly=otf)
        out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
        tr.nonlinear_cycle(d, out)
        outs.append(from_dev_fortran(out))
        tabs.append([tr.tables(mm)[2:] for mm in (0, 1, cfg.ltr // 2, cfg.ltr)])
        tr.close()
    assert col_relerr(outs[1], outs[0]).max() <= TOL
    tolP, toldP = table_tol(cfg.ltr)
    for (P0, dP0), (P1, dP1) in zip(tabs[0], tabs[1]):
        assert np.abs(P1 - P0).max() <= tolP * max(1.0, np.abs(P0).max())
        assert np.abs(dP1 - dP0).max() <= toldP * max(1.0, np.abs(dP0).max())
