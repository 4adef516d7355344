"""The split path's slice-product count and the autotuner that picks it.

A split-tier handle runs 26 slice products per Legendre GEMM (digit pairs
a + b <= 6 of six INT8 digits per operand) or, pinned or autotuned, 21 (the
highest group dropped); fp32acc 10 or 6.  The autotuner (KMHD_FLAG_AUTOTUNE,
first batch call) times the FP64 path and both split candidates on the call's
data, measures each split candidate's error against the FP64 path and keeps
the fastest candidate within a quarter of the tier's bound.
"""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_SPLIT_I8, TIER_FP32ACC
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.oracle import Oracle
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

BOUND = {TIER_SPLIT_I8: 1e-12, TIER_FP32ACC: 1e-6}
FULL = {TIER_SPLIT_I8: 26, TIER_FP32ACC: 10}
REDUCED = {TIER_SPLIT_I8: 21, TIER_FP32ACC: 6}


def _cycle(tr, cfg, d):
    import torch
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    return from_dev_fortran(out)


@pytest.mark.gpu
@pytest.mark.parametrize("tier", [TIER_SPLIT_I8, TIER_FP32ACC])
@pytest.mark.parametrize("cfg", [SphConfig(31, 48, 96, 9, name="L31"), SphConfig(127, 192, 384, 5, name="L127")],
                         ids=lambda c: c.name)
def test_pinned_products_vs_oracle(tier, cfg):
    """Both product counts against the oracle: the full count within the
    tier's bound, the reduced count within 256 times it (one base-256 digit
    group fewer), and the two runs differ."""
    from kemorin_mhd_b200.sph_trans import SphTransform
    d = make_d_rj(cfg, seed=91)
    ref = Oracle(cfg, nthreads=8).cycle(d)
    tr = SphTransform(cfg, tier=tier)
    assert tr.tuning()["products"] == FULL[tier]
    full = _cycle(tr, cfg, d)
    assert col_relerr(full, ref).max() <= BOUND[tier]
    tr.set_products(REDUCED[tier])
    assert tr.tuning()["products"] == REDUCED[tier]
    red = _cycle(tr, cfg, d)
    err = col_relerr(red, ref).max()
    assert err <= 256 * BOUND[tier], err
    assert not np.array_equal(red, full)
    tr.set_products(FULL[tier])
    assert np.array_equal(_cycle(tr, cfg, d), full)


@pytest.mark.gpu
def test_set_products_rejects_other_counts():
    from kemorin_mhd_b200.sph_trans import SphTransform, KmhdError
    from kemorin_mhd_b200.config import TIER_FP64
    cfg = SphConfig(15, 24, 48, 3)
    for tier, bad in ((TIER_SPLIT_I8, (10, 6, 25, 0)), (TIER_FP32ACC, (26, 21, 3))):
        tr = SphTransform(cfg, tier=tier)
        for b in bad:
            with pytest.raises(KmhdError):
                tr.set_products(b)
    with pytest.raises(KmhdError):
        SphTransform(cfg, tier=TIER_FP64).set_products(26)
    assert SphTransform(cfg, tier=TIER_FP64).tuning()["products"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("tier", [TIER_SPLIT_I8, TIER_FP32ACC])
def test_autotune_choice_and_result(tier):
    """After the first autotuned batch call every handle reports the three
    candidates' times and errors, its choice is the fastest candidate whose
    error is within a quarter of the bound, and the batch output meets the
    tier's bound against the oracle; a second call keeps the choice."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform, batch_cycle
    cfgs = [SphConfig(31, 48, 96, 5, name="a0"), SphConfig(63, 96, 192, 9, name="a1"),
            SphConfig(127, 192, 384, 5, name="a2")]
    trs = [SphTransform(c, tier=tier, autotune=True) for c in cfgs]
    d_np = [make_d_rj(c, seed=70 + i) for i, c in enumerate(cfgs)]
    refs = [Oracle(c, nthreads=8).cycle(d) for c, d in zip(cfgs, d_np)]
    d_in = [to_dev_fortran(d) for d in d_np]
    outs = [torch.zeros((c.ncf, c.J * c.nr), dtype=torch.float64, device="cuda") for c in cfgs]
    batch_cycle(trs, d_in, outs)
    for tr, c, o, ref in zip(trs, cfgs, outs, refs):
        t = tr.tuning()
        assert all(ms > 0 for ms in t["ms"]), t
        assert t["err"][0] == 0 and t["err"][1] > 0 and t["err"][2] > 0, t
        assert t["err"][1] <= BOUND[tier] / 4, t
        ok = [0] + [k for k in (1, 2) if t["err"][k] <= BOUND[tier] / 4]
        best = min(ok, key=lambda k: t["ms"][k])
        assert t["path"] == (1 if best > 0 else 0), t
        if best > 0:
            assert t["products"] == (FULL if best == 1 else REDUCED)[tier], t
        assert col_relerr(from_dev_fortran(o), ref).max() <= BOUND[tier], (c.name, t)
    before = [tr.tuning() for tr in trs]
    for o in outs:
        o.zero_()
    batch_cycle(trs, d_in, outs)
    for tr, b, c, o, ref in zip(trs, before, cfgs, outs, refs):
        a = tr.tuning()
        assert (a["path"], a["products"]) == (b["path"], b["products"])
        assert col_relerr(from_dev_fortran(o), ref).max() <= BOUND[tier], c.name


@pytest.mark.gpu
def test_grouped_gemm_mixed_product_counts():
    """Split instances pinned to different product counts form separate
    grouped GEMMs in one batch; each result equals the instance's own cycle."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform, batch_cycle
    cfgs = [SphConfig(31, 48, 96, 5, name="g0"), SphConfig(47, 72, 144, 3, name="g1"),
            SphConfig(31, 48, 96, 7, name="g2"), SphConfig(63, 96, 192, 4, name="g3")]
    prods = [26, 21, 21, 26]
    trs = [SphTransform(c, tier=TIER_SPLIT_I8) for c in cfgs]
    for tr, p in zip(trs, prods):
        tr.set_products(p)
    d_in = [to_dev_fortran(make_d_rj(c, seed=80 + i)) for i, c in enumerate(cfgs)]
    singles = []
    for tr, c, d in zip(trs, cfgs, d_in):
        o = torch.zeros((c.ncf, c.J * c.nr), dtype=torch.float64, device="cuda")
        tr.nonlinear_cycle(d, o)
        singles.append(o.cpu())
    outs = [torch.zeros((c.ncf, c.J * c.nr), dtype=torch.float64, device="cuda") for c in cfgs]
    batch_cycle(trs, d_in, outs)
    for c, o, ref in zip(cfgs, outs, singles):
        assert torch.equal(o.cpu(), ref), c.name
