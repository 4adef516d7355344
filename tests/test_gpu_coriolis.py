"""Curl of the Coriolis term (kmhd_sph_rot_coriolis) against the CPU oracle
of the reference's sum_rot_coriolis_rlm_10 with its Gaunt / Elsasser tables
(oracle/sph_coriolis.py): max-norm relative error <= 1e-13, device and host
pointers, the reference's mode order and a permuted one; the column that the
reference leaves to the forward transform (col_out + 1) stays untouched."""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_FP64, TIER_SPLIT_I8, rj_order
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.sph_coriolis import rot_coriolis
from tests.gpu_util import to_dev_fortran, from_dev_fortran

CFG = SphConfig(31, 48, 96, 9, name="L31")


def _relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("host,permuted", [(False, False), (True, False), (False, True)],
                         ids=["device", "host", "permuted_order"])
def test_rot_coriolis_matches_oracle(host, permuted):
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    L, J, nr = cfg.ltr, cfg.J, cfg.nr
    l, m = rj_order(L)
    perm = np.random.default_rng(3).permutation(J) if permuted else np.arange(J)
    lp, mp = l[perm], m[perm]
    tr = SphTransform(cfg, tier=TIER_FP64, idx_rj_lm=np.stack([lp, mp], 1).reshape(-1) if permuted else None)
    rng = np.random.default_rng(21)
    d = np.asfortranarray(rng.standard_normal((J * nr, 9)))
    coef = 2.5e3
    r = cfg.radius()
    ref_pol, ref_tor = rot_coriolis(r, L, lp, mp, [d[:, q] for q in range(3)], [d[:, 3 + q] for q in range(3)], coef)
    if host:
        arr = d.copy(order="F")
        tr.rot_coriolis(arr, 0, 3, 6, coef)
        got = arr
    else:
        t = to_dev_fortran(d)
        tr.rot_coriolis(t, 0, 3, 6, coef)
        got = from_dev_fortran(t)
    assert np.array_equal(got[:, :6], d[:, :6])
    assert np.array_equal(got[:, 7], d[:, 7])          # dpol/dr column not written
    assert _relerr(got[:, 6], ref_pol) <= 1e-13
    assert _relerr(got[:, 8], ref_tor) <= 1e-13


@pytest.mark.gpu
def test_rot_coriolis_rejects_output_over_inputs():
    import torch
    from kemorin_mhd_b200.sph_trans import KmhdError, SphTransform
    tr = SphTransform(CFG, tier=TIER_FP64)
    t = torch.zeros((9, CFG.J * CFG.nr), dtype=torch.float64, device="cuda")
    for col_out in (1, 3, 5):
        with pytest.raises(KmhdError):
            tr.rot_coriolis(t, 0, 3, col_out, 1.0)


@pytest.mark.gpu
def test_rot_coriolis_on_cycle_inputs():
    """On a split-tier handle, after a cycle: the curl of the Coriolis term
    of the cycle's own velocity and vorticity spectra (synthetic dynamo-like
    profiles) against the oracle."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_SPLIT_I8)
    d_np = make_d_rj(cfg, seed=41)                   # columns: u (0-2), omega (3-5), B (6-8), T (9)
    d = to_dev_fortran(d_np)
    out = torch.zeros((cfg.ncf + 3, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(d, out)
    cor = torch.zeros((3, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    both = torch.cat([d, cor], 0)                    # velocity, vorticity, ..., output columns 10-12
    tr.rot_coriolis(both, 0, 3, cfg.ncb, 1.0e2)
    got = from_dev_fortran(both)
    l, m = rj_order(cfg.ltr)
    ref_pol, ref_tor = rot_coriolis(cfg.radius(), cfg.ltr, l, m, [d_np[:, q] for q in range(3)],
                                    [d_np[:, 3 + q] for q in range(3)], 1.0e2)
    assert _relerr(got[:, cfg.ncb], ref_pol) <= 1e-13
    assert _relerr(got[:, cfg.ncb + 2], ref_tor) <= 1e-13


def _cycle_ref(cfg, tier, d_np, **kw):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    tr = SphTransform(cfg, tier=tier, **kw)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d_np), out)
    return from_dev_fortran(out)


@pytest.mark.gpu
@pytest.mark.parametrize("tier", [TIER_FP64, TIER_SPLIT_I8], ids=["fp64", "split"])
def test_cycle_with_coriolis_device(tier):
    """kmhd_sph_set_coriolis: the cycle also writes the Coriolis curl of its
    own velocity / vorticity inputs into columns ncf (pol) and ncf + 2 (tor);
    the forward fields are bit-identical to a cycle without it, ncf + 1 is
    untouched; switching it off leaves the columns alone."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    d_np = make_d_rj(cfg, seed=43)
    plain = _cycle_ref(cfg, tier, d_np)
    tr = SphTransform(cfg, tier=tier)
    coef = 3.0e2
    tr.set_coriolis(coef, 0, 1, cfg.ncf)
    out = torch.full((cfg.ncf + 3, cfg.J * cfg.nr), 7.0, dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d_np), out)
    got = from_dev_fortran(out)
    assert np.array_equal(got[:, :cfg.ncf], plain)
    assert (got[:, cfg.ncf + 1] == 7.0).all()
    l, m = rj_order(cfg.ltr)
    ref_pol, ref_tor = rot_coriolis(cfg.radius(), cfg.ltr, l, m, [d_np[:, q] for q in range(3)],
                                    [d_np[:, 3 + q] for q in range(3)], coef)
    assert _relerr(got[:, cfg.ncf], ref_pol) <= 1e-13
    assert _relerr(got[:, cfg.ncf + 2], ref_tor) <= 1e-13
    tr.set_coriolis(0.0, -1)
    out2 = torch.full_like(out, 5.0)
    tr.nonlinear_cycle(to_dev_fortran(d_np), out2)
    assert (from_dev_fortran(out2)[:, cfg.ncf:] == 5.0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [SphConfig(31, 48, 96, 9, name="L31"), SphConfig(127, 192, 384, 65, name="L127_Nr65")],
                         ids=["host_one_pass", "host_chunked"])
def test_cycle_with_coriolis_host_equals_device(cfg):
    """Host-pointer cycles (one pass; radial chunks above 64 MiB of copies)
    give the device cycle's Coriolis columns exactly, from the staged inputs."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    tr = SphTransform(cfg, tier=TIER_FP64)
    tr.set_coriolis(1.5e2, 0, 1, cfg.ncf)
    d_np = make_d_rj(cfg, seed=44)
    n = cfg.J * cfg.nr
    out = torch.zeros((cfg.ncf + 3, n), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d_np), out)
    ref = from_dev_fortran(out)
    h_out = np.full((n, cfg.ncf + 3), np.nan, order="F")
    tr.nonlinear_cycle(np.asfortranarray(d_np), h_out)
    assert np.array_equal(h_out[:, :cfg.ncf], ref[:, :cfg.ncf])
    assert np.array_equal(h_out[:, cfg.ncf], ref[:, cfg.ncf])
    assert np.array_equal(h_out[:, cfg.ncf + 2], ref[:, cfg.ncf + 2])
    assert np.isnan(h_out[:, cfg.ncf + 1]).all()


@pytest.mark.gpu
def test_batch_with_coriolis_equals_single_cycles():
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform, batch_cycle
    cfgs = [SphConfig(31, 48, 96, 5, name="c0"), SphConfig(47, 72, 144, 3, name="c1"),
            SphConfig(31, 48, 96, 4, name="c2")]
    tiers = [TIER_SPLIT_I8, TIER_SPLIT_I8, TIER_FP64]
    trs = [SphTransform(c, tier=t) for c, t in zip(cfgs, tiers)]
    for i, tr in enumerate(trs):
        if i != 2:                                   # the FP64 instance runs without it
            tr.set_coriolis(10.0 * (i + 1), 0, 1, cfgs[i].ncf)
    d_in = [to_dev_fortran(make_d_rj(c, seed=50 + i)) for i, c in enumerate(cfgs)]
    singles = []
    for tr, c, d in zip(trs, cfgs, d_in):
        o = torch.zeros((c.ncf + 3, c.J * c.nr), dtype=torch.float64, device="cuda")
        tr.nonlinear_cycle(d, o)
        singles.append(o.cpu())
    outs = [torch.zeros((c.ncf + 3, c.J * c.nr), dtype=torch.float64, device="cuda") for c in cfgs]
    for call in range(2):                            # capture, then replay
        for o in outs:
            o.zero_()
        batch_cycle(trs, d_in, outs)
        for c, o, ref in zip(cfgs, outs, singles):
            assert torch.equal(o.cpu(), ref), (call, c.name)


@pytest.mark.gpu
def test_cycle_with_coriolis_rejects_conflicting_columns():
    import torch
    from kemorin_mhd_b200.sph_trans import KmhdError, SphTransform
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    with pytest.raises(KmhdError):
        tr.set_coriolis(1.0, 0, 0, cfg.ncf)          # velocity and vorticity the same vector
    with pytest.raises(KmhdError):
        tr.set_coriolis(1.0, 0, cfg.nvb, cfg.ncf)    # no such backward vector
    tr.set_coriolis(1.0, 0, 1, 2)                    # col_out + 0 / + 2 inside the first forward vector
    d = to_dev_fortran(make_d_rj(cfg, seed=45))
    out = torch.zeros((cfg.ncf + 3, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    with pytest.raises(KmhdError):
        tr.nonlinear_cycle(d, out)


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True], ids=["device", "host"])
def test_separable_transforms_carry_coriolis(host):
    """kmhd_sph_b_trans forms the registered Coriolis curl from its input and
    the next kmhd_sph_f_trans writes it out (sph_b_trans_w_coriolis /
    sph_f_trans_w_coriolis); equal to the standalone curl of the same input."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    d = make_d_rj(cfg, seed=47)
    n = cfg.J * cfg.nr
    ref_in = np.asfortranarray(np.concatenate([d, np.zeros((n, 3))], 1))
    ref_t = to_dev_fortran(ref_in)
    tr.rot_coriolis(ref_t, 0, 3, cfg.ncb, 5.0)
    ref = from_dev_fortran(ref_t)
    tr.set_coriolis(5.0, 0, 1, cfg.ncf)
    nnod = cfg.nr * cfg.nth * cfg.nph
    if host:
        grid = np.zeros((nnod, cfg.ncb), order="F")
        tr.sph_b_trans(np.asfortranarray(d), grid)
        frc = np.zeros((nnod, cfg.ncf), order="F")
        out = np.full((n, cfg.ncf + 3), 9.0, order="F")
        tr.sph_f_trans(frc, out)
        got = out
    else:
        grid = torch.zeros((cfg.ncb, nnod), dtype=torch.float64, device="cuda")
        tr.sph_b_trans(to_dev_fortran(d), grid)
        frc = torch.zeros((cfg.ncf, nnod), dtype=torch.float64, device="cuda")
        out = torch.full((cfg.ncf + 3, n), 9.0, dtype=torch.float64, device="cuda")
        tr.sph_f_trans(frc, out)
        got = from_dev_fortran(out)
    assert np.array_equal(got[:, cfg.ncf], ref[:, cfg.ncb])
    assert np.array_equal(got[:, cfg.ncf + 2], ref[:, cfg.ncb + 2])
    assert (got[:, cfg.ncf + 1] == 9.0).all()
