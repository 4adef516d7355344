"""Backward transform at the poles (kmhd_sph_b_trans_pole) against the CPU
oracle of schmidt_b_trans_pole_vect / _scalar (oracle/sph_pole.py): <= 1e-13
of each field's maximum, device and host pointers, permuted field columns."""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_FP64, TIER_SPLIT_I8, rj_order
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.sph_pole import b_trans_pole
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

CFG = SphConfig(31, 48, 96, 9, name="L31")


@pytest.mark.gpu
@pytest.mark.parametrize("host,tier", [(False, TIER_FP64), (True, TIER_FP64), (False, TIER_SPLIT_I8)],
                         ids=["device", "host", "split_handle"])
def test_pole_values_match_oracle(host, tier):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    tr = SphTransform(cfg, tier=tier)
    d = make_d_rj(cfg, seed=91)
    d[:, 2] += np.random.default_rng(3).standard_normal(d.shape[0])   # toroidal u of every order
    l, m = rj_order(cfg.ltr)
    ref = b_trans_pole(cfg.radius(), cfg.ltr, l, m, d, cfg.nvb, cfg.nsb)
    # the fields in other columns of a wider array: [T, B, pad, u, omega]
    wide = np.zeros((d.shape[0], 12), order="F")
    wide[:, 0] = d[:, 9]
    wide[:, 1:4] = d[:, 6:9]
    wide[:, 5:8] = d[:, 0:3]
    wide[:, 8:11] = d[:, 3:6]
    cols = [5, 8, 1, 0]
    if host:
        got = np.zeros((2 * cfg.nr, cfg.ncb), order="F")
        tr.b_trans_pole(wide, got, cols_b=cols)
    else:
        out = torch.zeros((cfg.ncb, 2 * cfg.nr), dtype=torch.float64, device="cuda")
        tr.b_trans_pole(to_dev_fortran(wide), out, cols_b=cols)
        got = from_dev_fortran(out)
    assert col_relerr(got, ref).max() <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True], ids=["device", "host"])
def test_center_values_match_oracle(host):
    """Centre node of a full-sphere grid (kmhd_sph_b_trans_center) against the
    oracle of schmidt_b_trans_center_vect: vector entries bit-identical,
    scalar entries untouched, fields in permuted columns."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_pole import b_trans_center
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    d = make_d_rj(cfg, seed=17)
    l, m = rj_order(cfg.ltr)
    v0 = np.full(cfg.ncb, 5.25)
    ref = b_trans_center(cfg.radius(), l, m, d, cfg.nvb, cfg.nsb, v_in=v0)
    wide = np.zeros((d.shape[0], 12), order="F")
    wide[:, 0] = d[:, 9]
    wide[:, 1:4] = d[:, 6:9]
    wide[:, 5:8] = d[:, 0:3]
    wide[:, 8:11] = d[:, 3:6]
    cols = [5, 8, 1, 0]
    if host:
        got = v0.copy()
        tr.b_trans_center(wide, got, cols_b=cols)
    else:
        out = torch.from_numpy(v0.copy()).cuda()
        tr.b_trans_center(to_dev_fortran(wide), out, cols_b=cols)
        got = out.cpu().numpy()
    assert np.array_equal(got, ref), (got, ref)
