"""Host-pointer cycles in radial chunks, copies overlapping the kernels.

Every stage of the cycle is independent per radius (per-(m, r) Legendre
columns, per-(r, theta) FFT lines, pointwise products), so a handle whose
host copies exceed 64 MiB runs kmhd_sph_cycle with host pointers over radial
chunks of a multiple of 16 radii: chunk c + 1's spectra are copied in and
chunk c - 1's results copied out while chunk c's kernels run.  The chunked
call must reproduce the device-pointer call exactly (the same kernels on the
same radii), honour the caller's leading dimension and column map, and leave
every other host element untouched.
"""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_FP64, TIER_SPLIT_I8, TIER_FP32ACC
from kemorin_mhd_b200.synthetic import make_d_rj
from tests.gpu_util import to_dev_fortran, from_dev_fortran

# 2 x 10 columns x 16384 modes x 65 radii x 8 B = 170 MB of copies: chunks of
# 16, 16, 16 and 17 radii
CFG = SphConfig(127, 192, 384, 65, name="L127_Nr65")


@pytest.mark.gpu
@pytest.mark.parametrize("tier,otf", [(TIER_FP64, False), (TIER_FP64, True), (TIER_SPLIT_I8, False),
                                      (TIER_FP32ACC, False)],
                         ids=["fp64", "fp64_p_on_the_fly", "split", "fp32acc"])
def test_host_chunked_cycle_equals_device_cycle(tier, otf):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    tr = SphTransform(cfg, tier=tier, p_on_the_fly=otf)
    d = make_d_rj(cfg, seed=31)
    n = cfg.J * cfg.nr
    out_dev = torch.zeros((cfg.ncf, n), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out_dev)
    ref = from_dev_fortran(out_dev)

    # host arrays with a wider leading dimension and shifted field columns
    ld = n + 40
    h_in = np.zeros((ld, cfg.ncb + 2), order="F")
    h_in[:n, 2:] = d
    h_out = np.full((ld, cfg.ncf + 1), np.nan, order="F")
    cols_b = [c + 2 for c in cfg.cols_b()]
    cols_f = [c + 1 for c in cfg.cols_f()]
    for _ in range(2):  # the second call reuses the streams, events and staging
        h_out[:n, 1:] = np.nan
        tr.nonlinear_cycle(h_in, h_out, cols_b=cols_b, cols_f=cols_f, ld_in=ld, ld_out=ld)
        assert np.array_equal(h_out[:n, 1:], ref)
    assert np.isnan(h_out[:, 0]).all() and np.isnan(h_out[n:, :]).all()
    t = tr.last_timing()
    # chunked calls time only the whole call (the stages overlap)
    assert t["leg_bwd"] == 0.0 and t["fft_nl"] == 0.0 and t["leg_fwd"] == 0.0 and t["total"] > 0.0
    tr.close()


@pytest.mark.gpu
def test_host_unchunked_small_cycle_times_stages():
    """Below 64 MiB of copies the host call stays one serial pass, with stage times."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(31, 48, 96, 9, name="L31")
    tr = SphTransform(cfg, tier=TIER_SPLIT_I8)
    d = make_d_rj(cfg, seed=32)
    n = cfg.J * cfg.nr
    out_dev = torch.zeros((cfg.ncf, n), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out_dev)
    h_out = np.zeros((n, cfg.ncf), order="F")
    tr.nonlinear_cycle(np.asfortranarray(d), h_out)
    assert np.array_equal(h_out, from_dev_fortran(out_dev))
    t = tr.last_timing()
    assert t["leg_bwd"] > 0.0 and t["fft_nl"] > 0.0 and t["leg_fwd"] > 0.0
    tr.close()
