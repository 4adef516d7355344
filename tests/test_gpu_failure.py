"""Failure detection without a GPU fault.

Every spin-wait of the library's kernels (the tcgen05 pipeline's mbarrier
waits, the FFT's staging wait) is bounded: on expiry the kernel records
KMHD_ERR_TIMEOUT in a device error word, skips the remaining waits and
returns, and the host call returns the status.  The self-test entry point
runs each wait on an mbarrier that nothing completes; afterwards the same
process runs a normal cycle, so the CUDA context is still usable.
"""
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_SPLIT_I8
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.oracle import Oracle
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

KMHD_ERR_TIMEOUT = 6


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1], ids=["tcgen05_pipeline_wait", "fft_staging_wait"])
def test_bounded_wait_reports_timeout_and_context_survives(which):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform, load_library, strerror
    lib = load_library()
    st = lib.kmhd_selftest_wait_timeout(0, which)
    assert st == KMHD_ERR_TIMEOUT, st
    assert strerror(st) == "bounded device wait expired"
    # the context still runs a full split-tier cycle correctly
    cfg = SphConfig(31, 48, 96, 5, name="L31")
    tr = SphTransform(cfg, tier=TIER_SPLIT_I8)
    d = make_d_rj(cfg, seed=90)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    assert col_relerr(from_dev_fortran(out), Oracle(cfg, nthreads=8).cycle(d)).max() <= 1e-12
    tr.close()


def test_selftest_rejects_unknown_wait():
    # argument check before any device call
    from kemorin_mhd_b200.sph_trans import load_library
    assert load_library().kmhd_selftest_wait_timeout(0, 7) == 1
