"""kmhd_sph_cycle_noalloc: the FP64 cycle for callers that cannot allocate device memory.

Some callers of this library may not call cudaMalloc themselves -- a solver
whose host framework owns the whole device pool, or a time-step loop that must
not allocate after set-up.  kmhd_sph_cycle_noalloc serves them from one static
32 MiB device array instead of a handle's buffers.  These tests call it
through the C-ABI and check it against kmhd_sph_cycle (FP64 tier) on the same
inputs, to the FP64 tier's tolerance, on consecutive calls that reuse the
array's stale contents.  This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig
from kemorin_mhd_b200.synthetic import make_d_rj
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

TOL = 1e-13

CFG_A = SphConfig(31, 48, 96, 9, name="L31_Nr9")
CFG_B = SphConfig(47, 73, 144, 6, name="L47_odd_nth")


class _Args:
    """Descriptor and host column arrays of one configuration (kept alive)."""

    def __init__(self, cfg, tier=0):
        from kemorin_mhd_b200 import sph_trans as st
        self.r = np.ascontiguousarray(cfg.radius(), np.float64)
        self.prods = (st.Product * len(cfg.products))(
            *[st.Product(int(k), int(a), int(b), float(c)) for (k, a, b, c) in cfg.products])
        d = st.Desc()
        d.ltr, d.nth, d.nph, d.nr = cfg.ltr, cfg.nth, cfg.nph, cfg.nr
        d.radius = self.r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.nvector_b, d.nscalar_b, d.nvector_f, d.nscalar_f = cfg.nvb, cfg.nsb, cfg.nvf, cfg.nsf
        d.nproduct, d.products = len(cfg.products), self.prods
        d.tier, d.device = tier, 0
        self.desc = d
        nb, nf = cfg.nvb + cfg.nsb, cfg.nvf + cfg.nsf
        self.cols_b = (ctypes.c_int32 * nb)(*[3 * f if f < cfg.nvb else 3 * cfg.nvb + f - cfg.nvb
                                              for f in range(nb)])
        self.cols_f = (ctypes.c_int32 * nf)(*[3 * f if f < cfg.nvf else 3 * cfg.nvf + f - cfg.nvf
                                              for f in range(nf)])


def _noalloc(lib, cfg, d_in, d_out):
    a = _Args(cfg)
    n = cfg.J * cfg.nr
    return lib.kmhd_sph_cycle_noalloc(ctypes.byref(a.desc), d_in.data_ptr(), n, a.cols_b,
                                      d_out.data_ptr(), n, a.cols_f, None)


def _reference(cfg, d_in):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    SphTransform(cfg, tier=0).nonlinear_cycle(d_in, out)
    torch.cuda.synchronize()
    return from_dev_fortran(out)


def test_noalloc_rejects_without_touching_the_gpu():
    # argument and size checks come before any CUDA call
    from kemorin_mhd_b200 import sph_trans as st
    lib = st.load_library()
    big = _Args(SphConfig(127, 192, 384, 33, name="L127"))
    dummy = ctypes.c_void_p(16)
    n = 128 * 128 * 33
    assert lib.kmhd_sph_cycle_noalloc(ctypes.byref(big.desc), dummy, n, big.cols_b, dummy, n,
                                      big.cols_f, None) == 2  # beyond the 32 MiB work area
    split = _Args(CFG_A, tier=1)
    n = CFG_A.J * CFG_A.nr
    assert lib.kmhd_sph_cycle_noalloc(ctypes.byref(split.desc), dummy, n, split.cols_b, dummy, n,
                                      split.cols_f, None) == 1  # FP64 tier only
    ok = _Args(CFG_A)
    assert lib.kmhd_sph_cycle_noalloc(ctypes.byref(ok.desc), dummy, n - 1, ok.cols_b, dummy, n,
                                      ok.cols_f, None) == 1  # leading dimension too small
    flagged = _Args(CFG_A)
    flagged.desc.flags = 2  # on-the-fly tables are a handle option, not offered here
    assert lib.kmhd_sph_cycle_noalloc(ctypes.byref(flagged.desc), dummy, n, flagged.cols_b, dummy, n,
                                      flagged.cols_f, None) == 1


@pytest.mark.gpu
def test_noalloc_matches_cycle_two_calls():
    import torch
    from kemorin_mhd_b200 import sph_trans as st
    lib = st.load_library()
    d_in = to_dev_fortran(make_d_rj(CFG_A, seed=21))
    ref = _reference(CFG_A, d_in)
    for call in range(2):
        out = torch.zeros((CFG_A.ncf, CFG_A.J * CFG_A.nr), dtype=torch.float64, device="cuda")
        assert _noalloc(lib, CFG_A, d_in, out) == 0
        assert torch.cuda.current_device() == 0  # the caller's device is current again
        err = col_relerr(from_dev_fortran(out), ref)
        assert err.max() <= TOL, (call, err)


@pytest.mark.gpu
def test_noalloc_after_a_different_size():
    # a call of another size leaves different data in the shared array
    import torch
    from kemorin_mhd_b200 import sph_trans as st
    lib = st.load_library()
    for cfg, seed in ((CFG_B, 22), (CFG_A, 23)):
        d_in = to_dev_fortran(make_d_rj(cfg, seed=seed))
        ref = _reference(cfg, d_in)
        out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
        assert _noalloc(lib, cfg, d_in, out) == 0
        err = col_relerr(from_dev_fortran(out), ref)
        assert err.max() <= TOL, (cfg.name, err)
