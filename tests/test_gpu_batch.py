"""Batched uneven instances (kmhd_sph_batch_cycle) vs the CPU FP64 oracle.

Instances of different L, Nr and field counts run as one captured CUDA graph;
a second call replays it and a call with other output buffers recaptures it.
Tolerances per tier as in the single-instance tests (FP64 1e-13, split 1e-12).
"""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_FP64, TIER_SPLIT_I8
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.oracle import Oracle
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

CFGS = [
    SphConfig(31, 48, 96, 5, name="b0"),
    SphConfig(15, 24, 48, 4, nvb=1, nsb=1, nvf=1, nsf=0, products=((1, 0, 0, 1.0),), name="b1"),
    SphConfig(47, 72, 144, 3, nvb=2, nsb=1, nvf=2, nsf=1,
              products=((0, 1, 0, 1.0), (1, 0, 0, 1.0), (2, 0, 1, 1.0)), name="b2"),
    SphConfig(63, 96, 192, 3, name="b3"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("tier", [TIER_FP64, TIER_SPLIT_I8])
def test_batch_matches_oracle(tier):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform, batch_cycle
    tol = 1e-13 if tier == TIER_FP64 else 1e-12
    trs = [SphTransform(c, tier=tier, autotune=(tier != TIER_FP64)) for c in CFGS]
    d_np = [make_d_rj(c, seed=30 + i) for i, c in enumerate(CFGS)]
    refs = [Oracle(c, nthreads=8).cycle(d) for c, d in zip(CFGS, d_np)]
    d_in = [to_dev_fortran(d) for d in d_np]
    outs = [torch.zeros((c.ncf, c.J * c.nr), dtype=torch.float64, device="cuda") for c in CFGS]
    for call in range(2):  # capture, then replay
        for o in outs:
            o.zero_()
        batch_cycle(trs, d_in, outs)
        for c, o, ref in zip(CFGS, outs, refs):
            err = col_relerr(from_dev_fortran(o), ref)
            assert err.max() <= tol, (call, c.name, err)
    outs2 = [torch.zeros_like(o) for o in outs]  # new pointers: recapture
    batch_cycle(trs, d_in, outs2)
    for c, o, ref in zip(CFGS, outs2, refs):
        assert col_relerr(from_dev_fortran(o), ref).max() <= tol, c.name


@pytest.mark.gpu
def test_grouped_gemm_batch_equals_single_cycles():
    """Split-path instances of one tier share one grouped GEMM launch per
    direction (work units of every instance in one persistent grid); the
    results are bit-identical to each instance's own cycle, with instances of
    both split tiers and an FP64 instance in the same batch."""
    import torch
    from kemorin_mhd_b200.config import TIER_FP32ACC
    from kemorin_mhd_b200.sph_trans import SphTransform, batch_cycle
    tiers = [TIER_SPLIT_I8, TIER_SPLIT_I8, TIER_SPLIT_I8, TIER_FP32ACC, TIER_FP32ACC, TIER_FP64]
    cfgs = CFGS + [SphConfig(31, 48, 96, 7, name="b4"), SphConfig(63, 96, 192, 4, name="b5")]
    cfgs = [cfgs[i] for i in (0, 2, 3, 4, 1, 5)]
    trs = [SphTransform(c, tier=t) for c, t in zip(cfgs, tiers)]
    d_in = [to_dev_fortran(make_d_rj(c, seed=60 + i)) for i, c in enumerate(cfgs)]
    singles = []
    for tr, c, d in zip(trs, cfgs, d_in):
        o = torch.zeros((c.ncf, c.J * c.nr), dtype=torch.float64, device="cuda")
        tr.nonlinear_cycle(d, o)
        singles.append(o.cpu())
    outs = [torch.zeros((c.ncf, c.J * c.nr), dtype=torch.float64, device="cuda") for c in cfgs]
    for call in range(2):
        for o in outs:
            o.zero_()
        batch_cycle(trs, d_in, outs)
        for c, o, ref in zip(cfgs, outs, singles):
            assert torch.equal(o.cpu(), ref), (call, c.name)
