"""Split-precision tiers on the tcgen05 tensor cores vs the CPU FP64 oracle.

Tolerances (max-norm relative error per field): tier "split" (6 INT8 slices,
26 slice products) <= 1e-12; tier "fp32acc" (4 slices, 10 products) <= 1e-6.
"""
import ctypes

import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_SPLIT_I8, TIER_FP32ACC
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.oracle import Oracle
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

TOL = {TIER_SPLIT_I8: 1e-12, TIER_FP32ACC: 1e-6}


@pytest.mark.gpu
def test_i8_mma_tile_layout():
    from kemorin_mhd_b200.sph_trans import load_library
    lib = load_library()
    f = lib.kmhd_selftest_i8_mma
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    rng = np.random.default_rng(0)
    A = rng.integers(-128, 128, (128, 32)).astype(np.int8)
    B = rng.integers(-128, 128, (64, 32)).astype(np.int8)
    D = np.zeros((128, 64), np.int32)
    assert f(128, 256, A.ctypes.data, B.ctypes.data, D.ctypes.data) == 0
    ref = A.astype(np.int64) @ B.astype(np.int64).T
    assert np.array_equal(D.astype(np.int64), ref)


CFGS = [
    SphConfig(31, 48, 96, 9, name="L31"),
    SphConfig(47, 73, 144, 6, name="L47_odd_nth"),
    SphConfig(16, 26, 40, 5, nvb=1, nsb=2, nvf=1, nsf=1,
              products=((1, 0, 1, 0.5), (3, 0, 1, 2.0)), name="L16_mixed"),
    SphConfig(127, 192, 384, 17, name="L127"),
    SphConfig(63, 96, 3072, 3, name="L63_wide"),
]


@pytest.fixture(scope="module", params=[(c, t) for c in CFGS for t in (TIER_SPLIT_I8, TIER_FP32ACC)],
                ids=lambda p: f"{p[0].name}-tier{p[1]}")
def case(request):
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg, tier = request.param
    return cfg, tier, SphTransform(cfg, tier=tier), Oracle(cfg, nthreads=8)


@pytest.mark.gpu
def test_split_b_trans(case):
    import torch
    cfg, tier, tr, orc = case
    d = make_d_rj(cfg, seed=21)
    ref = orc.b_trans(d)
    fld = torch.empty((cfg.ncb, cfg.nr * cfg.nth * cfg.nph), dtype=torch.float64, device="cuda")
    tr.sph_b_trans(to_dev_fortran(d), fld)
    err = col_relerr(from_dev_fortran(fld), ref)
    assert err.max() <= TOL[tier], err


@pytest.mark.gpu
def test_split_f_trans(case):
    import torch
    cfg, tier, tr, orc = case
    rng = np.random.default_rng(8)
    frc = np.asfortranarray(rng.standard_normal((cfg.nr * cfg.nth * cfg.nph, cfg.ncf)))
    ref = orc.f_trans(frc)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.sph_f_trans(to_dev_fortran(frc), out)
    err = col_relerr(from_dev_fortran(out), ref)
    assert err.max() <= TOL[tier], err


@pytest.mark.gpu
def test_split_cycle(case):
    import torch
    cfg, tier, tr, orc = case
    d = make_d_rj(cfg, seed=22)
    ref = orc.cycle(d)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    err = col_relerr(from_dev_fortran(out), ref)
    assert err.max() <= TOL[tier], err


@pytest.mark.gpu
@pytest.mark.parametrize("tier", [TIER_SPLIT_I8, TIER_FP32ACC])
def test_split_dipole_modes_fp64(tier):
    """The orders m <= 2 (all dipole l <= 2 modes among them) of the forward
    transform are accumulated in FP64 in both split tiers: FP64 tolerance 1e-13
    on those rows of sph_f_trans, whatever the tier's bound on the others."""
    import torch
    from kemorin_mhd_b200.config import rj_order
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(31, 48, 96, 5, name="L31_dipole")
    tr = SphTransform(cfg, tier=tier)
    orc = Oracle(cfg, nthreads=8)
    rng = np.random.default_rng(17)
    nnod = cfg.nr * cfg.nth * cfg.nph
    frc = np.asfortranarray(rng.standard_normal((nnod, cfg.ncf)))
    ref = orc.f_trans(frc)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.sph_f_trans(to_dev_fortran(frc), out)
    got = from_dev_fortran(out)
    l, m = rj_order(cfg.ltr)
    rows = np.concatenate([np.where(np.abs(m) <= 2)[0] + cfg.J * k for k in range(cfg.nr)])
    den = np.abs(ref).max(axis=0)
    err = (np.abs(got[rows] - ref[rows]).max(axis=0) / den).max()
    assert err <= 1e-13, err


@pytest.mark.gpu
def test_split_vs_fp64_L1023():
    """cfg5 angular grid (L=1023, Ntheta=1536, Nphi=3072; wide lines go through
    the FFT pair by pair): split tier against the FP64 GPU tier on the same
    input (the CPU oracle at this L takes minutes; the FP64 tier is pinned to
    the oracle at L <= 511 and on the wide-line path at L=63)."""
    import torch
    from kemorin_mhd_b200.config import TIER_FP64
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(1023, 1536, 3072, 3, name="L1023_Nr3")
    d = to_dev_fortran(make_d_rj(cfg, seed=19))
    outs = []
    for tier in (TIER_FP64, TIER_SPLIT_I8):
        tr = SphTransform(cfg, tier=tier)
        out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
        tr.nonlinear_cycle(d, out)
        outs.append(from_dev_fortran(out))
        tr.close()
    err = col_relerr(outs[1], outs[0])
    assert err.max() <= TOL[TIER_SPLIT_I8], err


# The benchmark's angular grids with their own default field set (u, omega, B
# + T backward; omega x u, u x B, u T + u.omega forward): cfg3's L=511,
# Ntheta=768, Nphi=1536 and cfg2's L=255, Ntheta=384, Nphi=768, on a few
# radii so the CPU oracle finishes in seconds.  Every tier against the oracle,
# per field, at its stated bound.
BENCH_GRIDS = [
    SphConfig(511, 768, 1536, 3, name="L511_Nr3"),
    SphConfig(255, 384, 768, 5, name="L255_Nr5"),
]


@pytest.fixture(scope="module")
def bench_oracle_outputs():
    cache = {}

    def get(cfg, what, seed):
        key = (cfg.name, what, seed)
        if key not in cache:
            orc = Oracle(cfg, nthreads=8)
            if what == "cycle":
                cache[key] = orc.cycle(make_d_rj(cfg, seed=seed))
            else:
                cache[key] = orc.b_trans(make_d_rj(cfg, seed=seed))
        return cache[key]
    return get


@pytest.mark.gpu
@pytest.mark.parametrize("tier", [TIER_SPLIT_I8, TIER_FP32ACC], ids=["split", "fp32acc"])
@pytest.mark.parametrize("cfg", BENCH_GRIDS, ids=lambda c: c.name)
def test_split_tiers_at_benchmark_grids(cfg, tier, bench_oracle_outputs):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    tr = SphTransform(cfg, tier=tier)
    d = make_d_rj(cfg, seed=31)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    err = col_relerr(from_dev_fortran(out), bench_oracle_outputs(cfg, "cycle", 31))
    fld = torch.empty((cfg.ncb, cfg.nr * cfg.nth * cfg.nph), dtype=torch.float64, device="cuda")
    tr.sph_b_trans(to_dev_fortran(d), fld)
    err_b = col_relerr(from_dev_fortran(fld), bench_oracle_outputs(cfg, "b_trans", 31))
    tr.close()
    assert err.max() <= TOL[tier], err
    assert err_b.max() <= TOL[tier], err_b
