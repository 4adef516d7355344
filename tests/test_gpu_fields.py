"""The reference's fuller MHD field sets against the CPU oracle: the dynamo
benchmark set with the current density and the Lorentz force (backward u,
omega, B, J + T; forward omega x u, J x B, u x B, u T:
set_address_sph_trans_MHD.f90, f_trans_address_vector_MHD /
b_trans_address_vector_MHD with the Lorentz force on), and six fields per
direction (+ composition C, u C, u.omega, B.J) -- more radial-component and
scalar fields than one 8-column block of the split path holds, so its
slicers and GEMM epilogues use two field groups per radius; and the full MHD
set with the composition flux u C as a fifth forward vector (f_trns%i_c_flux).  Tolerances per
tier: FP64 1e-13, split 1e-12, FP32-accurate 1e-6 (max-norm per field)."""
import numpy as np
import pytest

from kemorin_mhd_b200.config import (PROD_CROSS, PROD_DOT, PROD_VEC_SCALAR, SphConfig, TIER_FP32ACC, TIER_FP64,
                                     TIER_SPLIT_I8)
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.oracle import Oracle
from tests.gpu_util import col_relerr, to_dev_fortran, from_dev_fortran

DYNAMO = dict(nvb=4, nsb=1, nvf=4, nsf=0,
              products=((PROD_CROSS, 1, 0, 1.0), (PROD_CROSS, 3, 2, 1.0), (PROD_CROSS, 0, 2, 1.0),
                        (PROD_VEC_SCALAR, 0, 0, 1.0)))
SIX = dict(nvb=4, nsb=2, nvf=4, nsf=2,
           products=((PROD_CROSS, 1, 0, 1.0), (PROD_CROSS, 3, 2, 0.5), (PROD_CROSS, 0, 2, 1.0),
                     (PROD_VEC_SCALAR, 0, 1, 1.0), (PROD_DOT, 0, 1, 1.0), (PROD_DOT, 2, 3, 2.0)))
# the full MHD set: composition C, and its flux u C as a fifth forward vector
FULL = dict(nvb=4, nsb=2, nvf=5, nsf=1,
            products=((PROD_CROSS, 1, 0, 1.0), (PROD_CROSS, 3, 2, 1.0), (PROD_CROSS, 0, 2, 1.0),
                      (PROD_VEC_SCALAR, 0, 0, 1.0), (PROD_VEC_SCALAR, 0, 1, 1.0), (PROD_DOT, 0, 1, 1.0)))
TOL = {TIER_FP64: 1e-13, TIER_SPLIT_I8: 1e-12, TIER_FP32ACC: 1e-6}


@pytest.mark.gpu
@pytest.mark.parametrize("fields", ["dynamo", "six", "full"])
@pytest.mark.parametrize("tier", [TIER_FP64, TIER_SPLIT_I8, TIER_FP32ACC], ids=["fp64", "split", "fp32acc"])
def test_field_sets_match_oracle(fields, tier):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(31, 48, 96, 5, name="L31_" + fields, **{"dynamo": DYNAMO, "six": SIX, "full": FULL}[fields])
    d = make_d_rj(cfg, seed=81)
    ref = Oracle(cfg, nthreads=8).cycle(d)
    tr = SphTransform(cfg, tier=tier)
    assert tr.uses_split() == (tier != TIER_FP64)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    err = col_relerr(from_dev_fortran(out), ref)
    assert err.max() <= TOL[tier], err


@pytest.mark.gpu
def test_six_fields_host_chunked_equals_device():
    """Radial chunks of a host-pointer cycle with two field groups per radius
    (tile radii taken within a group) reproduce the device cycle exactly."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(127, 192, 384, 65, name="L127_six", **SIX)
    tr = SphTransform(cfg, tier=TIER_SPLIT_I8)
    d = make_d_rj(cfg, seed=82)
    n = cfg.J * cfg.nr
    out = torch.zeros((cfg.ncf, n), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    h_out = np.zeros((n, cfg.ncf), order="F")
    tr.nonlinear_cycle(np.asfortranarray(d), h_out)
    assert np.array_equal(h_out, from_dev_fortran(out))


@pytest.mark.gpu
@pytest.mark.parametrize("fields", ["dynamo", "full"])
@pytest.mark.parametrize("tier", [TIER_FP64, TIER_SPLIT_I8], ids=["fp64", "split"])
def test_wide_grid_field_sets_read_spectra_in_place(tier, fields):
    """L=255 on a 1536-point phi grid with the dynamo and full sets: the
    line's grid pairs (7 or 8, up to 197 KB) fit in shared memory but not with
    the staged spectra, so the specialised FFT passes read the spectra in
    place (instantiated at each set's own counts)."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(255, 384, 1536, 3, name="L255_wide_" + fields, **(FULL if fields == "full" else DYNAMO))
    d = make_d_rj(cfg, seed=83)
    ref = Oracle(cfg, nthreads=16).cycle(d)
    tr = SphTransform(cfg, tier=tier)
    out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(to_dev_fortran(d), out)
    err = col_relerr(from_dev_fortran(out), ref)
    assert err.max() <= TOL[tier], err
