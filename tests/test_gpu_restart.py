"""A dynamo state read from the reference's field-file formats goes through
the cycle unchanged: the binary file's spectra give the same cycle as the
arrays they were written from, bit for bit, and the forward fields written
back and read again are those of the cycle."""
import numpy as np
import pytest

from kemorin_mhd_b200 import restart
from kemorin_mhd_b200.config import SphConfig, TIER_SPLIT_I8
from kemorin_mhd_b200.synthetic import make_d_rj
from tests.gpu_util import to_dev_fortran, from_dev_fortran


@pytest.mark.gpu
def test_cycle_of_a_restart_file(tmp_path):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = SphConfig(31, 48, 96, 9, name="L31")
    d = make_d_rj(cfg, seed=71)
    names = ["velocity", "vorticity", "magnetic_field", "temperature"]
    p = str(tmp_path / restart.file_name("rst", 40, 0, "binary"))
    restart.write(p, restart.from_d_rj(d, names, [3, 3, 3, 1], step=40, time=0.5))
    f = restart.read(p)
    tr = SphTransform(cfg, tier=TIER_SPLIT_I8)
    outs = []
    for src in (d, f.d_rj(names)):
        o = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
        tr.nonlinear_cycle(to_dev_fortran(src), o)
        outs.append(from_dev_fortran(o))
    assert np.array_equal(outs[0], outs[1])
    q = str(tmp_path / restart.file_name("nl", 40, 0, "gz_binary"))
    restart.write(q, restart.from_d_rj(outs[1], ["m_advect", "vp_induct", "h_flux", "k_heli"], [3, 3, 3, 1]))
    assert np.array_equal(restart.read(q).data, outs[1])


@pytest.mark.gpu
def test_real_state_pipeline_from_restart(tmp_path):
    """A restart holds u, B, T (not omega, J): read it, form omega = curl u
    (non-slip) and J = curl B (insulating) on the GPU, and run the dynamo
    benchmark cycle (u, omega, B, J + T -> omega x u, J x B, u x B, u T);
    against the oracle chain on the same file (FP64 tier, <= 1e-12)."""
    import torch
    from kemorin_mhd_b200.config import PROD_CROSS, PROD_VEC_SCALAR, rj_order
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.oracle import Oracle
    from oracle.sph_div import current, vorticity
    from tests.gpu_util import col_relerr
    dyn = SphConfig(31, 48, 96, 9, nvb=4, nsb=1, nvf=4, nsf=0,
                    products=((PROD_CROSS, 1, 0, 1.0), (PROD_CROSS, 3, 2, 1.0), (PROD_CROSS, 0, 2, 1.0),
                              (PROD_VEC_SCALAR, 0, 0, 1.0)), name="L31_dynamo")
    src = make_d_rj(SphConfig(31, 48, 96, 9, name="L31"), seed=73)      # u, omega, B, T: keep u, B, T
    n = dyn.J * dyn.nr
    p = str(tmp_path / restart.file_name("rst", 7, 0, "text"))
    restart.write(p, restart.from_d_rj(np.asfortranarray(np.concatenate([src[:, 0:3], src[:, 6:9], src[:, 9:10]], 1)),
                                       ["velocity", "magnetic_field", "temperature"], [3, 3, 1], step=7))
    f = restart.read(p)
    u, B, T = f.field("velocity"), f.field("magnetic_field"), f.field("temperature")
    # device: columns u (0-2), omega (3-5), B (6-8), J (9-11), T (12)
    d = np.zeros((n, 13), order="F")
    d[:, 0:3], d[:, 6:9], d[:, 12:13] = u, B, T
    tr = SphTransform(dyn, tier=0)
    t = to_dev_fortran(d)
    tr.vorticity(t, 0, 3)
    tr.current(t, 6, 9)
    out = torch.zeros((dyn.ncf, n), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(t, out)
    got = from_dev_fortran(out)
    # oracle chain
    l, _ = rj_order(dyn.ltr)
    r = dyn.radius()
    w = np.stack(vorticity(r, l, u[:, 0], u[:, 1], u[:, 2]), 1)
    J = np.stack(current(r, l, B[:, 0], B[:, 1], B[:, 2]), 1)
    dref = np.asfortranarray(np.concatenate([u, w, B, J, T], 1))
    ref = Oracle(dyn, nthreads=8).cycle(dref)
    assert col_relerr(got, ref).max() <= 1e-12
