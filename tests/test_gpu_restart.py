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
