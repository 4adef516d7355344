"""Radial slabs on the GPU: the ranks' handles over their local radii (owned
plus one halo radius each side) run one after another on one GPU -- no
collective is involved, so nothing waits on another launch -- and their
cycles and spectral post-processing equal the whole-shell handle's on every
owned radius, bit for bit (every stage is independent per radius; the radial
FDM rows see the same three radii)."""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_FP64, TIER_SPLIT_I8
from kemorin_mhd_b200.synthetic import make_d_rj
from tests.gpu_util import to_dev_fortran, from_dev_fortran

CFG = SphConfig(31, 48, 96, 13, name="L31_Nr13")


@pytest.mark.gpu
@pytest.mark.parametrize("tier", [TIER_FP64, TIER_SPLIT_I8], ids=["fp64", "split"])
@pytest.mark.parametrize("world", [2, 3])
def test_slab_cycles_and_post_processing_equal_whole_shell(tier, world):
    import torch
    from kemorin_mhd_b200.slabs import SlabTransform, radial_slab
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    J, n = cfg.J, cfg.J * cfg.nr
    d_np = make_d_rj(cfg, seed=61)
    # forward fields, then div(u T) (1 column), curl(u x B) (3), curl(omega x u) (3), div(omega x u) (1)
    ncol = cfg.ncf + 8

    def run(tr, d, nrows):
        out = torch.zeros((ncol, nrows), dtype=torch.float64, device="cuda")
        tr.nonlinear_cycle(d, out)
        tr.div_flux(out, 6, cfg.ncf)             # -div(u T) source
        tr.rot_induction(out, 3, cfg.ncf + 1)    # curl(u x B): 3 columns
        tr.rot_force(out, 0, cfg.ncf + 4)        # curl(omega x u), non-slip: 3 columns
        tr.div_force(out, 0, cfg.ncf + 7)
        return from_dev_fortran(out)

    whole = run(SphTransform(cfg, tier=tier), to_dev_fortran(d_np), n)
    for rank in range(world):
        s = radial_slab(cfg.nr, world, rank)
        st = SlabTransform(cfg, s, tier=tier)
        rows = slice(s.lo * J, s.hi * J)
        got = run(st.tr, to_dev_fortran(np.asfortranarray(d_np[rows])), J * s.nr_local)
        own = st.owned
        assert np.array_equal(got[own, :cfg.ncf], whole[s.r0 * J:s.r1 * J, :cfg.ncf]), rank
        assert np.array_equal(got[own, cfg.ncf:cfg.ncf + 8], whole[s.r0 * J:s.r1 * J, cfg.ncf:cfg.ncf + 8]), rank
        st.close()
