"""Spectral divergence of a flux vector (kmhd_sph_div_flux) against the CPU
oracle of the reference's const_sph_scalar_advect with fixed-field
boundaries (oracle/sph_div.py): max-norm relative error <= 1e-13, device and
host pointers; and on the heat flux uT produced by the split-tier cycle."""
import numpy as np
import pytest

from kemorin_mhd_b200.config import SphConfig, TIER_FP64, TIER_SPLIT_I8, rj_order
from kemorin_mhd_b200.synthetic import make_d_rj
from oracle.sph_div import div_flux
from tests.gpu_util import to_dev_fortran, from_dev_fortran

CFG = SphConfig(31, 48, 96, 9, name="L31")


def _relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True], ids=["device", "host"])
def test_div_flux_matches_oracle(host):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    n = cfg.J * cfg.nr
    rng = np.random.default_rng(7)
    d = np.asfortranarray(rng.standard_normal((n, 4)))
    fin, fout = rng.standard_normal(cfg.J), rng.standard_normal(cfg.J)
    l, _ = rj_order(cfg.ltr)
    ref = div_flux(cfg.radius(), l, d[:, 1], d[:, 2], fin, fout)
    if host:
        arr = d.copy(order="F")
        tr.div_flux(arr, 1, 3, fin, fout)
        got = arr[:, 3]
        assert np.array_equal(arr[:, :3], d[:, :3])
    else:
        t = to_dev_fortran(d)
        tr.div_flux(t, 1, 3, torch.from_numpy(fin).cuda(), torch.from_numpy(fout).cuda())
        got = from_dev_fortran(t)[:, 3]
    assert _relerr(got, ref) <= 1e-13


@pytest.mark.gpu
def test_div_flux_rejects_overlapping_columns():
    import torch
    from kemorin_mhd_b200.sph_trans import KmhdError, SphTransform
    tr = SphTransform(CFG, tier=TIER_FP64)
    t = torch.zeros((4, CFG.J * CFG.nr), dtype=torch.float64, device="cuda")
    for col_div in (1, 2):
        with pytest.raises(KmhdError):
            tr.div_flux(t, 1, col_div)


@pytest.mark.gpu
def test_heat_advection_after_split_cycle():
    """-div(u T) from the cycle's heat-flux output, GPU end to end, against the
    oracle applied to the same uT spectra."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_SPLIT_I8)
    d = to_dev_fortran(make_d_rj(cfg, seed=8))
    out = torch.zeros((cfg.ncf + 1, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(d, out)                      # columns: omega x u (0-2), u x B (3-5), uT (6-8), u.omega (9)
    uT = from_dev_fortran(out)[:, 6:9].copy()
    tr.div_flux(out, 6, cfg.ncf)                    # div(uT) into the spare column
    got = from_dev_fortran(out)[:, cfg.ncf]
    l, _ = rj_order(cfg.ltr)
    ref = div_flux(cfg.radius(), l, uT[:, 0], uT[:, 1])
    assert _relerr(got, ref) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True], ids=["device", "host"])
def test_rot_induction_matches_oracle(host):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_div import rot_uxb
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    n = cfg.J * cfg.nr
    rng = np.random.default_rng(11)
    d = np.asfortranarray(rng.standard_normal((n, 7)))
    l, _ = rj_order(cfg.ltr)
    ref = np.stack(rot_uxb(cfg.radius(), l, d[:, 0], d[:, 1], d[:, 2]), axis=1)
    if host:
        arr = d.copy(order="F")
        tr.rot_induction(arr, 0, 4)
        got = arr[:, 4:7]
        assert np.array_equal(arr[:, :4], d[:, :4])
    else:
        t = to_dev_fortran(d)
        tr.rot_induction(t, 0, 4)
        got = from_dev_fortran(t)[:, 4:7]
    for q in range(3):
        assert _relerr(got[:, q], ref[:, q]) <= 1e-13, q


@pytest.mark.gpu
def test_induction_after_split_cycle():
    """curl(u x B) from the cycle's u x B output (columns 3-5), on the GPU."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_div import rot_uxb
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_SPLIT_I8)
    d = to_dev_fortran(make_d_rj(cfg, seed=12))
    out = torch.zeros((cfg.ncf + 3, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(d, out)
    uxb = from_dev_fortran(out)[:, 3:6].copy()
    tr.rot_induction(out, 3, cfg.ncf)
    got = from_dev_fortran(out)[:, cfg.ncf:cfg.ncf + 3]
    l, _ = rj_order(cfg.ltr)
    ref = rot_uxb(cfg.radius(), l, uxb[:, 0], uxb[:, 1], uxb[:, 2])
    for q in range(3):
        assert _relerr(got[:, q], ref[q]) <= 1e-13, q


@pytest.mark.gpu
@pytest.mark.parametrize("bc_icb,bc_cmb,host", [(0, 0, False), (1, 1, False), (0, 1, True), (1, 0, False)],
                         ids=["non_slip", "free_slip", "mixed_host", "free_in_non_slip_out"])
def test_rot_force_matches_oracle(bc_icb, bc_cmb, host):
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_div import FREE_SLIP, NON_SLIP, rot_force
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    n = cfg.J * cfg.nr
    rng = np.random.default_rng(13 + bc_icb + 2 * bc_cmb)
    d = np.asfortranarray(rng.standard_normal((n, 6)))
    l, _ = rj_order(cfg.ltr)
    names = {0: NON_SLIP, 1: FREE_SLIP}
    ref = rot_force(cfg.radius(), l, d[:, 0], d[:, 1], d[:, 2], names[bc_icb], names[bc_cmb])
    if host:
        arr = d.copy(order="F")
        tr.rot_force(arr, 0, 3, bc_icb, bc_cmb)
        got = arr[:, 3:6]
        assert np.array_equal(arr[:, :3], d[:, :3])
    else:
        t = to_dev_fortran(d)
        tr.rot_force(t, 0, 3, bc_icb, bc_cmb)
        got = from_dev_fortran(t)[:, 3:6]
    for q in range(3):
        assert _relerr(got[:, q], ref[q]) <= 1e-13, q


@pytest.mark.gpu
def test_rot_force_rejects_unknown_condition():
    import torch
    from kemorin_mhd_b200.sph_trans import KmhdError, SphTransform
    tr = SphTransform(CFG, tier=TIER_FP64)
    t = torch.zeros((6, CFG.J * CFG.nr), dtype=torch.float64, device="cuda")
    with pytest.raises(KmhdError):
        tr.rot_force(t, 0, 3, 2, 0)
    with pytest.raises(KmhdError):
        tr.rot_force(t, 0, 2)      # overlapping columns


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True], ids=["device", "host"])
def test_div_force_matches_oracle(host):
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_div import div_force
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    n = cfg.J * cfg.nr
    rng = np.random.default_rng(17)
    d = np.asfortranarray(rng.standard_normal((n, 3)))
    l, _ = rj_order(cfg.ltr)
    ref = div_force(cfg.radius(), l, d[:, 0], d[:, 1])
    if host:
        arr = d.copy(order="F")
        tr.div_force(arr, 0, 2)
        got = arr[:, 2]
    else:
        t = to_dev_fortran(d)
        tr.div_force(t, 0, 2)
        got = from_dev_fortran(t)[:, 2]
    assert _relerr(got, ref) <= 1e-13


@pytest.mark.gpu
def test_vorticity_source_after_split_cycle():
    """curl and div of the advection force omega x u (cycle columns 0-2),
    non-slip boundaries, on the GPU against the oracle on the same spectra."""
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_div import div_force, rot_force
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_SPLIT_I8)
    d = to_dev_fortran(make_d_rj(cfg, seed=14))
    out = torch.zeros((cfg.ncf + 4, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")
    tr.nonlinear_cycle(d, out)
    adv = from_dev_fortran(out)[:, 0:3].copy()
    tr.rot_force(out, 0, cfg.ncf)
    tr.div_force(out, 0, cfg.ncf + 3)
    res = from_dev_fortran(out)
    l, _ = rj_order(cfg.ltr)
    ref = rot_force(cfg.radius(), l, adv[:, 0], adv[:, 1], adv[:, 2])
    for q in range(3):
        assert _relerr(res[:, cfg.ncf + q], ref[q]) <= 1e-13, q
    assert _relerr(res[:, cfg.ncf + 3], div_force(cfg.radius(), l, adv[:, 0], adv[:, 1])) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("bc_icb,bc_cmb,host", [(1, 1, False), (0, 1, True), (1, 0, False)],
                         ids=["flux_flux", "field_flux_host", "flux_field"])
def test_div_flux_bc_matches_oracle(bc_icb, bc_cmb, host):
    import torch
    from kemorin_mhd_b200.sph_trans import SphTransform
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    n = cfg.J * cfg.nr
    rng = np.random.default_rng(19)
    d = np.asfortranarray(rng.standard_normal((n, 3)))
    vi, vo = rng.standard_normal(cfg.J), rng.standard_normal(cfg.J)
    l, _ = rj_order(cfg.ltr)
    names = {0: "field", 1: "flux"}
    ref = div_flux(cfg.radius(), l, d[:, 0], d[:, 1], vi, vo, names[bc_icb], names[bc_cmb])
    if host:
        arr = d.copy(order="F")
        tr.div_flux_bc(arr, 0, 2, bc_icb, bc_cmb, vi, vo)
        got = arr[:, 2]
    else:
        t = to_dev_fortran(d)
        tr.div_flux_bc(t, 0, 2, bc_icb, bc_cmb, torch.from_numpy(vi).cuda(), torch.from_numpy(vo).cuda())
        got = from_dev_fortran(t)[:, 2]
    assert _relerr(got, ref) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("bc_icb,bc_cmb", [(1, 1), (0, 1), (1, 0)], ids=["qvac_qvac", "ins_qvac", "qvac_ins"])
def test_rot_induction_bc_matches_oracle(bc_icb, bc_cmb):
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_div import rot_uxb
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    n = cfg.J * cfg.nr
    d = np.asfortranarray(np.random.default_rng(20).standard_normal((n, 6)))
    l, _ = rj_order(cfg.ltr)
    names = {0: "insulator", 1: "pseudo_vacuum"}
    ref = rot_uxb(cfg.radius(), l, d[:, 0], d[:, 1], d[:, 2], names[bc_icb], names[bc_cmb])
    t = to_dev_fortran(d)
    tr.rot_induction_bc(t, 0, 3, bc_icb, bc_cmb)
    got = from_dev_fortran(t)
    for q in range(3):
        assert _relerr(got[:, 3 + q], ref[q]) <= 1e-13, q


@pytest.mark.gpu
@pytest.mark.parametrize("which,bc_icb,bc_cmb,host", [("vort", 0, 0, False), ("vort", 1, 0, True),
                                                      ("cur", 0, 0, False), ("cur", 1, 0, False),
                                                      ("cur", 0, 1, True)],
                         ids=["vort_nonslip", "vort_free_nonslip_host", "cur_ins", "cur_qvac_ins",
                              "cur_ins_qvac_host"])
def test_vorticity_current_match_oracle(which, bc_icb, bc_cmb, host):
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_div import FREE_SLIP, INSULATOR, NON_SLIP, PSEUDO_VACUUM, current, vorticity
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    n = cfg.J * cfg.nr
    d = np.asfortranarray(np.random.default_rng(23).standard_normal((n, 6)))
    l, _ = rj_order(cfg.ltr)
    if which == "vort":
        names = {0: NON_SLIP, 1: FREE_SLIP}
        ref = vorticity(cfg.radius(), l, d[:, 0], d[:, 1], d[:, 2], names[bc_icb], names[bc_cmb])
        call = tr.vorticity
    else:
        names = {0: INSULATOR, 1: PSEUDO_VACUUM}
        ref = current(cfg.radius(), l, d[:, 0], d[:, 1], d[:, 2], names[bc_icb], names[bc_cmb])
        call = tr.current
    if host:
        arr = d.copy(order="F")
        call(arr, 0, 3, bc_icb, bc_cmb)
        got = arr
    else:
        t = to_dev_fortran(d)
        call(t, 0, 3, bc_icb, bc_cmb)
        got = from_dev_fortran(t)
    for q in range(3):
        assert _relerr(got[:, 3 + q], ref[q]) <= 1e-13, q


@pytest.mark.gpu
@pytest.mark.parametrize("double,host", [(False, False), (True, False), (True, True)],
                         ids=["thermal", "double", "double_host"])
def test_rot_buoyancy_matches_oracle(double, host):
    from kemorin_mhd_b200.sph_trans import SphTransform
    from oracle.sph_div import rot_buoyancy
    cfg = CFG
    tr = SphTransform(cfg, tier=TIER_FP64)
    n = cfg.J * cfg.nr
    d = np.asfortranarray(np.random.default_rng(24).standard_normal((n, 3)))
    ref = rot_buoyancy(cfg.radius(), cfg.J, d[:, 0], 2.5, d[:, 1] if double else None, -0.75)
    kw = dict(col_c=1, coef_c=-0.75) if double else {}
    if host:
        arr = d.copy(order="F")
        tr.rot_buoyancy(arr, 0, 2.5, 2, **kw)
        got = arr[:, 2]
    else:
        t = to_dev_fortran(d)
        tr.rot_buoyancy(t, 0, 2.5, 2, **kw)
        got = from_dev_fortran(t)[:, 2]
    assert _relerr(got, ref) <= 1e-14
