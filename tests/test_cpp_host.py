"""The C++ mirror of the reference entry points compiles against the C-ABI
(CPU) and matches the oracle when driven like the reference's MHD loop (GPU)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_sph_trans_mhd.cpp")
EXE = os.path.join(ROOT, "tests", "cpp", "test_sph_trans_mhd")


def build_driver():
    from kemorin_mhd_b200 import build as kbuild
    lib = kbuild.build()
    subprocess.check_call(["/usr/bin/g++", "-O2", "-std=c++17", SRC, "-o", EXE,
                           lib, "-ldl", f"-Wl,-rpath,{os.path.dirname(lib)}"])
    return EXE


def test_cpp_mirror_compiles():
    assert os.path.exists(build_driver())


@pytest.mark.gpu
@pytest.mark.parametrize("tier", [0, 1])
def test_cpp_mirror_cycle_matches_oracle(tier):
    from oracle import oracle
    exe = build_driver()
    r = subprocess.run([exe, oracle.build(), str(tier)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_mirror_spectral_steps_match_oracle(tmp_path):
    """The mirror driven through the spectral steps of a time step (vorticity
    and current, the cycle with the Coriolis curl, rot_momentum_eq_exp_sph,
    the buoyancy curl) on the full MHD field set equals the oracle chain on
    the same input columns (FP64 tier, <= 1e-12 of each result's maximum)."""
    import numpy as np
    from kemorin_mhd_b200.config import PROD_CROSS, PROD_DOT, PROD_VEC_SCALAR, SphConfig, chebyshev_radii, rj_order
    from oracle import oracle
    from oracle.oracle import Oracle
    from oracle.sph_coriolis import rot_coriolis
    from oracle.sph_div import current, div_flux, rot_buoyancy, rot_force, rot_uxb, vorticity
    exe = build_driver()
    out = str(tmp_path / "d_fld.bin")
    r = subprocess.run([exe, oracle.build(), "0", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    L, nr = 15, 6
    J = (L + 1) ** 2
    d = np.fromfile(out, dtype=np.float64).reshape(47, J * nr).T
    rad = chebyshev_radii(nr)
    l, m = rj_order(L)
    u, B, T, C = d[:, 0:3], d[:, 6:9], d[:, 12], d[:, 13]
    w = np.stack(vorticity(rad, l, u[:, 0], u[:, 1], u[:, 2]), 1)
    Jc = np.stack(current(rad, l, B[:, 0], B[:, 1], B[:, 2]), 1)
    cfg = SphConfig(L, 24, 48, nr, nvb=4, nsb=2, nvf=5, nsf=1,
                    products=((PROD_CROSS, 1, 0, 1.0), (PROD_CROSS, 3, 2, 1.0), (PROD_CROSS, 0, 2, 1.0),
                              (PROD_VEC_SCALAR, 0, 0, 1.0), (PROD_VEC_SCALAR, 0, 1, 1.0), (PROD_DOT, 0, 1, 1.0)))
    fw = Oracle(cfg, nthreads=4, radius=rad).cycle(np.asfortranarray(np.column_stack([u, w, B, Jc, T, C])))
    adv, lor, uxb, uT, uC = (fw[:, 3 * i:3 * i + 3] for i in range(5))
    ref = {3: w, 9: Jc, 14: fw[:, 0:16],
           30: np.stack(rot_force(rad, l, *adv.T), 1), 33: np.stack(rot_force(rad, l, *lor.T), 1),
           36: np.stack(rot_uxb(rad, l, *uxb.T), 1),
           39: div_flux(rad, l, uT[:, 0], uT[:, 1])[:, None], 40: div_flux(rad, l, uC[:, 0], uC[:, 1])[:, None],
           46: rot_buoyancy(rad, J, T, 3.0, C, -1.5)[:, None]}
    pol, tor = rot_coriolis(rad, L, l, m, u.T, w.T, 2.0e2)
    for c0, R in ref.items():
        got = d[:, c0:c0 + R.shape[1]]
        err = np.abs(got - R).max(axis=0) / np.maximum(np.abs(R).max(axis=0), 1e-300)
        assert err.max() <= 1e-12, (c0, err)
    for c0, R in ((41, pol), (43, tor)):
        assert np.abs(d[:, c0] - R).max() <= 1e-12 * np.abs(R).max(), c0
