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
