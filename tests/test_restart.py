"""Spectral field files of the reference (kemorin_mhd_b200/restart.py): the
text layout of field_file_IO.f90 / field_data_IO.f90 / time_data_IO.f90 and
the binary layouts of field_file_IO_b.f90 (raw bytes or Fortran records,
either byte order), gzip or not."""
import gzip

import numpy as np
import pytest

from kemorin_mhd_b200 import restart


def _sample(nnod=37, seed=0):
    rng = np.random.default_rng(seed)
    names = ["velocity", "vorticity", "temperature", "magnetic_field"]
    ncomp = [3, 3, 1, 3]
    d = rng.standard_normal((nnod, sum(ncomp))) * np.logspace(-150, 150, nnod)[:, None]
    return restart.from_d_rj(d, names, ncomp, rank=3, step=120, time=1.25e-2, dt=2.5e-5)


@pytest.mark.parametrize("name", ["rst.120.3.fst", "rst.120.3.fst.gz"])
def test_text_round_trip(tmp_path, name):
    f = _sample()
    p = str(tmp_path / name)
    restart.write(p, f)
    g = restart.read(p)
    assert (g.rank, g.step, g.names, g.ncomp) == (3, 120, f.names, f.ncomp)
    assert g.time == f.time and g.dt == f.dt
    # 1pE25.15e3 keeps 16 significant digits
    assert np.all(np.abs(g.data - f.data) <= 1e-15 * np.abs(f.data))


@pytest.mark.parametrize("records", [False, True], ids=["raw", "fortran_records"])
@pytest.mark.parametrize("byteorder", ["<", ">"], ids=["little", "big"])
@pytest.mark.parametrize("gz", [False, True], ids=["plain", "gzip"])
def test_binary_round_trip_exact(tmp_path, records, byteorder, gz):
    f = _sample(seed=1)
    p = str(tmp_path / ("rst.120.3.fsb" + (".gz" if gz else "")))
    restart.write_binary(p, f, records=records, byteorder=byteorder)
    g = restart.read(p)
    assert (g.rank, g.step, g.time, g.dt, g.names, g.ncomp) == (f.rank, f.step, f.time, f.dt, f.names, f.ncomp)
    assert np.array_equal(g.data, f.data)


def test_text_in_the_reference_layout(tmp_path):
    """A file laid out as the reference's writer lays it out: comment lines,
    i16 / 1pE25.15e3 / 2i16 / 10i5 formats, eleven component counts over two
    lines, one line of components per node; and a time line without dt."""
    ncomp = [1] * 11
    lines = ["!  domain ID", "%16d" % 0, "!  time step number", "%16d" % 7, "!  time, Delta t",
             "  1.000000000000000E-001",
             "! Number of field and component", "%16d%16d" % (2, 11),
             "".join("%5d" % c for c in ncomp[:10]), "".join("%5d" % c for c in ncomp[10:])]
    for i in range(11):
        lines += ["# a comment line", "field_%d" % i, " -1.500000000000000E+000", "  2.000000000000000E-300"]
    p = tmp_path / "snap.7.0.fst"
    p.write_text("\n".join(lines) + "\n")
    g = restart.read(str(p))
    assert g.step == 7 and g.time == 0.1 and g.dt == 0.0 and g.ncomp == ncomp and g.nnod == 2
    assert g.names == ["field_%d" % i for i in range(11)]
    assert np.array_equal(g.data, np.tile([[-1.5], [2e-300]], (1, 11)))


def test_d_rj_columns_and_file_names():
    f = _sample()
    d = f.d_rj(["temperature", "velocity"])
    assert d.flags.f_contiguous and d.shape == (f.nnod, 4)
    assert np.array_equal(d[:, 0], f.data[:, 6]) and np.array_equal(d[:, 1:], f.data[:, 0:3])
    assert restart.file_name("rst", 12, 5) == "rst.12.5.fst"
    assert restart.file_name("rst", 12, 5, "gz_binary") == "rst.12.5.fsb.gz"


def test_truncated_binary_is_an_error(tmp_path):
    f = _sample()
    p = str(tmp_path / "t.fsb")
    restart.write_binary(p, f)
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[:-8])
    with pytest.raises(ValueError):
        restart.read(p)
