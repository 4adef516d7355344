"""Spectral field files (restart and snapshot data) of the reference, so that
dynamo states it wrote can be transformed here, and the transform's outputs
written in the same formats.

Formats, as the reference writes them (file `<prefix>.<step>.<rank>.fst`
text, `.fsb` binary, `.gz` gzip of either; set_SPH_fld_file_name,
CORE_src/IO/set_field_file_names.f90:136-175):

- text (write_step_field_file / read_and_alloc_step_field,
  CORE_src/IO/field_file_IO.f90:51-187; write_step_data / read_step_data,
  time_data_IO.f90:97-138; write_field_data / read_field_data,
  field_data_IO.f90:321-389): comment lines start with '!' or '#';
  rank (i16), step (i16), time and dt (1p E25.15e3); nnod and the field count
  (2i16); the component counts (10i5 per line); per field its name, then nnod
  lines of its components;
- binary (write_step_field_file_b, CORE_src/IO_BINARY/field_file_IO_b.f90:46-69;
  field_data_IO_b.f90:37-118; binary_IO.F90): an endian flag int32 'UNIX',
  rank int32, step int32, time f64, dt f64, nnod int64, field count int32,
  component counts int32[n], names char[255][n] (blank padded), data f64
  (nnod, ntot) column-major -- either as raw bytes (the build with zlib IO)
  or as Fortran unformatted records (4-byte length markers around each
  write); both are read, the flag gives the byte order.

The data rows are the rank's rj nodes, inod = j + J (k - 1): the d_rj layout
the transform takes.
"""
from __future__ import annotations

import dataclasses
import gzip
import io
import itertools
import struct
from typing import Dict, List, Sequence

import numpy as np

KCHARA = 255
I_UNIX = (ord("U") << 24) | (ord("N") << 16) | (ord("I") << 8) | ord("X")


@dataclasses.dataclass
class SphFieldFile:
    rank: int
    step: int
    time: float
    dt: float
    names: List[str]
    ncomp: List[int]
    data: np.ndarray            # (nnod, sum(ncomp)), float64, column-major

    @property
    def nnod(self) -> int:
        return int(self.data.shape[0])

    def field(self, name: str) -> np.ndarray:
        """The components of one field, (nnod, ncomp)."""
        i = self.names.index(name)
        c0 = int(sum(self.ncomp[:i]))
        return self.data[:, c0:c0 + self.ncomp[i]]

    def d_rj(self, names: Sequence[str]) -> np.ndarray:
        """The named fields side by side, column-major: the transform's input
        array with the fields' first columns at the running component sums."""
        return np.asfortranarray(np.concatenate([self.field(n) for n in names], axis=1))


def file_name(prefix: str, step: int, rank: int, fmt: str = "text") -> str:
    """`<prefix>.<step>.<rank>` plus `.fst`, `.fsb`, `.fst.gz` or `.fsb.gz`."""
    ext = {"text": ".fst", "binary": ".fsb", "gz_text": ".fst.gz", "gz_binary": ".fsb.gz"}[fmt]
    return "%s.%d.%d%s" % (prefix, step, rank, ext)


# ---------------------------------------------------------------- text
def _fortran_e(x: float) -> str:
    """1pE25.15e3: one digit before the point, 15 after, a 3-digit exponent."""
    if not np.isfinite(x):
        return "%25s" % ("NaN" if np.isnan(x) else ("Infinity" if x > 0 else "-Infinity"))
    m, e = ("%.15E" % x).split("E")
    return "%25s" % ("%sE%s%03d" % (m, "-" if int(e) < 0 else "+", abs(int(e))))


def write_text(path: str, f: SphFieldFile) -> None:
    op = gzip.open if path.endswith(".gz") else open
    with op(path, "wt") as fh:
        fh.write("!  domain ID\n%16d\n!  time step number\n%16d\n!  time, Delta t\n" % (f.rank, f.step))
        fh.write(_fortran_e(f.time) + _fortran_e(f.dt) + "\n")
        fh.write("! Number of field and component\n%16d%16d\n" % (f.nnod, len(f.names)))
        for i in range(0, len(f.ncomp), 10):
            fh.write("".join("%5d" % c for c in f.ncomp[i:i + 10]) + "\n")
        c0 = 0
        for name, nc in zip(f.names, f.ncomp):
            fh.write(name + "\n")
            block = f.data[:, c0:c0 + nc]
            fh.write("\n".join("".join(_fortran_e(v) for v in row) for row in block) + "\n")
            c0 += nc


def _next_data_line(fh) -> str:
    """The next line that is neither blank nor a comment (skip_comment)."""
    for line in fh:
        s = line.strip()
        if s and s[0] not in "!#":
            return s
    raise ValueError("unexpected end of field file")


def _read_text(fh) -> SphFieldFile:
    rank = int(_next_data_line(fh).split()[0])
    step = int(_next_data_line(fh).split()[0])
    tv = _next_data_line(fh).split()
    time = float(tv[0].replace("D", "E"))
    dt = float(tv[1].replace("D", "E")) if len(tv) > 1 else 0.0
    nnod, nfld = (int(x) for x in _next_data_line(fh).split()[:2])
    ncomp: List[int] = []
    while len(ncomp) < nfld:                       # list-directed: may span lines
        ncomp += [int(x) for x in fh.readline().split()]
    ncomp = ncomp[:nfld]
    data = np.empty((nnod, sum(ncomp)), order="F")
    names, c0 = [], 0
    for nc in ncomp:
        names.append(_next_data_line(fh).split()[0])
        text = "".join(itertools.islice(fh, nnod)).replace("D", "E").replace("d", "e")
        vals = np.array(text.split(), dtype=np.float64)
        if vals.size != nnod * nc:
            raise ValueError("field %s: %d values for %d nodes x %d components" % (names[-1], vals.size, nnod, nc))
        data[:, c0:c0 + nc] = vals.reshape(nnod, nc)
        c0 += nc
    return SphFieldFile(rank, step, time, dt, names, ncomp, data)


# ---------------------------------------------------------------- binary
def write_binary(path: str, f: SphFieldFile, records: bool = False, byteorder: str = "<") -> None:
    """Raw bytes (records=False, the zlib-IO build) or Fortran unformatted
    records (records=True)."""
    bo = byteorder
    items = [struct.pack(bo + "i", I_UNIX), struct.pack(bo + "i", f.rank), struct.pack(bo + "i", f.step),
             struct.pack(bo + "d", f.time), struct.pack(bo + "d", f.dt), struct.pack(bo + "q", f.nnod),
             struct.pack(bo + "i", len(f.names)),
             struct.pack(bo + "%di" % len(f.ncomp), *f.ncomp),
             b"".join(n.encode().ljust(KCHARA, b" ") for n in f.names),
             np.asfortranarray(f.data, dtype=np.dtype(bo + "f8")).tobytes(order="F")]
    op = gzip.open if path.endswith(".gz") else open
    with op(path, "wb") as fh:
        for it in items:
            if records:
                fh.write(struct.pack(bo + "i", len(it)) + it + struct.pack(bo + "i", len(it)))
            else:
                fh.write(it)


class _Reader:
    def __init__(self, buf: bytes):
        self.b, self.p = buf, 0
        flag_le = struct.unpack_from("<i", buf, 0)[0]
        flag_be = struct.unpack_from(">i", buf, 0)[0]
        self.records = False
        if I_UNIX not in (flag_le, flag_be):
            # a 4-byte record marker first: Fortran unformatted records
            self.records = True
            flag_le = struct.unpack_from("<i", buf, 4)[0]
            flag_be = struct.unpack_from(">i", buf, 4)[0]
            if I_UNIX not in (flag_le, flag_be):
                raise ValueError("not a binary field file (no endian flag)")
        self.bo = "<" if flag_le == I_UNIX else ">"

    def take(self, n: int) -> bytes:
        if self.records:
            ln = struct.unpack_from(self.bo + "i", self.b, self.p)[0]
            if ln != n:
                raise ValueError("record of %d bytes where %d expected" % (ln, n))
            self.p += 4
        out = self.b[self.p:self.p + n]
        if len(out) != n:
            raise ValueError("unexpected end of binary field file")
        self.p += n + (4 if self.records else 0)
        return out

    def ints(self, n: int, fmt: str = "i"):
        size = struct.calcsize(fmt)
        return struct.unpack(self.bo + "%d%s" % (n, fmt), self.take(n * size))


def _read_binary(buf: bytes) -> SphFieldFile:
    r = _Reader(buf)
    r.take(4)                                       # endian flag
    rank, = r.ints(1)
    step, = r.ints(1)
    time, = struct.unpack(r.bo + "d", r.take(8))
    dt, = struct.unpack(r.bo + "d", r.take(8))
    nnod, = r.ints(1, "q")
    nfld, = r.ints(1)
    ncomp = list(r.ints(nfld))
    raw = r.take(KCHARA * nfld)
    names = [raw[i * KCHARA:(i + 1) * KCHARA].decode(errors="replace").strip() for i in range(nfld)]
    ntot = sum(ncomp)
    data = np.frombuffer(r.take(8 * nnod * ntot), dtype=np.dtype(r.bo + "f8"))
    data = np.asfortranarray(data.reshape((nnod, ntot), order="F").astype(np.float64))
    return SphFieldFile(rank, step, time, dt, names, ncomp, data)


# ---------------------------------------------------------------- entry
def read(path: str) -> SphFieldFile:
    """Reads a text or binary field file, gzip-compressed or not (detected
    from the content, not the name)."""
    with open(path, "rb") as fh:
        head = fh.read(2)
    op = gzip.open if head == b"\x1f\x8b" else open
    with op(path, "rb") as fh:
        buf = fh.read()
    try:
        return _read_binary(buf)
    except (ValueError, struct.error):
        return _read_text(io.StringIO(buf.decode("ascii", errors="replace")))


def write(path: str, f: SphFieldFile, fmt: str | None = None) -> None:
    """Writes in the format the name asks for (.fst text, .fsb binary, + .gz)."""
    fmt = fmt or ("binary" if ".fsb" in path else "text")
    (write_binary if fmt == "binary" else write_text)(path, f)


def from_d_rj(d_rj: np.ndarray, names: Sequence[str], ncomp: Sequence[int], rank: int = 0, step: int = 0,
              time: float = 0.0, dt: float = 0.0) -> SphFieldFile:
    """A field file holding the columns of d_rj as the named fields."""
    d = np.asfortranarray(d_rj, dtype=np.float64)
    if d.shape[1] != sum(ncomp):
        raise ValueError("%d columns for %d components" % (d.shape[1], sum(ncomp)))
    return SphFieldFile(rank, step, float(time), float(dt), list(names), [int(c) for c in ncomp], d)
