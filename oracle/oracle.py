"""ctypes wrapper of the CPU FP64 oracle -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg, always as the checker.  The product path never imports this module.
Parity status: unpinned against the reference's own outputs (see
kmhd_oracle.cpp header); pinned by invariants and scipy in tests/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "kmhd_oracle.cpp")
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = ctypes.CDLL(_LIB)
        _lib.oracle_create.restype = ctypes.c_void_p
        _lib.oracle_create.argtypes = [ctypes.c_int] * 4 + [_dp] + [ctypes.c_int] * 5 + \
            [_ip, _ip, _ip, _dp, ctypes.c_int]
        _lib.oracle_destroy.argtypes = [ctypes.c_void_p]
        _lib.oracle_J.restype = ctypes.c_longlong
        _lib.oracle_J.argtypes = [ctypes.c_void_p]
        _lib.oracle_tables.argtypes = [ctypes.c_void_p] + [_dp] * 7 + [_ip, _ip]
        _lib.oracle_b_trans.argtypes = [ctypes.c_void_p, _dp, ctypes.c_longlong, _ip, _dp]
        _lib.oracle_f_trans.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_longlong, _ip]
        _lib.oracle_cycle.argtypes = [ctypes.c_void_p, _dp, ctypes.c_longlong, _ip, _dp,
                                      ctypes.c_longlong, _ip]
        _lib.oracle_leg_bwd.argtypes = [ctypes.c_void_p, _dp, _dp]
        _lib.oracle_leg_fwd.argtypes = [ctypes.c_void_p, _dp, _dp]
        _lib.oracle_last_timing.argtypes = [_dp]
        _lib.oracle_set_dgemm.argtypes = [ctypes.c_void_p]
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def use_openblas(path: str | None = None) -> bool:
    """Route the oracle's DGEMMs to numpy's bundled OpenBLAS (single-threaded
    per calling thread), as the reference links BLAS DGEMM."""
    import glob
    if path is None:
        import numpy
        cands = glob.glob(os.path.join(os.path.dirname(numpy.__file__), os.pardir,
                                       "numpy.libs", "libscipy_openblas64_*.so"))
        if not cands:
            return False
        path = cands[0]
    blas = ctypes.CDLL(path)
    try:
        blas.scipy_openblas_set_num_threads64_(ctypes.c_int(1))
    except AttributeError:
        pass
    fn = ctypes.cast(blas.scipy_dgemm_64_, ctypes.c_void_p)
    lib().oracle_set_dgemm(fn)
    use_openblas._keep = blas
    return True


def use_builtin_dgemm():
    lib().oracle_set_dgemm(None)


class Oracle:
    """CPU FP64 restatement of the reference cycle for one configuration."""

    def __init__(self, cfg, nthreads: int | None = None, radius=None):
        self.cfg = cfg
        L = lib()
        r = np.ascontiguousarray(cfg.radius() if radius is None else radius, np.float64)
        kinds = np.asarray([p[0] for p in cfg.products], np.int32)
        pa = np.asarray([p[1] for p in cfg.products], np.int32)
        pb = np.asarray([p[2] for p in cfg.products], np.int32)
        pc = np.asarray([p[3] for p in cfg.products], np.float64)
        nthreads = nthreads or os.cpu_count() or 1
        self.nthreads = nthreads
        self._h = L.oracle_create(cfg.ltr, cfg.nth, cfg.nph, cfg.nr, _d(r), cfg.nvb, cfg.nsb,
                                  cfg.nvf, cfg.nsf, len(cfg.products), _i(kinds), _i(pa), _i(pb),
                                  _d(pc), nthreads)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().oracle_destroy(h)
            self._h = None

    @property
    def J(self):
        return int(lib().oracle_J(self._h))

    def tables(self):
        c = self.cfg
        J = self.J
        colat = np.zeros(c.nth)
        w = np.zeros(c.nth)
        P = np.zeros(J * c.nth)
        dP = np.zeros(J * c.nth)
        g3, g6, g7 = np.zeros(J), np.zeros(J), np.zeros(J)
        jl, jm = np.zeros(J, np.int32), np.zeros(J, np.int32)
        lib().oracle_tables(self._h, _d(colat), _d(w), _d(P), _d(dP), _d(g3), _d(g6), _d(g7),
                            _i(jl), _i(jm))
        return dict(colat=colat, weight=w, P=P.reshape(J, c.nth), dP=dP.reshape(J, c.nth),
                    g3=g3, g6=g6, g7=g7, l=jl, m=jm)

    def b_trans(self, d_rj: np.ndarray, cols=None) -> np.ndarray:
        """d_rj (J*Nr x ncol, F-order) -> fld_rtp (nnod_rtp x ncb, F-order)."""
        c = self.cfg
        d_rj = np.asfortranarray(d_rj, np.float64)
        cols = np.ascontiguousarray(c.cols_b() if cols is None else cols, np.int32)
        nnod = c.nr * c.nth * c.nph
        out = np.zeros((nnod, c.ncb), np.float64, order="F")
        lib().oracle_b_trans(self._h, _d(d_rj), d_rj.shape[0], _i(cols), _d(out))
        return out

    def f_trans(self, frc_rtp: np.ndarray, cols=None) -> np.ndarray:
        c = self.cfg
        frc_rtp = np.asfortranarray(frc_rtp, np.float64)
        cols = np.ascontiguousarray(c.cols_f() if cols is None else cols, np.int32)
        out = np.zeros((c.J * c.nr, c.ncf), np.float64, order="F")
        lib().oracle_f_trans(self._h, _d(frc_rtp), _d(out), out.shape[0], _i(cols))
        return out

    def cycle(self, d_rj: np.ndarray, cols_in=None, cols_out=None) -> np.ndarray:
        c = self.cfg
        d_rj = np.asfortranarray(d_rj, np.float64)
        ci = np.ascontiguousarray(c.cols_b() if cols_in is None else cols_in, np.int32)
        co = np.ascontiguousarray(c.cols_f() if cols_out is None else cols_out, np.int32)
        out = np.zeros((c.J * c.nr, c.ncf), np.float64, order="F")
        lib().oracle_cycle(self._h, _d(d_rj), d_rj.shape[0], _i(ci), _d(out), out.shape[0],
                           _i(co))
        return out

    def last_timing(self):
        t = np.zeros(5)
        lib().oracle_last_timing(_d(t))
        return dict(leg_bwd=t[0], fft_bwd=t[1], products=t[2], fft_fwd=t[3], leg_fwd=t[4])
