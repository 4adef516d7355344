"""Host-side mirror of the reference's transform entry points over the C-ABI.

``SphTransform.sph_b_trans`` / ``sph_f_trans`` stand in for
sph_b_trans_w_coriolis / sph_f_trans_w_coriolis (MHD_src/sph_MHD/sph_trans_w_coriols.f90:113,189)
and ``nonlinear_cycle`` for the transform segment of nonlinear_by_pseudo_sph
(MHD_src/sph_MHD/cal_nonlinear.f90:118-171).  Arrays keep the reference's
layouts: d_rj is (J*Nr, ncol) column-major; fld_rtp / frc_rtp are
(Nr*Ntheta*Nphi, ncomp) column-major with r fastest.  Torch CUDA tensors are
passed as device pointers; numpy arrays as host pointers (copies are then
part of the call).  Errors raise ``KmhdError`` with the C-ABI status text;
the reference aborts instead.

There is no CPU fallback: if the extension cannot be loaded the import fails.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

from .config import SphConfig

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "libkmhd_sph.so")

KMHD_PTR_DEVICE = 0
KMHD_PTR_HOST = 1
# kmhd_sph_desc.flags bits (include/kmhd_sph.h)
FLAG_AUTOTUNE = 1
FLAG_P_ON_THE_FLY = 2
BC_NON_SLIP = 0       # KMHD_BC_NON_SLIP
BC_FREE_SLIP = 1      # KMHD_BC_FREE_SLIP
BC_FIXED_FIELD = 0    # KMHD_BC_FIXED_FIELD
BC_FIXED_FLUX = 1     # KMHD_BC_FIXED_FLUX
BC_INSULATOR = 0      # KMHD_BC_INSULATOR
BC_PSEUDO_VACUUM = 1  # KMHD_BC_PSEUDO_VACUUM


class KmhdError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {status} ({strerror(status)})")


class Product(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("a", ctypes.c_int32), ("b", ctypes.c_int32),
                ("coef", ctypes.c_double)]


class Desc(ctypes.Structure):
    _fields_ = [("ltr", ctypes.c_int32), ("nth", ctypes.c_int32), ("nph", ctypes.c_int32),
                ("nr", ctypes.c_int32), ("radius", ctypes.POINTER(ctypes.c_double)),
                ("idx_rj_lm", ctypes.POINTER(ctypes.c_int32)),
                ("nvector_b", ctypes.c_int32), ("nscalar_b", ctypes.c_int32),
                ("nvector_f", ctypes.c_int32), ("nscalar_f", ctypes.c_int32),
                ("nproduct", ctypes.c_int32), ("products", ctypes.POINTER(Product)),
                ("tier", ctypes.c_int32), ("nslice", ctypes.c_int32), ("device", ctypes.c_int32),
                ("flags", ctypes.c_int32)]


EXPORTS = ["kmhd_sph_create", "kmhd_sph_destroy", "kmhd_sph_set_stream", "kmhd_sph_b_trans",
           "kmhd_sph_f_trans", "kmhd_sph_cycle", "kmhd_sph_batch_cycle", "kmhd_sph_last_timing",
           "kmhd_sph_get_tables", "kmhd_sph_device_bytes", "kmhd_strerror", "kmhd_sph_cycle_noalloc",
           "kmhd_sph_last_kernel_timing", "kmhd_sph_get_path", "kmhd_selftest_wait_timeout",
           "kmhd_sph_div_flux", "kmhd_sph_rot_induction", "kmhd_sph_rot_force", "kmhd_sph_div_force",
           "kmhd_sph_rot_coriolis", "kmhd_sph_set_coriolis", "kmhd_sph_b_trans_pole",
           "kmhd_sph_div_flux_bc", "kmhd_sph_rot_induction_bc", "kmhd_sph_vorticity", "kmhd_sph_current",
           "kmhd_sph_rot_buoyancy", "kmhd_sph_get_tuning", "kmhd_sph_set_products", "kmhd_sph_b_trans_center"]

_lib = None


def load_library(path: str | None = None):
    """Loads libkmhd_sph.so (built by kemorin_mhd_b200.build); raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or _LIBPATH
    if not os.path.exists(path):
        raise ImportError(f"CUDA extension not built: {path} (run kemorin_mhd_b200/build.py)")
    lib = ctypes.CDLL(path)
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
    ip = ctypes.POINTER(ctypes.c_int32)
    lib.kmhd_sph_create.argtypes = [ctypes.POINTER(Desc), ctypes.POINTER(vp)]
    lib.kmhd_sph_destroy.argtypes = [vp]
    lib.kmhd_sph_set_stream.argtypes = [vp, vp]
    lib.kmhd_sph_b_trans.argtypes = [vp, vp, i64, ip, vp, i32]
    lib.kmhd_sph_f_trans.argtypes = [vp, vp, vp, i64, ip, i32]
    lib.kmhd_sph_cycle.argtypes = [vp, vp, i64, ip, vp, i64, ip, i32]
    lib.kmhd_sph_batch_cycle.argtypes = [ctypes.POINTER(vp), i32, ctypes.POINTER(vp),
                                         ctypes.POINTER(i64), ctypes.POINTER(ip),
                                         ctypes.POINTER(vp), ctypes.POINTER(i64), ctypes.POINTER(ip)]
    lib.kmhd_sph_last_timing.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    lib.kmhd_sph_last_kernel_timing.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    lib.kmhd_sph_get_path.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    lib.kmhd_sph_get_tuning.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                        ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)]
    lib.kmhd_sph_set_products.argtypes = [vp, i32]
    lib.kmhd_sph_div_flux.argtypes = [vp, vp, i64, i32, i32, vp, vp, i32]
    lib.kmhd_sph_rot_induction.argtypes = [vp, vp, i64, i32, i32, i32]
    lib.kmhd_sph_rot_force.argtypes = [vp, vp, i64, i32, i32, i32, i32, i32]
    lib.kmhd_sph_div_force.argtypes = [vp, vp, i64, i32, i32, i32]
    lib.kmhd_sph_rot_coriolis.argtypes = [vp, vp, i64, i32, i32, i32, ctypes.c_double, i32]
    lib.kmhd_sph_set_coriolis.argtypes = [vp, ctypes.c_double, i32, i32, i32]
    lib.kmhd_sph_b_trans_pole.argtypes = [vp, vp, i64, vp, vp, i32]
    lib.kmhd_sph_b_trans_center.argtypes = [vp, vp, i64, vp, vp, i32]
    lib.kmhd_sph_div_flux_bc.argtypes = [vp, vp, i64, i32, i32, i32, i32, vp, vp, i32]
    lib.kmhd_sph_rot_induction_bc.argtypes = [vp, vp, i64, i32, i32, i32, i32, i32]
    lib.kmhd_sph_vorticity.argtypes = [vp, vp, i64, i32, i32, i32, i32, i32]
    lib.kmhd_sph_current.argtypes = [vp, vp, i64, i32, i32, i32, i32, i32]
    lib.kmhd_sph_rot_buoyancy.argtypes = [vp, vp, i64, i32, ctypes.c_double, i32, ctypes.c_double, i32, i32]
    lib.kmhd_selftest_wait_timeout.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.kmhd_sph_get_tables.argtypes = [vp, i32] + [ctypes.POINTER(ctypes.c_double)] * 4
    lib.kmhd_sph_device_bytes.restype = i64
    lib.kmhd_sph_device_bytes.argtypes = [vp]
    lib.kmhd_sph_cycle_noalloc.argtypes = [ctypes.POINTER(Desc), vp, i64, ip, vp, i64, ip, vp]
    lib.kmhd_strerror.restype = ctypes.c_char_p
    lib.kmhd_strerror.argtypes = [ctypes.c_int]
    _lib = lib
    return lib


def strerror(status: int) -> str:
    return load_library().kmhd_strerror(status).decode()


def _check(st: int, where: str):
    if st != 0:
        raise KmhdError(st, where)


def _ptr(a):
    """(address, ptr_kind) of a torch tensor or numpy array."""
    try:
        import torch
        if isinstance(a, torch.Tensor):
            if not a.is_cuda:
                if not a.is_contiguous():
                    raise ValueError("host tensor must be contiguous")
                return a.data_ptr(), KMHD_PTR_HOST
            return a.data_ptr(), KMHD_PTR_DEVICE
    except ImportError:
        pass
    if isinstance(a, np.ndarray):
        return a.ctypes.data, KMHD_PTR_HOST
    raise TypeError(type(a))


def _i32(seq):
    arr = (ctypes.c_int32 * len(seq))(*[int(x) for x in seq])
    return arr


class SphTransform:
    """One transform instance on one GPU (handle of the C-ABI)."""

    def __init__(self, cfg: SphConfig, tier: int = 0, nslice: int = 0, device: int = 0,
                 radius=None, idx_rj_lm=None, autotune: bool = False, p_on_the_fly: bool = False):
        lib = load_library()
        self.cfg = cfg
        self.tier = tier
        r = np.ascontiguousarray(cfg.radius() if radius is None else radius, np.float64)
        self._r = r
        prods = (Product * max(1, len(cfg.products)))(
            *[Product(int(k), int(a), int(b), float(c)) for (k, a, b, c) in cfg.products])
        self._prods = prods
        d = Desc()
        d.ltr, d.nth, d.nph, d.nr = cfg.ltr, cfg.nth, cfg.nph, cfg.nr
        d.radius = r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if idx_rj_lm is not None:
            self._idx = np.ascontiguousarray(idx_rj_lm, np.int32)
            d.idx_rj_lm = self._idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        d.nvector_b, d.nscalar_b, d.nvector_f, d.nscalar_f = cfg.nvb, cfg.nsb, cfg.nvf, cfg.nsf
        d.nproduct = len(cfg.products)
        d.products = prods
        flags = (FLAG_AUTOTUNE if autotune else 0) | (FLAG_P_ON_THE_FLY if p_on_the_fly else 0)
        d.tier, d.nslice, d.device, d.flags = tier, nslice, device, flags
        self._desc = d
        h = ctypes.c_void_p()
        _check(lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)), "kmhd_sph_create")
        self._h = h
        self._cols_b = _i32(cfg.cols_b())
        self._cols_f = _i32(cfg.cols_f())

    def close(self):
        if getattr(self, "_h", None):
            load_library().kmhd_sph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int | None):
        _check(load_library().kmhd_sph_set_stream(self._h, stream_ptr), "set_stream")

    def device_bytes(self) -> int:
        return int(load_library().kmhd_sph_device_bytes(self._h))

    def last_timing(self):
        t = (ctypes.c_double * 4)()
        _check(load_library().kmhd_sph_last_timing(self._h, t), "last_timing")
        return dict(leg_bwd=t[0], fft_nl=t[1], leg_fwd=t[2], total=t[3])

    def uses_split(self) -> bool:
        """True when the handle runs the split-precision Legendre path."""
        v = ctypes.c_int32()
        _check(load_library().kmhd_sph_get_path(self._h, ctypes.byref(v)), "get_path")
        return v.value == 1

    def tuning(self) -> dict:
        """Legendre path, slice products per GEMM and, after an autotuned batch
        call, the candidates' times (ms) and errors against the FP64 path."""
        path, prod = ctypes.c_int32(), ctypes.c_int32()
        ms, err = (ctypes.c_float * 3)(), (ctypes.c_double * 3)()
        _check(load_library().kmhd_sph_get_tuning(self._h, ctypes.byref(path), ctypes.byref(prod), ms, err),
               "get_tuning")
        return dict(path=path.value, products=prod.value, ms=list(ms), err=list(err))

    def set_products(self, products: int):
        """Pins the split path's slice products per GEMM (26/21 split, 10/6 fp32acc)."""
        _check(load_library().kmhd_sph_set_products(self._h, int(products)), "set_products")

    def kernel_timing(self):
        """Per-launch ms of the last cycle (CUDA events on the handle's stream)."""
        t = (ctypes.c_double * 5)()
        _check(load_library().kmhd_sph_last_kernel_timing(self._h, t), "last_kernel_timing")
        return dict(slice_bwd=t[0], gemm_bwd=t[1], fft_nl=t[2], slice_fwd=t[3], gemm_fwd=t[4])

    def tables(self, m: int):
        c = self.cfg
        colat, w = np.zeros(c.nth), np.zeros(c.nth)
        P = np.zeros((c.ltr - m + 1, c.nh))
        dP = np.zeros_like(P)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        _check(load_library().kmhd_sph_get_tables(self._h, m, dp(colat), dp(w), dp(P), dp(dP)),
               "get_tables")
        return colat, w, P, dP

    # --- reference-named entry points -----------------------------------
    def sph_b_trans(self, d_rj, fld_rtp, cols_b: Sequence[int] | None = None, ld: int | None = None):
        """d_rj (J*Nr x ncol) -> fld_rtp (nnod_rtp x ncb), both column-major."""
        src, kind = _ptr(d_rj)
        dst, kind2 = _ptr(fld_rtp)
        assert kind == kind2, "d_rj and fld_rtp must both be host or both device"
        cols = self._cols_b if cols_b is None else _i32(cols_b)
        ld = self.cfg.J * self.cfg.nr if ld is None else ld
        _check(load_library().kmhd_sph_b_trans(self._h, src, ld, cols, dst, kind), "sph_b_trans")
        return fld_rtp

    def sph_f_trans(self, frc_rtp, d_rj, cols_f: Sequence[int] | None = None, ld: int | None = None):
        src, kind = _ptr(frc_rtp)
        dst, kind2 = _ptr(d_rj)
        assert kind == kind2
        cols = self._cols_f if cols_f is None else _i32(cols_f)
        ld = self.cfg.J * self.cfg.nr if ld is None else ld
        _check(load_library().kmhd_sph_f_trans(self._h, src, dst, ld, cols, kind), "sph_f_trans")
        return d_rj

    def nonlinear_cycle(self, d_rj_in, d_rj_out, cols_b=None, cols_f=None, ld_in=None, ld_out=None):
        """bwd transform -> grid products -> fwd transform, d_rj_in -> d_rj_out."""
        src, kind = _ptr(d_rj_in)
        dst, kind2 = _ptr(d_rj_out)
        assert kind == kind2
        cb = self._cols_b if cols_b is None else _i32(cols_b)
        cf = self._cols_f if cols_f is None else _i32(cols_f)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_cycle(self._h, src, ld_in or n, cb, dst, ld_out or n, cf, kind),
               "kmhd_sph_cycle")
        return d_rj_out


    def div_flux(self, d_rj, col_flux: int, col_div: int, fix_in=None, fix_out=None, ld: int | None = None):
        """Divergence of the flux vector in columns col_flux (S), col_flux + 1
        (dS/dr) into column col_div, fixed-field boundary values fix_in /
        fix_out (J each, same host/device kind as d_rj, None = zero)."""
        p, kind = _ptr(d_rj)
        fi = _ptr(fix_in)[0] if fix_in is not None else None
        fo = _ptr(fix_out)[0] if fix_out is not None else None
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_div_flux(self._h, p, ld or n, col_flux, col_div, fi, fo, kind),
               "kmhd_sph_div_flux")
        return d_rj


    def div_flux_bc(self, d_rj, col_flux: int, col_div: int, bc_icb: int = 0, bc_cmb: int = 0, val_in=None,
                    val_out=None, ld: int | None = None):
        """div_flux with a boundary condition per side (BC_FIXED_FIELD /
        BC_FIXED_FLUX); val_in / val_out the fixed field or flux spectra."""
        p, kind = _ptr(d_rj)
        vi = _ptr(val_in)[0] if val_in is not None else None
        vo = _ptr(val_out)[0] if val_out is not None else None
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_div_flux_bc(self._h, p, ld or n, col_flux, col_div, bc_icb, bc_cmb, vi, vo,
                                                   kind), "kmhd_sph_div_flux_bc")
        return d_rj

    def rot_induction_bc(self, d_rj, col_fld: int, col_rot: int, bc_icb: int = 0, bc_cmb: int = 0,
                         ld: int | None = None):
        """rot_induction with BC_INSULATOR / BC_PSEUDO_VACUUM per side."""
        p, kind = _ptr(d_rj)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_rot_induction_bc(self._h, p, ld or n, col_fld, col_rot, bc_icb, bc_cmb, kind),
               "kmhd_sph_rot_induction_bc")
        return d_rj

    def vorticity(self, d_rj, col_velo: int, col_vort: int, bc_icb: int = 0, bc_cmb: int = 0,
                  ld: int | None = None):
        """curl u into col_vort.. with BC_NON_SLIP / BC_FREE_SLIP per side."""
        p, kind = _ptr(d_rj)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_vorticity(self._h, p, ld or n, col_velo, col_vort, bc_icb, bc_cmb, kind),
               "kmhd_sph_vorticity")
        return d_rj

    def current(self, d_rj, col_magne: int, col_current: int, bc_icb: int = 0, bc_cmb: int = 0,
                ld: int | None = None):
        """curl B into col_current.. with BC_INSULATOR / BC_PSEUDO_VACUUM per side."""
        p, kind = _ptr(d_rj)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_current(self._h, p, ld or n, col_magne, col_current, bc_icb, bc_cmb, kind),
               "kmhd_sph_current")
        return d_rj

    def rot_buoyancy(self, d_rj, col_t: int, coef_t: float, col_out: int, col_c: int = -1, coef_c: float = 0.0,
                     ld: int | None = None):
        """Toroidal curl of the radial buoyancy: (coef_t T [+ coef_c C]) r into col_out."""
        p, kind = _ptr(d_rj)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_rot_buoyancy(self._h, p, ld or n, col_t, float(coef_t), col_c, float(coef_c),
                                                    col_out, kind), "kmhd_sph_rot_buoyancy")
        return d_rj

    def rot_induction(self, d_rj, col_fld: int, col_rot: int, ld: int | None = None):
        """Curl of the vector (S, dS/dr, T) in columns col_fld.. into
        col_rot.. (pol, dpol/dr, tor), insulating boundaries."""
        p, kind = _ptr(d_rj)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_rot_induction(self._h, p, ld or n, col_fld, col_rot, kind),
               "kmhd_sph_rot_induction")
        return d_rj

    def rot_force(self, d_rj, col_fld: int, col_rot: int, bc_icb: int = 0, bc_cmb: int = 0,
                  ld: int | None = None):
        """Curl of the force (S, dS/dr, T) in columns col_fld.. into col_rot..
        with the velocity conditions bc_icb / bc_cmb (BC_NON_SLIP, BC_FREE_SLIP)."""
        p, kind = _ptr(d_rj)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_rot_force(self._h, p, ld or n, col_fld, col_rot, bc_icb, bc_cmb, kind),
               "kmhd_sph_rot_force")
        return d_rj

    def div_force(self, d_rj, col_fld: int, col_div: int, ld: int | None = None):
        """Divergence of the force (S, dS/dr) in columns col_fld.. into col_div."""
        p, kind = _ptr(d_rj)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_div_force(self._h, p, ld or n, col_fld, col_div, kind),
               "kmhd_sph_div_force")
        return d_rj

    def rot_coriolis(self, d_rj, col_velo: int, col_vort: int, col_out: int, coef_cor: float,
                     ld: int | None = None):
        """Curl of the Coriolis term -coef_cor z x u: poloidal part into
        col_out, toroidal part into col_out + 2 (col_out + 1 untouched)."""
        p, kind = _ptr(d_rj)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_rot_coriolis(self._h, p, ld or n, col_velo, col_vort, col_out,
                                                    float(coef_cor), kind), "kmhd_sph_rot_coriolis")
        return d_rj

    def b_trans_pole(self, d_rj, v_pole, cols_b=None, ld: int | None = None):
        """Values at the poles: v_pole (2 Nr x ncomp_b; torch CUDA tensor of shape
        (ncomp_b, 2 Nr) or F-order numpy array), rows k north / Nr + k south."""
        p, kind = _ptr(d_rj)
        q, kind2 = _ptr(v_pole)
        if kind != kind2:
            raise ValueError("d_rj and v_pole must both be host or both be device arrays")
        cb = self._cols_b if cols_b is None else _i32(cols_b)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_b_trans_pole(self._h, p, ld or n, cb, q, kind), "kmhd_sph_b_trans_pole")
        return v_pole

    def b_trans_center(self, d_rj, v_center, cols_b=None, ld: int | None = None):
        """Values at the centre node of a full-sphere grid: v_center (ncomp_b;
        torch CUDA tensor or numpy array); vector entries are written, scalar
        entries left as they are."""
        p, kind = _ptr(d_rj)
        q, kind2 = _ptr(v_center)
        if kind != kind2:
            raise ValueError("d_rj and v_center must both be host or both be device arrays")
        cb = self._cols_b if cols_b is None else _i32(cols_b)
        n = self.cfg.J * self.cfg.nr
        _check(load_library().kmhd_sph_b_trans_center(self._h, p, ld or n, cb, q, kind), "kmhd_sph_b_trans_center")
        return v_center

    def set_coriolis(self, coef_cor: float, iv_velo: int = 0, iv_vort: int = 1, col_out: int = -1):
        """Every following cycle also writes the curl of the Coriolis term of
        backward vectors iv_velo / iv_vort into output columns col_out (pol)
        and col_out + 2 (tor); iv_velo < 0 switches it off."""
        _check(load_library().kmhd_sph_set_coriolis(self._h, float(coef_cor), iv_velo, iv_vort, col_out),
               "kmhd_sph_set_coriolis")


def batch_cycle(transforms: Sequence[SphTransform], d_in, d_out):
    """Runs the cycle of every instance (device tensors) as one batch."""
    lib = load_library()
    n = len(transforms)
    hs = (ctypes.c_void_p * n)(*[t.handle.value for t in transforms])
    ins = (ctypes.c_void_p * n)(*[x.data_ptr() for x in d_in])
    outs = (ctypes.c_void_p * n)(*[x.data_ptr() for x in d_out])
    lds = (ctypes.c_int64 * n)(*[t.cfg.J * t.cfg.nr for t in transforms])
    cbs = (ctypes.POINTER(ctypes.c_int32) * n)(*[ctypes.cast(t._cols_b, ctypes.POINTER(ctypes.c_int32)) for t in transforms])
    cfs = (ctypes.POINTER(ctypes.c_int32) * n)(*[ctypes.cast(t._cols_f, ctypes.POINTER(ctypes.c_int32)) for t in transforms])
    _check(lib.kmhd_sph_batch_cycle(hs, n, ins, lds, cbs, outs, lds, cfs), "kmhd_sph_batch_cycle")
