"""Seeded synthetic spectra for the transform cycle.

Each field quantity q and mode (l, m) draws one N(0,1) value a_q(l,m); the
coefficient at radius r is a_q(l,m) * (l+1)^-2 * sin(pi (r-r_i)/(r_o-r_i)).
The radial derivative column of a vector field is seeded analytically from the
poloidal draw: a_S(l,m) * (l+1)^-2 * (pi/(r_o-r_i)) * cos(pi (r-r_i)/(r_o-r_i)).
The l = 0 slots of vector fields are zero.  The m = 0 mode has a single (cos)
slot in the rj layout, so it carries no imaginary part.
"""
from __future__ import annotations

import math

import numpy as np

from .config import SphConfig, rj_order, R_ICB, R_CMB


def draws(cfg: SphConfig, seed: int = 1234) -> np.ndarray:
    """Per-mode amplitudes, shape (ncb_draws, J): vectors use 2 draws (S, T), scalars 1."""
    rng = np.random.default_rng(seed)
    l, _ = rj_order(cfg.ltr)
    decay = (l.astype(np.float64) + 1.0) ** -2
    n = 2 * cfg.nvb + cfg.nsb
    a = rng.standard_normal((n, cfg.J)) * decay[None, :]
    for v in range(cfg.nvb):
        a[2 * v, l == 0] = 0.0
        a[2 * v + 1, l == 0] = 0.0
    return a


def radial_profiles(cfg: SphConfig):
    r = cfg.radius()
    pi = 4.0 * math.atan(1.0)
    x = pi * (r - R_ICB) / (R_CMB - R_ICB)
    return np.sin(x), (pi / (R_CMB - R_ICB)) * np.cos(x)


def make_d_rj(cfg: SphConfig, seed: int = 1234) -> np.ndarray:
    """Host d_rj (J*Nr x ncb), Fortran order (column-major), float64."""
    a = draws(cfg, seed)
    f, df = radial_profiles(cfg)
    J, nr = cfg.J, cfg.nr
    out = np.empty((J * nr, cfg.ncb), dtype=np.float64, order="F")
    for v in range(cfg.nvb):
        out[:, 3 * v + 0] = np.outer(f, a[2 * v]).reshape(-1)
        out[:, 3 * v + 1] = np.outer(df, a[2 * v]).reshape(-1)
        out[:, 3 * v + 2] = np.outer(f, a[2 * v + 1]).reshape(-1)
    for s in range(cfg.nsb):
        out[:, 3 * cfg.nvb + s] = np.outer(f, a[2 * cfg.nvb + s]).reshape(-1)
    return out


def make_d_rj_torch(cfg: SphConfig, seed: int = 1234, device="cuda"):
    """Same spectra built directly on the device (column-major: shape (ncb, J*Nr))."""
    import torch
    a = torch.from_numpy(draws(cfg, seed)).to(device)
    f, df = (torch.from_numpy(x).to(device) for x in radial_profiles(cfg))
    out = torch.empty((cfg.ncb, cfg.J * cfg.nr), dtype=torch.float64, device=device)
    for v in range(cfg.nvb):
        out[3 * v + 0] = torch.outer(f, a[2 * v]).reshape(-1)
        out[3 * v + 1] = torch.outer(df, a[2 * v]).reshape(-1)
        out[3 * v + 2] = torch.outer(f, a[2 * v + 1]).reshape(-1)
    for s in range(cfg.nsb):
        out[3 * cfg.nvb + s] = torch.outer(f, a[2 * cfg.nvb + s]).reshape(-1)
    return out
