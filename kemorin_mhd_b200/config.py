"""Transform configurations, radial grids and the field/product layout.

The spectral layout is the reference's single-domain rj layout:
``d_rj(inod, icomp)`` column-major with ``inod = j + J*k`` (j fastest), and the
j order "m = -L..L, then l = |m|..L" produced by
PARALLEL_src/CONST_SPH_GRID/set_sph_tranform_ordering.f90:64-206
(set_zonal_wavenum_4_legendre + set_merged_index_4_sph_trans with one domain).
A vector field occupies three consecutive columns (S, dS/dr, T)
(SOLVER_src/send_recv/field_to_send_buffer.f90:62-64).

The grid-space products follow MHD_src/sph_MHD/cal_nonlinear_sph_MHD.f90:64-128
(m_advect = coef*(omega x u), vp_induct = coef*(u x B), h_flux = coef*u*T) and the
reference's kinetic-helicity field u.omega (MHD_src/evolution/cal_helicities.f90).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Sequence, Tuple

import numpy as np

# product kinds (kmhd_product.kind in include/kmhd_sph.h)
PROD_CROSS = 0        # fwd vector = coef * (bwd_vec[a] x bwd_vec[b])
PROD_VEC_SCALAR = 1   # fwd vector = coef * bwd_vec[a] * bwd_scl[b]
PROD_DOT = 2          # fwd scalar = coef * (bwd_vec[a] . bwd_vec[b])
PROD_SCALAR = 3       # fwd scalar = coef * bwd_scl[a] * bwd_scl[b]

# tiers (kmhd_sph_desc.tier)
TIER_FP64 = 0
TIER_SPLIT_I8 = 1
TIER_FP32ACC = 2

# shell radii ratio 0.35 (programs/mesh_utilities/spherical_shell/control_sph_shell)
R_ICB = 0.35 / 0.65
R_CMB = 1.0 / 0.65


def chebyshev_radii(nr: int, r_icb: float = R_ICB, r_cmb: float = R_CMB) -> np.ndarray:
    """Chebyshev-Gauss-Lobatto radii between ICB and CMB.

    Follows set_chebyshev_distance_shell
    (CORE_src/SPH_SPECTR_src/chebyshev_radial_grid.f90:29-80), shell part:
    r_k = r_ICB + 0.5*(r_CMB - r_ICB)*(1 - cos(pi*k/(Nr-1))).
    """
    pi = 4.0 * math.atan(1.0)
    shell = r_cmb - r_icb
    k = np.arange(nr, dtype=np.float64)
    return r_icb + 0.5 * shell * (1.0 - np.cos(pi * k / float(nr - 1)))


def rj_order(L: int) -> Tuple[np.ndarray, np.ndarray]:
    """(l, m) of every rj mode j in the reference's single-domain order."""
    ls, ms = [], []
    for m in range(-L, L + 1):
        for l in range(abs(m), L + 1):
            ls.append(l)
            ms.append(m)
    return np.asarray(ls, np.int32), np.asarray(ms, np.int32)


@dataclasses.dataclass
class SphConfig:
    """One transform instance: truncation, grid and field counts."""
    ltr: int
    nth: int
    nph: int
    nr: int
    nvb: int = 3          # backward vectors (u, omega, B)
    nsb: int = 1          # backward scalars (T)
    nvf: int = 3          # forward vectors (omega x u, u x B, u T)
    nsf: int = 1          # forward scalars (u . omega)
    products: Sequence[Tuple[int, int, int, float]] = (
        (PROD_CROSS, 1, 0, 1.0),       # m_advect  = omega x u
        (PROD_CROSS, 0, 2, 1.0),       # vp_induct = u x B
        (PROD_VEC_SCALAR, 0, 0, 1.0),  # h_flux    = u T
        (PROD_DOT, 0, 1, 1.0),         # kinetic helicity u . omega
    )
    name: str = ""

    @property
    def J(self) -> int:
        return (self.ltr + 1) ** 2

    @property
    def ncb(self) -> int:
        return 3 * self.nvb + self.nsb

    @property
    def ncf(self) -> int:
        return 3 * self.nvf + self.nsf

    @property
    def nh(self) -> int:
        return (self.nth + 1) // 2

    def radius(self) -> np.ndarray:
        return chebyshev_radii(self.nr)

    def cols_b(self) -> np.ndarray:
        """First d_rj column of each backward field (vectors, then scalars)."""
        return np.asarray([3 * v for v in range(self.nvb)] +
                          [3 * self.nvb + s for s in range(self.nsb)], np.int32)

    def cols_f(self) -> np.ndarray:
        return np.asarray([3 * v for v in range(self.nvf)] +
                          [3 * self.nvf + s for s in range(self.nsf)], np.int32)

    def legendre_flops(self) -> float:
        """2*Nh*(L+1)^2*Nr*[(5 n_vb + n_sb) + (5 n_vf + n_sf)] per cycle."""
        return 2.0 * self.nh * self.J * self.nr * (
            (5 * self.nvb + self.nsb) + (5 * self.nvf + self.nsf))


# Named workloads (sizes as specified for this path).
CFG1 = SphConfig(31, 48, 96, 33, name="L31_Nr33")
CFG2 = SphConfig(255, 384, 768, 129, name="L255_Nr129")
CFG3 = SphConfig(511, 768, 1536, 257, name="L511_Nr257")
CFG5 = SphConfig(1023, 1536, 3072, 129, name="L1023_Nr129")

NAMED = {"cfg1": CFG1, "cfg2": CFG2, "cfg3": CFG3, "cfg5": CFG5}

# Field sets of the reference's MHD transforms (set_address_sph_trans_MHD.f90):
# "default" = u, omega, B + T -> omega x u, u x B, u T + u.omega;
# "dynamo" = u, omega, B, J + T -> omega x u, J x B, u x B, u T (the dynamo
# benchmark set with the Lorentz force);
# "full" = u, omega, B, J + T, C -> omega x u, J x B, u x B, u T, u C + u.omega.
FIELD_SETS = {
    "default": dict(nvb=3, nsb=1, nvf=3, nsf=1,
                    products=((PROD_CROSS, 1, 0, 1.0), (PROD_CROSS, 0, 2, 1.0), (PROD_VEC_SCALAR, 0, 0, 1.0),
                              (PROD_DOT, 0, 1, 1.0))),
    "dynamo": dict(nvb=4, nsb=1, nvf=4, nsf=0,
                   products=((PROD_CROSS, 1, 0, 1.0), (PROD_CROSS, 3, 2, 1.0), (PROD_CROSS, 0, 2, 1.0),
                             (PROD_VEC_SCALAR, 0, 0, 1.0))),
    "full": dict(nvb=4, nsb=2, nvf=5, nsf=1,
                 products=((PROD_CROSS, 1, 0, 1.0), (PROD_CROSS, 3, 2, 1.0), (PROD_CROSS, 0, 2, 1.0),
                           (PROD_VEC_SCALAR, 0, 0, 1.0), (PROD_VEC_SCALAR, 0, 1, 1.0), (PROD_DOT, 0, 1, 1.0))),
}
FIELD_NAMES = {
    "default": ("u,omega,B + T", "omega x u, u x B, u T + u.omega"),
    "dynamo": ("u,omega,B,J + T", "omega x u, J x B, u x B, u T"),
    "full": ("u,omega,B,J + T,C", "omega x u, J x B, u x B, u T, u C + u.omega"),
}


def with_fields(cfg: SphConfig, fields: str) -> SphConfig:
    """The configuration's grid with one of the FIELD_SETS."""
    if fields == "default":
        return cfg
    return dataclasses.replace(cfg, name=f"{cfg.name}_{fields}", **FIELD_SETS[fields])


def batch_configs(n: int = 64, seed: int = 2024) -> List[SphConfig]:
    """Uneven instances: L from {63,127,255}, Nr from {33,65,129}, 2-4 fields.

    Nth = 3(L+1)/2, Nph = 3(L+1).  Field mixes keep the product list valid:
    2 fields = {u, T}, 3 = {u, omega, T}, 4 = {u, omega, B, T}.
    """
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L = int(rng.choice([63, 127, 255]))
        nr = int(rng.choice([33, 65, 129]))
        nf = int(rng.integers(2, 5))
        nth, nph = 3 * (L + 1) // 2, 3 * (L + 1)
        if nf == 2:
            c = SphConfig(L, nth, nph, nr, nvb=1, nsb=1, nvf=1, nsf=0,
                          products=((PROD_VEC_SCALAR, 0, 0, 1.0),), name=f"b{i}")
        elif nf == 3:
            c = SphConfig(L, nth, nph, nr, nvb=2, nsb=1, nvf=2, nsf=1,
                          products=((PROD_CROSS, 1, 0, 1.0), (PROD_VEC_SCALAR, 0, 0, 1.0),
                                    (PROD_DOT, 0, 1, 1.0)), name=f"b{i}")
        else:
            c = SphConfig(L, nth, nph, nr, name=f"b{i}")
        out.append(c)
    return out
