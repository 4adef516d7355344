"""Radial slabs: one transform instance spread over several GPUs by radius.

Every stage of the cycle is independent per radius (the Legendre GEMMs'
columns are (radius, component), the phi-FFT runs per (radius, theta) line,
the products are pointwise), so rank i of N holds a handle over its own
contiguous radii [r0, r1) -- the reference's radial domain split
(`num_domain_sph_grid radial`, programs/mesh_utilities/spherical_shell/
control_sph_shell) -- and the cycle has no collective.  The P tables are
replicated per GPU.

The spectral post-processing after the forward transform (divergence and
curl rows, MHD_src/sph_MHD/cal_sph_exp_rotation.f90) takes a 3-point radial
stencil, so each handle also carries one halo radius on each side that
another rank owns: the cycle computes the halo radii redundantly and the
post-processing's rows on the owned radii need no further exchange.  The
only data exchange is the halo of the input spectra (`exchange_halo`, one
radius row per column and neighbour, torch.distributed send/recv: NCCL over
NVLink on GPUs, gloo on CPUs) for callers that hold only their owned radii.
Local rows k of the slab arrays are global radii lo + k, j fastest, in the
d_rj layout.
"""
from __future__ import annotations

import dataclasses
from typing import Sequence

import numpy as np

from .config import SphConfig


@dataclasses.dataclass(frozen=True)
class RadialSlab:
    """Rank `rank` of `world`: owned radii [r0, r1), local radii [lo, hi)
    (owned plus one halo radius on each side, clipped at the shell)."""
    nr: int
    world: int
    rank: int
    r0: int
    r1: int
    lo: int
    hi: int

    @property
    def nr_local(self) -> int:
        return self.hi - self.lo

    def owned_rows(self, J: int) -> slice:
        """Rows of the local d_rj arrays that hold the owned radii."""
        return slice((self.r0 - self.lo) * J, (self.r1 - self.lo) * J)


def radial_slab(nr: int, world: int, rank: int, halo: int = 1) -> RadialSlab:
    """Balanced contiguous split of nr radii over `world` ranks (the first
    nr % world ranks own one radius more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of %d" % (rank, world))
    if nr < world:
        raise ValueError("%d radii over %d ranks" % (nr, world))
    base, extra = divmod(nr, world)
    r0 = rank * base + min(rank, extra)
    r1 = r0 + base + (1 if rank < extra else 0)
    return RadialSlab(nr, world, rank, r0, r1, max(r0 - halo, 0), min(r1 + halo, nr))


class SlabTransform:
    """One rank's transform handle over its slab's local radii.  `radius` is
    the global radial grid (default: the configuration's)."""

    def __init__(self, cfg: SphConfig, slab: RadialSlab, tier: int = 0, radius=None, **kw):
        from .sph_trans import SphTransform
        if cfg.nr != slab.nr:
            raise ValueError("configuration has %d radii, slab plan %d" % (cfg.nr, slab.nr))
        r = np.asarray(cfg.radius() if radius is None else radius, np.float64)
        self.slab = slab
        self.cfg = dataclasses.replace(cfg, nr=slab.nr_local, name=(cfg.name or "slab") + "_r%d" % slab.rank)
        self.radius = np.ascontiguousarray(r[slab.lo:slab.hi])
        self.tr = SphTransform(self.cfg, tier=tier, radius=self.radius, **kw)

    @property
    def owned(self) -> slice:
        return self.slab.owned_rows(self.cfg.J)

    def close(self):
        self.tr.close()


def _neighbours(slab: RadialSlab):
    lower = slab.rank - 1 if slab.lo < slab.r0 else None
    upper = slab.rank + 1 if slab.hi > slab.r1 else None
    return lower, upper


def exchange_halo(slab: RadialSlab, J: int, d_local, cols: Sequence[int], group=None) -> None:
    """Fills the halo radii of the columns `cols` of d_local (a torch tensor
    of shape (ncols, >= J * nr_local), one d_rj column per row; CUDA tensors
    over NCCL, CPU tensors over gloo) from the neighbouring ranks' owned
    radii.  Every rank of the group calls it with the same columns."""
    import torch
    import torch.distributed as dist
    lower, upper = _neighbours(slab)
    idx = torch.as_tensor(list(cols), dtype=torch.long, device=d_local.device)
    ops, recvs = [], []
    k_first, k_last = slab.r0 - slab.lo, slab.r1 - 1 - slab.lo
    if lower is not None:
        ops.append(dist.P2POp(dist.isend, d_local[idx, k_first * J:(k_first + 1) * J].contiguous(), lower, group))
        buf = torch.empty((len(cols), J), dtype=d_local.dtype, device=d_local.device)
        ops.append(dist.P2POp(dist.irecv, buf, lower, group))
        recvs.append((0, buf))
    if upper is not None:
        ops.append(dist.P2POp(dist.isend, d_local[idx, k_last * J:(k_last + 1) * J].contiguous(), upper, group))
        buf = torch.empty((len(cols), J), dtype=d_local.dtype, device=d_local.device)
        ops.append(dist.P2POp(dist.irecv, buf, upper, group))
        recvs.append((slab.nr_local - 1, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for k, buf in recvs:
        d_local[idx, k * J:(k + 1) * J] = buf
