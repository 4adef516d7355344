"""Radial slabs (kemorin_mhd_b200/slabs.py), host logic on CPU: the
partition of the radii and the halo exchange over gloo with 2 and 3 ranks."""
import os
import socket

import numpy as np
import pytest

from kemorin_mhd_b200.slabs import radial_slab


@pytest.mark.parametrize("nr", [3, 9, 65, 257])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_radial_slab_partition(nr, world):
    if nr < world:
        with pytest.raises(ValueError):
            radial_slab(nr, world, 0)
        return
    slabs = [radial_slab(nr, world, r) for r in range(world)]
    assert slabs[0].r0 == 0 and slabs[-1].r1 == nr
    for a, b in zip(slabs, slabs[1:]):
        assert a.r1 == b.r0
    sizes = [s.r1 - s.r0 for s in slabs]
    assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    for s in slabs:
        assert s.lo == max(s.r0 - 1, 0) and s.hi == min(s.r1 + 1, nr)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _halo_worker(rank, world, port, J, nr, ncol, cols, q):
    import torch
    import torch.distributed as dist
    from kemorin_mhd_b200.slabs import exchange_halo, radial_slab
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        glob = torch.arange(ncol * J * nr, dtype=torch.float64).reshape(ncol, J * nr)
        s = radial_slab(nr, world, rank)
        loc = torch.full((ncol, J * s.nr_local), float("nan"), dtype=torch.float64)
        own = s.owned_rows(J)
        loc[:, own] = glob[:, s.r0 * J:s.r1 * J]
        exchange_halo(s, J, loc, cols)
        ref = glob[:, s.lo * J:s.hi * J]
        ok = bool(torch.equal(loc[cols], ref[cols]))
        others = [c for c in range(ncol) if c not in cols]
        halo_rows = [k for k in range(s.nr_local) if not s.r0 <= s.lo + k < s.r1]
        for c in others:   # columns not asked for keep their (unset) halo rows
            for k in halo_rows:
                ok = ok and bool(torch.isnan(loc[c, k * J:(k + 1) * J]).all())
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_halo_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    J, nr, ncol, cols = 6, 8, 5, [0, 2, 3]
    port = _free_port()
    procs = [ctx.Process(target=_halo_worker, args=(r, world, port, J, nr, ncol, cols, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(res[r] for r in range(world)), res
