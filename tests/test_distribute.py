"""Multi-rank host logic on the CPU (gloo): box balancing, slab ranges, and the
z-slab halo exchange, whose result must equal the single-box periodic ghost
fill of the whole patch on every rank's planes."""
import socket

import numpy as np
import pytest

from asterx_b200 import distribute as D
from asterx_b200.abi import Layout
from tests.helpers import periodic_sync

NAMES = ["rho", "Avec_x", "Avec_z", "Psi"]
NG_ = (10, 7, 12)


def test_balance_boxes():
    rng = np.random.default_rng(1)
    zones = [int(v) for v in rng.integers(16 ** 3, 64 ** 3, 97)]
    for world in (1, 2, 3, 8):
        parts = D.balance_boxes(zones, world)
        flat = sorted(b for p in parts for b in p)
        assert flat == list(range(len(zones)))
        loads = [sum(zones[b] for b in p) for p in parts]
        assert max(loads) <= 4 / 3 * max(sum(zones) / world, max(zones)) + 1


def test_slab_ranges():
    for nz, world in ((256, 2), (257, 3), (9, 4)):
        r = D.slab_ranges(nz, world)
        assert sum(n for _, n in r) == nz
        assert all(r[q][0] == sum(n for _, n in r[:q]) for q in range(world))
        assert max(n for _, n in r) - min(n for _, n in r) <= 1


def _global_reference():
    G = Layout(NG_, 3, tuple(1.0 / v for v in NG_), (0.0, 0.0, 0.0))
    rng = np.random.default_rng(5)
    f = {n: rng.normal(size=G.size) for n in NAMES}
    periodic_sync(G, f, NAMES)
    return G, f


def _rank_main(rank, world, port):
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                world_size=world)
    try:
        G, gf = _global_reference()
        L, k0 = D.slab_layout(NG_, 3, rank, world)
        loc = {}
        for n in NAMES:
            a = np.zeros(L.size)
            v, gv = L.view(a), G.view(gf[n])
            # interior planes (and, for simplicity, all i, j) from the patch
            nplanes = L.n[2] + (1 if D.vertex_in_z(n) else 0)
            v[L.ng:L.ng + nplanes] = gv[L.ng + k0:L.ng + k0 + nplanes]
            loc[n] = a
        periodic_sync(L, loc, NAMES)  # local fill: x, y right, z wrong
        t = {n: torch.from_numpy(loc[n]) for n in NAMES}
        D.SlabHalo(L, rank, world).exchange(t, NAMES)
        from tests.helpers import CENTRING
        for n in NAMES:
            c = CENTRING.get(n, (1, 1, 1))
            v, gv = L.view(loc[n]), G.view(gf[n])
            # the points of this field's centring (padding excluded)
            ext = [L.n[d] + 2 * L.ng + (0 if c[d] else 1) for d in range(3)]
            got = v[:ext[2], :ext[1], :ext[0]]
            want = gv[k0:k0 + ext[2], :ext[1], :ext[0]]
            assert np.array_equal(got, want), (rank, n)
    finally:
        if world > 1:
            dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [1, 2, 3])
def test_slab_halo_matches_global_periodic_fill(world):
    if world == 1:
        _rank_main(0, 1, 0)
        return
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(world, _free_port()), nprocs=world,
                       start_method="spawn", join=True)


def test_cfl_dt():
    dx = (1 / 64, 1 / 32, 1 / 16)
    # the fixed dtfac governs while the characteristic speeds allow it
    assert D.cfl_dt(0.1, dx, 0.25) == 0.25 / 64
    # otherwise dt * smax * sum(1/dx) equals the CFL number
    dt = D.cfl_dt(4.0, dx, 0.25, cfl=0.9)
    assert dt < 0.25 / 64
    assert abs(dt * 4.0 * (64 + 32 + 16) - 0.9) < 1e-12


def _cfl_main(rank, world, port):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        # each rank's faces saw a different maximum speed; every rank must
        # take the same (largest) one and so the same time step
        smax = D.allreduce_max(1.0 + 0.5 * rank)
        assert smax == 1.0 + 0.5 * (world - 1)
        dts = [None] * world
        dist.all_gather_object(dts, D.cfl_dt(smax, (1 / 8,) * 3, 0.25))
        assert len(set(dts)) == 1
    finally:
        dist.destroy_process_group()


def test_allreduce_max_speed_two_ranks():
    import torch.multiprocessing as mp
    assert D.allreduce_max(3.5) == 3.5  # no process group: the identity
    mp.start_processes(_cfl_main, args=(2, _free_port()), nprocs=2, start_method="spawn",
                       join=True)
