"""The z-slab halo exchange behind the C ABI (axb_halo_*, NCCL), on the one
GPU a test gets: with one rank the exchange is the periodic wrap in z, so
after it every ghost k-plane of every listed grid function (cell- and
vertex-centred in z) equals what the single-box periodic fill gives.  The
two-rank plane mapping is tested on CPU with gloo ranks
(tests/test_distribute.py, SlabHalo), which uses the same mapping.  The
exchange copies whole padded k-planes; the comparison covers each field's
own extent."""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import workloads as W
from asterx_b200.distribute import EVOLVED, NcclSlabHalo, prims_to_sync
from asterx_b200.driver import CENTRING
from tests.helpers import full_fields


def extent(L, name):
    """(k, j, i) extents of a grid function in the padded layout: n + 2 ng
    points along a cell-centred axis, one more along a vertex-centred one;
    the padding beyond is no point of the field."""
    cent = CENTRING.get(name, (1, 1, 1))
    return tuple(L.n[d] + 2 * L.ng + (0 if cent[d] else 1) for d in (2, 1, 0))


@pytest.mark.gpu
def test_halo_one_rank_is_the_periodic_wrap(engine):
    torch = engine.torch
    L, f = W.curved_box(n=(12, 10, 9), ng=3, seed=21, wmax=2.0)
    W.cons_from_prims(L, f)
    f = full_fields(L, f)
    evolved = EVOLVED
    prims = prims_to_sync(abi.default_params(recon_type=1))
    names = evolved + prims
    # scramble the z ghosts so the exchange has to fill them
    rng = np.random.default_rng(5)
    for n in names:
        v = L.view(f[n])
        top = extent(L, n)[0] - L.ng
        v[:L.ng] = rng.standard_normal(v[:L.ng].shape)
        v[top:] = rng.standard_normal(v[top:].shape)
    want = engine.upload(L, f)
    engine.sync_periodic(L, want, names)
    got = engine.upload(L, f)
    engine.sync_periodic(L, got, names)  # x and y ghosts; the z wrap is undone below
    for n in names:  # put the scrambled z ghosts back: the exchange alone fills them
        top = extent(L, n)[0] - L.ng
        g = got[n].view(L.npts[2], L.npts[1], L.sy)
        src = torch.from_numpy(L.view(f[n])).to(got[n].device)
        g[:L.ng] = src[:L.ng]
        g[top:] = src[top:]
    halo = NcclSlabHalo(engine, L, 0, 1)
    try:
        halo.exchange(got, evolved)
        halo.exchange(got, prims)
        torch.cuda.synchronize()
    finally:
        halo.close()
    for n in names:
        ek, ej, ei = extent(L, n)
        a = L.view(got[n].cpu().numpy())[:ek, :ej, :ei]
        b = L.view(want[n].cpu().numpy())[:ek, :ej, :ei]
        assert np.array_equal(a, b), n
