"""The slab driver of the multi-GPU path on one GPU: with a single rank the
halo exchange is the periodic wrap, so slab_substep must reproduce
axb_substep bit for bit over an SSP-RK3 step.  (The exchange between ranks
is checked against the whole patch's periodic fill on the CPU with gloo in
test_distribute.py.)"""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import distribute as D
from asterx_b200 import workloads as W
from tests.helpers import full_fields

SSPRK3 = [(0.0, 1.0, 1.0), (0.75, 0.25, 0.25), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)]


@pytest.mark.gpu
def test_slab_substep_single_rank_matches_substep(engine):
    L, f = W.curved_box(n=(12, 10, 9), ng=3, seed=77, wmax=2.0, sigma=(1e-3, 0.3),
                        theta=(0.1, 1.0))
    W.cons_from_prims(L, f)
    W.saved_from_prims(f)
    f = full_fields(L, f)
    p = abi.default_params(reconstruction_method="wenoz", flux_type="hlle",
                           c2p_prime="palenzuela", c2p_second="noble")
    eos = engine.eos_idealgas(4.0 / 3.0, rho=(1e-40, 1e10), eps=(0.0, 1e10))
    a, b = engine.upload(L, f), engine.upload(L, f)
    an = {k: a[k].clone() for k in D.EVOLVED}
    bn = {k: b[k].clone() for k in D.EVOLVED}
    halo = D.SlabHalo(L, 0, 1)
    dt = 0.25 * L.dx[0]
    for s, (x, y, z) in enumerate(SSPRK3):
        if s == 0:
            for k in D.EVOLVED:
                an[k].copy_(a[k])
                bn[k].copy_(b[k])
        engine.substep(L, a, an, p, eos, x, y, z, dt, periodic=True)
        D.slab_substep(engine, L, b, bn, p, eos, x, y, z, dt, halo)
    engine.torch.cuda.synchronize()
    from tests.helpers import CENTRING
    for k in D.EVOLVED + D.PRIMS + ["con2prim_flag"]:
        # every point of the field's centring (the halo also copies the row
        # padding of whole planes, which no kernel reads)
        c = CENTRING.get(k, (1, 1, 1))
        ext = [L.n[d] + 2 * L.ng + (0 if c[d] else 1) for d in range(3)]
        x = L.view(a[k].cpu().numpy())[:ext[2], :ext[1], :ext[0]]
        y = L.view(b[k].cpu().numpy())[:ext[2], :ext[1], :ext[0]]
        assert np.array_equal(x, y, equal_nan=True), k
