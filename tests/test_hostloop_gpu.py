"""Substeps of a box whose state lives in pinned host memory
(asterx_b200.hostloop): with the copies of consecutive substeps overlapped on
two copy streams, the host state after two SSP-RK3 steps equals, bit for bit,
that of the same substeps run on device-resident fields.  The host loop runs
on a box whose every field is large enough that the copies of one substep
are still in flight when the next is issued."""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import distribute as D
from asterx_b200 import workloads as W
from asterx_b200.hostloop import HostStateLoop, substep_io
from tests.helpers import full_fields

SSPRK3 = [(0.0, 1.0, 1.0), (0.75, 0.25, 0.25), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)]


@pytest.mark.gpu
def test_host_state_loop_matches_device_loop(engine):
    torch = engine.torch
    L, f = W.curved_box(n=(40, 36, 32), ng=3, seed=78, wmax=3.0, sigma=(1e-3, 1.0),
                        theta=(0.1, 1.0))
    W.cons_from_prims(L, f)
    W.saved_from_prims(f)
    f = full_fields(L, f)
    p = abi.default_params(reconstruction_method="wenoz", flux_type="hlle",
                           c2p_prime="palenzuela", c2p_second="noble", recon_type=1)
    eos = engine.eos_idealgas(4.0 / 3.0, rho=(1e-40, 1e10), eps=(0.0, 1e10))
    dt = 0.25 * L.dx[0]
    inputs, outputs = substep_io(p.recon_type)

    # device-resident reference run
    a = engine.upload(L, f)
    an = {k: a[k].clone() for k in D.EVOLVED}
    # the host loop: the state in pinned host memory, the device fields
    # scrambled so that only the copies in can make them right
    b = engine.upload(L, f)
    bn = {k: b[k].clone() for k in D.EVOLVED}
    host = {k: torch.empty(L.size, dtype=torch.float64, pin_memory=True)
            for k in set(inputs) | set(outputs)}
    for k in host:
        host[k].copy_(b[k])
        if k in inputs:
            b[k].fill_(float("nan"))
    loop = HostStateLoop(torch, engine.device, b, host, inputs, outputs)

    def run(s, x, y, z):
        if s == 0:
            for k in D.EVOLVED:
                bn[k].copy_(b[k])
        engine.substep(L, b, bn, p, eos, x, y, z, dt, periodic=True)

    for step in range(2):
        for s, (x, y, z) in enumerate(SSPRK3):
            if s == 0:
                for k in D.EVOLVED:
                    an[k].copy_(a[k])
            engine.substep(L, a, an, p, eos, x, y, z, dt, periodic=True)
            loop.step(lambda s=s, x=x, y=y, z=z: run(s, x, y, z))
    loop.finish()
    torch.cuda.synchronize()
    for k in outputs:
        want = a[k].cpu().numpy()
        got = host[k].numpy()
        assert np.array_equal(got, want, equal_nan=True), k
    # every field the substeps only read still holds its value on the host
    for k in inputs:
        if k not in outputs:
            assert np.array_equal(host[k].numpy(), f[k]), k
