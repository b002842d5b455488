"""Parity of the RHS group (AsterX_Fluxes + AsterX_SourceTerms + AsterX_RHS)
on the GPU against the reference sources compiled on the host, on the same
seeded boxes.  Tolerance: normalised max error <= 1e-12 per field (north-star
RHS tolerance per substep)."""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import workloads as W
from tests.helpers import errors, full_fields, interior

RHS_OUT = abi.HYDRO_RHS + abi.AVEC_RHS
TOL = 1e-12


def run_both(engine, ref, L, f, params, gamma):
    f = full_fields(L, f)
    host = {n: a.copy() for n, a in f.items()}
    ref.setup(L, params, host)
    ref.eos_idealgas(gamma, rho=(1e-40, 1e10), eps=(0.0, 1e10))
    ref.rhs_group()
    eos = engine.eos_idealgas(gamma, rho=(1e-40, 1e10), eps=(0.0, 1e10))
    dev = engine.upload(L, f)
    engine.status_reset()
    engine.rhs_group(L, dev, params, eos)
    st = engine.status()
    return host, {n: dev[n].cpu().numpy() for n in RHS_OUT}, st


@pytest.mark.gpu
@pytest.mark.parametrize("recon,flux", [("ppm", "hlle"), ("wenoz", "hlle"),
                                        ("mp5", "hlle"), ("minmod", "lxf"),
                                        ("monocentral", "hlle"),
                                        ("godunov", "lxf")])
def test_rhs_curved(engine, ref, recon, flux):
    L, f = W.curved_box(n=12, ng=5, seed=11, wmax=3.0)
    p = abi.default_params(reconstruction_method=recon, flux_type=flux)
    host, gpu, st = run_both(engine, ref, L, f, p, 4.0 / 3.0)
    assert st["error_word"] == 0
    for n in RHS_OUT:
        emax, el2 = errors(interior(L, n, gpu[n]), interior(L, n, host[n]))
        assert emax <= TOL, (n, emax, el2)


@pytest.mark.gpu
@pytest.mark.parametrize("fd_order", [2, 4])
def test_rhs_balsara_and_fd4(engine, ref, fd_order):
    L, f = W.balsara_box(n=(16, 8, 8), ng=5, seed=5)
    p = abi.default_params(reconstruction_method="ppm", flux_type="hlle",
                           local_spatial_order=fd_order)
    host, gpu, st = run_both(engine, ref, L, f, p, 5.0 / 3.0)
    for n in RHS_OUT:
        emax, el2 = errors(interior(L, n, gpu[n]), interior(L, n, host[n]))
        assert emax <= TOL, (n, emax, el2)
