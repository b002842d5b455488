"""Batched level substep: one persistent launch per phase over boxes of
different shapes gives what one axb_substep per box gives (up to the
last-bit differences of the multiply-add contraction each kernel form
chooses, carried by the recovery to at most its tolerance), over a full
SSP-RK3 step, before and after the autotuner has changed the flux passes'
segment length and grid size; and the batched level against the reference
build box by box."""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import workloads as W
from tests.helpers import full_fields

SSPRK3 = [(0.0, 1.0, 1.0), (0.75, 0.25, 0.25), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)]
SHAPES = [(12, 10, 8), (8, 8, 8), (16, 8, 12), (10, 14, 9), (9, 9, 9), (20, 6, 7)]
EVOLVED = abi.CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]


def make_boxes(engine):
    boxes = []
    for q, n in enumerate(SHAPES):
        L, f = W.curved_box(n=n, ng=3, seed=40 + q, wmax=2.0, sigma=(1e-3, 0.3),
                            theta=(0.1, 1.0))
        W.cons_from_prims(L, f)
        W.saved_from_prims(f)
        f = full_fields(L, f)
        boxes.append((L, f))
    return boxes


def upload(engine, boxes):
    dev, devn = [], []
    for L, f in boxes:
        d = engine.upload(L, f)
        dev.append(d)
        devn.append({k: d[k].clone() for k in EVOLVED})
    return dev, devn


def rk3_step(engine, boxes, dev, devn, p, eos, batch=None):
    torch = engine.torch
    for s, (a, b, g) in enumerate(SSPRK3):
        if s == 0:
            for d, dn in zip(dev, devn):
                for k in EVOLVED:
                    dn[k].copy_(d[k])
        if batch is None:
            for (L, _), d, dn in zip(boxes, dev, devn):
                engine.substep(L, d, dn, p, eos, a, b, g, 0.25 * L.dx[0], periodic=True)
        else:
            # one dt for the level: all boxes here share the finest spacing rule
            engine.batch_substep(batch, a, b, g, DT, periodic=True)
    torch.cuda.synchronize()


DT = 0.01


@pytest.mark.gpu
@pytest.mark.parametrize("recon", ["wenoz", "mp5"])
def test_batch_matches_per_box(engine, recon):
    boxes = make_boxes(engine)
    p = abi.default_params(reconstruction_method=recon, flux_type="hlle",
                           c2p_prime="palenzuela", c2p_second="noble")
    eos = engine.eos_idealgas(4.0 / 3.0, rho=(1e-40, 1e10), eps=(0.0, 1e10))
    # per box, with the same dt for every box
    dev_a, devn_a = upload(engine, boxes)
    for s, (a, b, g) in enumerate(SSPRK3):
        if s == 0:
            for d, dn in zip(dev_a, devn_a):
                for k in EVOLVED:
                    dn[k].copy_(d[k])
        for (L, _), d, dn in zip(boxes, dev_a, devn_a):
            engine.substep(L, d, dn, p, eos, a, b, g, DT, periodic=True)
    engine.torch.cuda.synchronize()
    # batched, before and after tuning
    for tune in (False, True):
        dev_b, devn_b = upload(engine, boxes)
        batch = engine.batch_create([L for L, _ in boxes], dev_b, devn_b, p, eos)
        if tune:
            chosen = engine.batch_autotune(batch)
            assert chosen["seg_y"] in (8, 16, 32, 64) and chosen["ctas_per_sm"] in (2, 4, 8, 16)
            # the tuner leaves one RHS evaluation behind; the step below
            # recomputes it from the same state
        rk3_step(engine, boxes, dev_b, devn_b, p, eos, batch=batch)
        for q, ((L, _), da, db) in enumerate(zip(boxes, dev_a, dev_b)):
            for k in EVOLVED + ["rho", "velx", "eps", "press", "Bvecx", "con2prim_flag"]:
                x = da[k].cpu().numpy()
                y = db[k].cpu().numpy()
                if k == "con2prim_flag":
                    # a last-bit difference may move a bracket across the
                    # iteration cap: first and second scheme may swap
                    diff = x != y
                    ps = [abi.C2P_PRIME, abi.C2P_SECOND]
                    assert (np.isin(x[diff], ps) & np.isin(y[diff], ps)).all(), (tune, q, k)
                else:
                    # the flux kernels of the two forms fuse a few products
                    # into multiply-adds differently (contraction is decided
                    # per kernel): last-bit differences in some faces, which
                    # the recovery's Brent bracket (c2p_tol 1e-10) carries to
                    # at most its tolerance
                    sc = np.nanmax(np.abs(x)) or 1.0
                    assert np.nanmax(np.abs(x - y)) <= 1e-9 * sc, (tune, q, k)
        engine.batch_destroy(batch)


@pytest.mark.gpu
def test_batch_matches_reference(engine, ref):
    """Three boxes of different shapes advanced together by the batch (one
    full SSP-RK3 step, periodic fill per box) against the reference sources
    compiled on the host, run box by box (AsterX_RHSGroup, the stage
    combine, AsterX_Con2PrimGroup): recovery flags identical cell by cell
    (c2p_tol 1e-14, max_iter 100: no bracket near the cap), primitives and
    evolved variables within 1e-10 normalised and 1e-8 per point."""
    from tests.test_parity_full_gpu import (EVOLVED as EV, PRIM_OUT, TOL_STEP, TOL_STEP_PT,
                                            check_flags, compare, crop, ref_step,
                                            small_layout)
    gamma = 4.0 / 3.0
    shapes = [(12, 10, 8), (16, 8, 12), (10, 14, 9)]
    p = abi.default_params(reconstruction_method="wenoz", flux_type="hlle",
                           c2p_prime="palenzuela", c2p_second="noble", recon_type=1,
                           c2p_tol=1e-14, max_iter=100)
    big, small = [], []
    for q, n in enumerate(shapes):
        L5, f5 = W.curved_box(n=n, ng=5, seed=60 + q, wmax=5.0, sigma=(1e-3, 3.0))
        W.cons_from_prims(L5, f5)
        W.saved_from_prims(f5)
        f5 = full_fields(L5, f5)
        L3 = small_layout(L5)
        big.append((L5, f5))
        small.append((L3, {k: crop(L5, L3, a) for k, a in f5.items()}))
    dt = min(0.25 * L.dx[0] for L, _ in big)
    eos = engine.eos_idealgas(gamma, rho=(1e-40, 1e10), eps=(0.0, 1e10))
    dev, devn = upload(engine, small)
    batch = engine.batch_create([L for L, _ in small], dev, devn, p, eos)
    engine.status_reset()
    for s, (a, b, g) in enumerate(SSPRK3):
        if s == 0:
            for d, dn in zip(dev, devn):
                for k in EVOLVED:
                    dn[k].copy_(d[k])
        engine.batch_substep(batch, a, b, g, dt, periodic=True)
    engine.torch.cuda.synchronize()
    st = engine.status()
    engine.batch_destroy(batch)
    assert st["error_word"] & (abi.EW_NAN_FLUX | abi.EW_NAN_RHS) == 0
    for (L5, f5), (L3, _), d in zip(big, small, dev):
        host = {k: a.copy() for k, a in f5.items()}
        ref_step(ref, L5, host, p, gamma, dt, 3)
        got = {k: d[k].cpu().numpy() for k in d}
        check_flags(L3, L5, got, host, max_swaps=0.0)
        report = []
        compare(L3, L5, got, host, PRIM_OUT + EV, TOL_STEP, TOL_STEP_PT, report)
