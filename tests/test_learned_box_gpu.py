"""The learned guess inside the box recovery (axb_con2prim_group_guess): on
a curved-metric box whose recovery seeds are cold (half the density, a
small eps, v = 0, as a fresh patch or a regridded one may have them), the
guessed recovery gives the plain one's primitives (flags identical but
for rare cells the guessed Noble start recovers where the plain one needed
the second scheme) and Noble takes fewer steps; with Palenzuela first the
guessed bracket gives the plain primitives.  Runs on the GPU only; the
network is trained there by the engine's kernels."""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import workloads as W
from tests.helpers import errors, full_fields, interior
from tests.test_learned_gpu import train_guess

GAMMA = 5.0 / 3.0
EOS_KW = dict(rho=(1e-40, 1e10), eps=(0.0, 1e10))
PRIMS = ["rho", "eps", "press", "velx", "vely", "velz"]


def cold_box(n=24):
    L, f = W.curved_box(n=n, ng=3, seed=31, gamma=GAMMA, wmax=3.0, sigma=(1e-3, 0.3),
                        theta=(0.1, 1.0))
    W.cons_from_prims(L, f)
    f = full_fields(L, f)
    # cold seeds: half the density, a small eps, no velocity
    f["saved_rho"] = f["rho"] * 0.5
    f["saved_eps"] = np.full_like(f["rho"], 1e-3)
    for ax in "xyz":
        f["saved_vel" + ax] = np.zeros_like(f["rho"])
    f["saved_Ye"] = f["Ye"].copy()
    return L, f


def mean_iters(hist):
    h = np.asarray(hist, dtype=np.float64)
    return float((h * np.arange(h.size)).sum() / max(h.sum(), 1.0))


@pytest.mark.gpu
@pytest.mark.parametrize("prime,second", [("noble", "palenzuela"), ("palenzuela", "noble")])
def test_box_recovery_with_learned_guess(engine, prime, second):
    L, f = cold_box()
    rho = interior(L, "rho", f["rho"])
    eps = interior(L, "eps", f["eps"])
    mlp, final = train_guess(engine, 1 << 16, 505, GAMMA, "relu",
                             rho_range=(float(rho.min()), float(rho.max())),
                             eps_range=(float(eps.min()), float(eps.max())),
                             w_range=(1.0, 3.0), sigma_range=(1e-3, 0.3))
    assert np.isfinite(final)
    p = abi.default_params(c2p_prime=prime, c2p_second=second, c2p_tol=1e-12,
                           max_iter=100, vw_lim=1e3, B_lim=1e4)
    eos = engine.eos_idealgas(GAMMA, **EOS_KW)
    out = {}
    for name, m in (("plain", None), ("learned", mlp)):
        dev = engine.upload(L, f)
        engine.status_reset()
        engine.con2prim_group(L, dev, p, eos, mlp=m)
        st = engine.status()
        out[name] = ({k: dev[k].cpu().numpy() for k in PRIMS + ["con2prim_flag"]}, st)
    (a, sa), (b, sb) = out["plain"], out["learned"]
    fa = interior(L, "x", a["con2prim_flag"])
    fb = interior(L, "x", b["con2prim_flag"])
    same = fa == fb
    # a guessed Noble start may recover a cell whose plain start needed the
    # second scheme; nothing else may change
    swaps = ~same & (fa == abi.C2P_SECOND) & (fb == abi.C2P_PRIME)
    assert np.all(same | swaps)
    assert swaps.mean() < 0.01
    assert (fa == abi.C2P_PRIME).mean() > 0.9
    both = same & (fa == abi.C2P_PRIME)
    for k in PRIMS:
        x = interior(L, k, b[k])[both]
        y = interior(L, k, a[k])[both]
        emax, _ = errors(x, y)
        assert emax <= 1e-10, (k, emax)
    assert sb["c2p_fail"] == sa["c2p_fail"]
    ia, ib = mean_iters(sa["iter_hist"]), mean_iters(sb["iter_hist"])
    if prime == "noble":
        # the guess replaces cold seeds: far fewer Newton steps
        assert ib < 0.7 * ia, (ib, ia)
