"""Grid functions in the caller's own per-centring layouts (as CarpetX
allocates each centring of a box: a cell-centred field one point shorter
per cell direction than a vertex-centred one, each with its own j and k
strides), carried into the engine's one-layout box by axb_import_fields and
back by axb_export_fields.

The RHS group run on fields imported from per-centring layouts and exported
back must give exactly the RHS of the same box run in the engine's layout,
and a round trip leaves every point of every centring unchanged."""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import workloads as W
from asterx_b200.driver import CENTRING
from tests.helpers import full_fields

INPUTS = ([n for n in abi.GF_NAMES if n.startswith(("g", "k")) and len(n) == 3] +
          ["alp", "betax", "betay", "betaz", "rho", "velx", "vely", "velz", "eps", "press",
           "temperature", "Ye", "entropy", "Bvecx", "Bvecy", "Bvecz", "dBx_stag", "dBy_stag",
           "dBz_stag", "Avec_x", "Avec_y", "Avec_z", "Psi"])
OUTPUTS = abi.HYDRO_RHS + abi.AVEC_RHS


def per_centring(L, name):
    """Extents and strides of `name`'s own allocation (no padding)."""
    c = CENTRING.get(name, (1, 1, 1))
    N = [L.n[d] + 2 * L.ng + (0 if c[d] else 1) for d in range(3)]
    return N, N[0], N[0] * N[1]


def to_strided(engine, L, arr, name):
    N, sy, sz = per_centring(L, name)
    v = L.view(arr)[:N[2], :N[1], :N[0]]
    t = engine.torch.as_tensor(np.ascontiguousarray(v).reshape(-1), device=engine.device)
    return t, sy, sz


@pytest.mark.gpu
def test_rhs_group_through_per_centring_layouts(engine):
    torch = engine.torch
    L, f = W.curved_box(n=(14, 10, 12), ng=3, seed=51, wmax=3.0, sigma=(1e-3, 0.3))
    f = full_fields(L, f)
    p = abi.default_params(reconstruction_method="wenoz", flux_type="hlle")
    eos = engine.eos_idealgas(4.0 / 3.0, rho=(1e-40, 1e10), eps=(0.0, 1e10))
    # the engine's own layout
    dev = engine.upload(L, f)
    engine.rhs_group(L, dev, p, eos)
    want = {n: dev[n].cpu().numpy() for n in OUTPUTS}
    # the caller's per-centring layouts: import, RHS group, export
    strided_in = {n: to_strided(engine, L, f[n], n) for n in INPUTS}
    strided_out = {}
    for n in OUTPUTS:
        N, sy, sz = per_centring(L, n)
        strided_out[n] = (torch.full((N[0] * N[1] * N[2],), float("nan"), dtype=torch.float64,
                                     device=engine.device), sy, sz)
    work = engine.upload(L, {}, names=abi.GF_NAMES)
    engine.import_fields(L, strided_in, INPUTS, work)
    engine.rhs_group(L, work, p, eos)
    engine.export_fields(L, work, OUTPUTS, strided_out)
    torch.cuda.synchronize()
    for n in OUTPUTS:
        N, sy, sz = per_centring(L, n)
        got = strided_out[n][0].cpu().numpy().reshape(N[2], N[1], N[0])
        c = CENTRING.get(n, (1, 1, 1))
        sl = L.interior(c)
        ref = L.view(want[n])[sl]
        assert np.array_equal(got[sl], ref), n


@pytest.mark.gpu
def test_import_export_round_trip(engine):
    torch = engine.torch
    L = abi.Layout((9, 7, 5), 3, (0.1, 0.1, 0.1), (0.0, 0.0, 0.0))
    rng = np.random.default_rng(3)
    names = ["rho", "Avec_x", "Avec_y", "Avec_z", "Psi", "dBx_stag", "dBy_stag", "dBz_stag",
             "fxBy", "fyBz", "fzBx", "G"]
    src = {}
    for n in names:
        N, sy, sz = per_centring(L, n)
        src[n] = (torch.as_tensor(rng.normal(size=N[0] * N[1] * N[2]), device=engine.device),
                  sy, sz)
    work = engine.upload(L, {}, names=abi.GF_NAMES)
    engine.import_fields(L, src, names, work)
    back = {n: (torch.zeros_like(t), sy, sz) for n, (t, sy, sz) in src.items()}
    engine.export_fields(L, work, names, back)
    torch.cuda.synchronize()
    for n in names:
        assert torch.equal(back[n][0], src[n][0]), n
