"""Known answers of the reference's AsterX_Tmunu and regrid indicators as
the checker builds them (oracle/_ref), on the CPU: the checks that pin the
checker's wiring (field binding, loop ranges, interpolation order) before
the GPU tests compare the kernels with it.

* A uniform fluid at rest in flat space: T_tt = rho (1 + eps), T_ti = 0,
  T_ij = p delta_ij at every interior vertex, for both interpolation
  orders (both reproduce constants exactly).
* A uniform magnetic field added: T_ij gains b^2/2 delta_ij - b_i b_j.
* A linear ramp f = s x: first derivative and first gradient = |s| dx
  exactly, second derivative = 0.
"""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200.abi import Layout
from tests.helpers import full_fields


def uniform_box(L, rho=0.3, eps=0.7, press=0.14, B=(0.0, 0.0, 0.0)):
    f = full_fields(L, {})
    for n in ("gxx", "gyy", "gzz", "alp"):
        f[n][:] = 1.0
    f["rho"][:] = rho
    f["eps"][:] = eps
    f["press"][:] = press
    for d, n in enumerate(("Bvecx", "Bvecy", "Bvecz")):
        f[n][:] = B[d]
    for n in abi.TMUNU:
        f[n] = np.zeros(L.size)
    return f


@pytest.mark.parametrize("order", [2, 4])
def test_tmunu_fluid_at_rest(ref, order):
    L = Layout((6, 5, 4), 3, (0.1, 0.1, 0.1), (0.0, 0.0, 0.0))
    f = uniform_box(L)
    ref.setup(L, abi.default_params(), f)
    ref.tmunu(order)
    sl = L.interior((0, 0, 0))
    want = {"eTtt": 0.3 * 1.7, "eTxx": 0.14, "eTyy": 0.14, "eTzz": 0.14}
    for n in abi.TMUNU:
        v = L.view(f[n])[sl]
        assert np.allclose(v, want.get(n, 0.0), rtol=1e-14, atol=1e-15), n
    # only the interior vertices are written
    assert (f["eTtt"][:L.sy] == 0).all()


def test_tmunu_uniform_field(ref):
    L = Layout((5, 5, 5), 3, (0.1, 0.1, 0.1), (0.0, 0.0, 0.0))
    B = (0.2, -0.1, 0.05)
    f = uniform_box(L, B=B)
    ref.setup(L, abi.default_params(), f)
    ref.tmunu(2)
    sl = L.interior((0, 0, 0))
    b2 = sum(x * x for x in B)
    comps = {"eTxx": (0, 0), "eTxy": (0, 1), "eTxz": (0, 2), "eTyy": (1, 1),
             "eTyz": (1, 2), "eTzz": (2, 2)}
    for n, (i, j) in comps.items():
        want = 0.14 * (i == j) + 0.5 * b2 * (i == j) - B[i] * B[j]
        assert np.allclose(L.view(f[n])[sl], want, rtol=1e-13, atol=1e-15), n
    assert np.allclose(L.view(f["eTtt"])[sl], 0.3 * 1.7 + 0.5 * b2, rtol=1e-13)


@pytest.mark.parametrize("method,expect", [("first derivative", 0.25),
                                           ("first gradient", 0.25),
                                           ("second derivative", 0.0)])
def test_regrid_indicators_on_a_ramp(ref, method, expect):
    L = Layout((6, 5, 4), 2, (0.1, 0.1, 0.1), (0.0, 0.0, 0.0))
    ref.setup(L, abi.default_params(), full_fields(L, {}))
    i = np.arange(L.size) % L.sy
    ramp = 0.25 * i.astype(np.float64)  # slope 0.25 per point along x
    err = ref.estimate_error(abi.REGRID[method], [ramp])
    v = L.view(err)[L.interior((1, 1, 1))]
    assert np.allclose(v, expect, rtol=0, atol=1e-15), (method, v.min(), v.max())
