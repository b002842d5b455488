"""StellarCollapse tables: the engine's conversion of a table's datasets
(axb_eos_stellarcollapse_convert, host code) against the reference's own
reader (eos_3p_tabulated3d::init, EOSX/src/eos_3p_tabulated3d/
eos_3p_tabulated3d.hxx:53-193, compiled unmodified, its HDF5 calls served
from memory by the stand-in header), and a recovery on the GPU with the EOS
built from the datasets against the reference with the EOS its reader
built."""
import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import eos_tables as T
from asterx_b200 import workloads as W
from tests.helpers import errors, full_fields, interior


def lib():
    from asterx_b200.engine import load_library
    return load_library()


@pytest.mark.parametrize("shift", [0.0, 2.0e19])
def test_convert_matches_reference_reader(ref, shift):
    ds = T.synthetic_datasets(energy_shift_cgs=shift)
    lr, lt, y, table, es, ranges = T.convert(lib(), ds)
    rlr, rlt, ry, rtable, res = ref.eos_stellarcollapse(ds)
    # bit for bit: the same operations in the same order on the same host libm
    assert np.array_equal(lr, rlr)
    assert np.array_equal(lt, rlt)
    assert np.array_equal(y, ry)
    assert np.array_equal(table, rtable)
    assert es == res
    assert np.array_equal(ranges, ref.tab_ranges())


def test_convert_rejects_bad_sizes():
    ds = T.synthetic_datasets()
    ds["cs2"] = ds["cs2"][:-1]
    with pytest.raises(ValueError):
        T.convert(lib(), ds)


@pytest.mark.gpu
def test_con2prim_with_stellarcollapse_table(engine, ref):
    ds = T.synthetic_datasets(nrho=40, ntemp=30, nye=12, energy_shift_cgs=2.0e19)
    L, f = W.tabulated_box(n=8, ng=5, seed=35, wmax=3.0, sigma=(1e-3, 0.3),
                           theta=(0.1, 1.0), temp_scale=0.5)
    W.cons_from_prims(L, f)
    W.perturbed_saved(f, seed=36)
    f = full_fields(L, f)
    p = abi.default_params(c2p_prime="palenzuela", c2p_second="noble", c2p_tol=1e-12,
                           max_iter=60, reconstruct_with_temperature=1)
    host = {n: a.copy() for n, a in f.items()}
    ref.setup(L, p, host)
    ref.eos_stellarcollapse(ds)
    ref.con2prim_group()
    eos = engine.eos_stellarcollapse(ds)
    dev = engine.upload(L, f)
    engine.status_reset()
    engine.con2prim_group(L, dev, p, eos)
    st = engine.status()
    got = {n: dev[n].cpu().numpy() for n in dev}
    flags = interior(L, "x", host["con2prim_flag"])
    assert np.array_equal(interior(L, "x", got["con2prim_flag"]), flags)
    assert (flags == abi.C2P_PRIME).mean() > 0.9
    assert st["error_word"] & 0x8 == 0
    for n in ["rho", "eps", "press", "velx", "temperature", "entropy", "Ye"] + abi.CONS:
        emax, _ = errors(interior(L, n, got[n]), interior(L, n, host[n]))
        assert emax <= 1e-10, (n, emax)
