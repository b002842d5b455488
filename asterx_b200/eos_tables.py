"""StellarCollapse EOS tables for the tabulated3d EOS.

The reference reads the table's HDF5 file itself (eos_3p_tabulated3d::init,
EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:53-193) and converts it.
Here the file is read by the caller's HDF5 binding (``read_stellarcollapse``
uses h5py when it is installed; no HDF5 library is linked into the engine)
and the conversion is the engine's (``axb_eos_stellarcollapse_convert``,
host code, no device needed):

* ``read_stellarcollapse(path)`` -- the datasets as the file holds them;
* ``convert(lib, ds)`` -- init's conversion: natural logs in code units,
  19 variables interleaved per node, the ranges init sets;
* ``Engine.eos_stellarcollapse(ds)`` -- the device EOS from the datasets.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

# the 19 datasets of a StellarCollapse table, in the reference's order
# (eos_3p_tabulated3d.hxx:101-104)
DATASETS = ["logpress", "logenergy", "entropy", "munu", "cs2", "dedt", "dpdrhoe",
            "dpderho", "muhat", "mu_e", "mu_p", "mu_n", "Xa", "Xh", "Xn", "Xp", "Abar",
            "Zbar", "gamma"]
_dp = C.POINTER(C.c_double)


def read_stellarcollapse(path):
    """The datasets of a StellarCollapse HDF5 table: pointsrho, pointstemp,
    pointsye, logrho, logtemp, ye, energy_shift and DATASETS (each flattened
    with rho fastest, as stored)."""
    try:
        import h5py
    except ImportError as e:  # pragma: no cover - depends on the install
        raise ImportError("reading an HDF5 table needs h5py; pass the datasets "
                          "to convert() / Engine.eos_stellarcollapse() instead") from e
    out = {}
    with h5py.File(path, "r") as fh:
        for k in ("pointsrho", "pointstemp", "pointsye"):
            out[k] = int(np.asarray(fh[k]).reshape(-1)[0])
        for k in ["logrho", "logtemp", "ye", "energy_shift"] + DATASETS:
            out[k] = np.ascontiguousarray(np.asarray(fh[k], dtype=np.float64).reshape(-1))
    return out


def _args(ds):
    nrho, ntemp, nye = int(ds["pointsrho"]), int(ds["pointstemp"]), int(ds["pointsye"])
    nodes = nrho * ntemp * nye
    axes = [np.ascontiguousarray(ds[k], dtype=np.float64) for k in ("logrho", "logtemp", "ye")]
    sets = [np.ascontiguousarray(ds[k], dtype=np.float64).reshape(-1) for k in DATASETS]
    if [a.size for a in axes] != [nrho, ntemp, nye] or any(s.size != nodes for s in sets):
        raise ValueError("dataset sizes do not match pointsrho/pointstemp/pointsye")
    ptrs = (_dp * len(sets))(*[s.ctypes.data_as(_dp) for s in sets])
    shift = float(np.asarray(ds["energy_shift"]).reshape(-1)[0])
    return (nrho, ntemp, nye), axes, sets, ptrs, shift


def bind(lib):
    lib.axb_eos_stellarcollapse_convert.argtypes = [
        C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.POINTER(_dp), C.c_double, _dp, _dp, _dp,
        _dp, _dp, _dp]
    lib.axb_eos_create_stellarcollapse.argtypes = [
        C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.POINTER(_dp), C.c_double, C.c_double,
        C.c_double, C.POINTER(C.c_void_p)]


def convert(lib, ds):
    """init's conversion of the datasets: (logrho, logtemp, ye, table,
    energy_shift, ranges[8]) in the layout axb_eos_create_tabulated3d takes."""
    bind(lib)
    (nrho, ntemp, nye), axes, sets, ptrs, shift = _args(ds)
    lr, lt, y = np.empty(nrho), np.empty(ntemp), np.empty(nye)
    table = np.empty(19 * nrho * ntemp * nye)
    es = C.c_double()
    ranges = np.empty(8)
    rc = lib.axb_eos_stellarcollapse_convert(
        nrho, ntemp, nye, *[a.ctypes.data_as(_dp) for a in axes], ptrs, shift,
        lr.ctypes.data_as(_dp), lt.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
        table.ctypes.data_as(_dp), C.byref(es), ranges.ctypes.data_as(_dp))
    if rc != 0:
        raise RuntimeError(f"axb_eos_stellarcollapse_convert failed: {rc}")
    return lr, lt, y, table, es.value, ranges


# synthetic StellarCollapse datasets (tests): the synthetic table of
# workloads.synthetic_table written back in the file's units and layout
_LENGTHGF = 6.77269222552442e-06
_TIMEGF = 2.03040204956746e05
_RHOGF = 1.61887093132742e-18
_PRESSGF = 1.80123683248503e-39
_EPSGF = 1.11265005605362e-21


def synthetic_datasets(nrho=20, ntemp=12, nye=8, energy_shift_cgs=2.0e19, seed=3):
    """A table in the file's form (log10 CGS axes, one array per variable,
    rho fastest) whose conversion gives the thermodynamics of
    workloads.tab_thermo (in code units) plus seeded values for the
    variables the engine does not read."""
    from .workloads import tab_thermo
    rho_c = np.exp(np.linspace(np.log(1e-12), np.log(1e-2), nrho))
    temp = np.exp(np.linspace(np.log(0.01), np.log(100.0), ntemp))
    ye = np.linspace(0.05, 0.6, nye)
    Y, T, R = np.meshgrid(ye, temp, rho_c, indexing="ij")  # (ye, T, rho): rho fastest
    press, eps, ent, cs2 = tab_thermo(R, T, Y)
    shift = energy_shift_cgs * _EPSGF
    rng = np.random.default_rng(seed)
    ds = {"pointsrho": nrho, "pointstemp": ntemp, "pointsye": nye,
          "logrho": np.log10(rho_c / _RHOGF), "logtemp": np.log10(temp), "ye": ye,
          "energy_shift": np.array([energy_shift_cgs])}
    for k in DATASETS:
        ds[k] = rng.uniform(-1.0, 1.0, R.size)
    ds["logpress"] = np.log10((press / _PRESSGF).reshape(-1))
    ds["logenergy"] = np.log10(((eps + shift) / _EPSGF).reshape(-1))
    ds["entropy"] = ent.reshape(-1)
    ds["cs2"] = (cs2 / (_LENGTHGF ** 2 / _TIMEGF ** 2)).reshape(-1)
    return ds
