"""Python driver for the CPU checkers (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module, and only to check or time against the engine.  It wraps
the same ``ora_*`` C ABI exported by

* ``oracle/_build/libaxo.so`` -- the oracle restatement (``oracle/axo.cpp``),
* ``oracle/_ref/libaxref.so`` -- the reference sources compiled through the
  stand-in headers (``oracle/refshim``),

so a test can run either on identical inputs.

Evaluation ranges: the engine computes every face, edge and vertex quantity
the interior update needs from the ghost data it is given, where the
reference instead synchronises those intermediates from neighbouring boxes.
``rhs_group`` therefore widens the reference loops onto ghost points (face
fluxes by one layer transversally, the vertex auxiliaries by two layers),
which reproduces exactly what a neighbouring box would have computed there.
Boxes passed to it need ng >= 5 so the widened stencils stay in bounds.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from asterx_b200.abi import Box, Layout, Params

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "libaxo.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libaxref.so")

_dp = C.POINTER(C.c_double)

# Grid functions the reference routines write that the engine never
# materialises (the hydro face fluxes and the upwind-CT face data); the
# checker allocates them itself when the caller does not pass them.
REF_ONLY_FIELDS = (
    [f"f{d}{v}" for d in "xyz" for v in
     ("dens", "momx", "momy", "momz", "tau", "DYe", "DEnt", "Bx", "By", "Bz")]
    + ["vtilde_y_xface", "vtilde_z_xface", "vtilde_x_yface", "vtilde_z_yface",
       "vtilde_x_zface", "vtilde_y_zface", "amax_xface", "amin_xface",
       "amax_yface", "amin_yface", "amax_zface", "amin_zface",
       "aster_mask_vc", "aster_mask_cc"]
    + ["eTtt", "eTtx", "eTty", "eTtz", "eTxx", "eTxy", "eTxz", "eTyy", "eTyz", "eTzz",
       "regrid_error"])


def _ptr(a):
    return a.ctypes.data_as(_dp)


class Oracle:
    """One CPU checker library plus the host arrays bound to it."""

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = C.CDLL(path)
        L = self.lib
        L.ora_setup.argtypes = [C.POINTER(Box), C.POINTER(Params), C.c_int]
        L.ora_bind.argtypes = [C.c_char_p, C.c_void_p]
        L.ora_set_ext.argtypes = [C.c_int, C.c_int]
        L.ora_last_error.restype = C.c_char_p
        L.ora_eos_idealgas.argtypes = [C.c_double] * 10
        L.ora_eos_tabulated.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp,
                                        _dp, C.c_double, C.c_double, C.c_double]
        L.ora_eos_tab_ranges.argtypes = [_dp]
        L.ora_reconstruct.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_int, _dp]
        L.ora_eigen.argtypes = [_dp, _dp]
        L.ora_riemann.argtypes = [C.c_int, _dp] + [C.c_double] * 4
        L.ora_riemann.restype = C.c_double
        L.ora_prim2con.argtypes = [_dp, _dp, _dp]
        if hasattr(L, "ora_tmunu"):
            L.ora_tmunu.argtypes = [C.c_int]
            L.ora_estimate_error.argtypes = [C.c_int, C.c_int, C.POINTER(_dp), C.c_double]
        L.ora_c2p_point.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp,
                                    C.POINTER(C.c_int)]
        L.ora_eos_tab_query.argtypes = [C.c_int, C.c_double, C.c_double,
                                        C.c_double, _dp]
        L.ora_eos_tab_query.restype = C.c_double
        self._keep = []

    # -- set-up -------------------------------------------------------------
    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ora_last_error().decode())

    def setup(self, layout: Layout, params: Params, fields: dict, iteration=0):
        self.layout = layout
        self._box = layout.box()
        self._params = params
        self._check(self.lib.ora_setup(C.byref(self._box), C.byref(params),
                                       iteration))
        self._keep = []
        fields = dict(fields)
        for name in REF_ONLY_FIELDS:
            if name not in fields:
                fields[name] = (np.ones(layout.size) if name.startswith("aster_mask")
                                else np.zeros(layout.size))
        self.fields = fields
        for name, arr in fields.items():
            assert arr.dtype == np.float64 and arr.flags.c_contiguous
            self._keep.append(arr)
            self.lib.ora_bind(name.encode(), arr.ctypes.data)

    def eos_idealgas(self, gamma, umass=1.0, rho=(1e-40, 1.0), eps=(0.0, 2.0),
                     ye=(0.0, 1.0), poly_gamma=2.0, poly_k=100.0):
        self._check(self.lib.ora_eos_idealgas(gamma, umass, rho[0], rho[1],
                                              eps[0], eps[1], ye[0], ye[1],
                                              poly_gamma, poly_k))

    def eos_tabulated(self, logrho, logtemp, ye, table, energy_shift=0.0,
                      poly_gamma=2.0, poly_k=100.0):
        self._tab = [np.ascontiguousarray(a, dtype=np.float64)
                     for a in (logrho, logtemp, ye, table)]
        lr, lt, y, t = self._tab
        self._check(self.lib.ora_eos_tabulated(len(lr), len(lt), len(y), _ptr(lr),
                                               _ptr(lt), _ptr(y), _ptr(t),
                                               energy_shift, poly_gamma, poly_k))

    def eos_stellarcollapse(self, datasets, poly_gamma=2.0, poly_k=100.0):
        """The reference's own StellarCollapse reader (eos_3p_tabulated3d::init)
        on `datasets` served by the stand-in HDF5; returns the converted
        (logrho, logtemp, ye, table, energy_shift)."""
        L = self.lib
        L.ora_h5_clear()
        L.ora_h5_put_double.argtypes = [C.c_char_p, _dp, C.c_long]
        L.ora_h5_put_int.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.c_long]
        L.ora_eos_stellarcollapse.argtypes = [C.c_double, C.c_double]
        L.ora_eos_tab_export.argtypes = [_dp] * 5
        self._h5 = []
        for k, v in datasets.items():
            if k.startswith("points"):
                a = np.array([int(v)], dtype=np.int32)
                L.ora_h5_put_int(k.encode(), a.ctypes.data_as(C.POINTER(C.c_int)), 1)
            else:
                a = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
                L.ora_h5_put_double(k.encode(), _ptr(a), a.size)
            self._h5.append(a)
        self._check(L.ora_eos_stellarcollapse(poly_gamma, poly_k))
        nrho, ntemp, nye = (int(datasets[k]) for k in ("pointsrho", "pointstemp", "pointsye"))
        lr, lt, y = np.empty(nrho), np.empty(ntemp), np.empty(nye)
        table = np.empty(19 * nrho * ntemp * nye)
        es = np.empty(1)
        L.ora_eos_tab_export(_ptr(lr), _ptr(lt), _ptr(y), _ptr(table), _ptr(es))
        return lr, lt, y, table, float(es[0])

    def tab_ranges(self):
        out = np.zeros(8)
        self.lib.ora_eos_tab_ranges(_ptr(out))
        return out

    # -- scheduled routines ---------------------------------------------------
    def run(self, routine, ext_c=0, ext_v=0):
        self.lib.ora_set_ext(ext_c, ext_v)
        self._check(getattr(self.lib, "ora_" + routine)())
        self.lib.ora_set_ext(0, 0)

    def rhs_group(self):
        """AsterX_RHSGroup (AsterX/schedule.ccl:169-228): Fluxes, SourceTerms,
        RHS, with the fluxes and auxiliaries widened onto ghost points (the
        fluxes by three cell layers with upwind CT, whose edge
        reconstructions reach three faces out)."""
        assert self.layout.ng >= 5
        self.run("fluxes", ext_c=3 if self._params.use_uct else 1, ext_v=2)
        self.run("sources")
        self.run("rhs")

    def con2prim_group(self):
        """AsterX_Con2PrimGroup (AsterX/schedule.ccl:119-165): curl A on the
        interior faces widened by one transverse layer, centred dB, c2p."""
        self.run("bstag", ext_c=3 if self._params.use_uct else 1)
        self.run("dB")
        self.run("c2p")

    def tmunu(self, interp_order=2):
        """AsterX_Tmunu: adds T_{mu nu} to the bound eTtt .. eTzz."""
        self._check(self.lib.ora_tmunu(interp_order))

    def estimate_error(self, method, arrays, epsilon_err=0.0):
        """AsterX_EstimateError's loop with the reference's indicators over
        `arrays` (the box's layout); returns the bound regrid_error."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in arrays]
        ptrs = (_dp * len(arrs))(*[_ptr(a) for a in arrs])
        self._check(self.lib.ora_estimate_error(method, len(arrs), ptrs, epsilon_err))
        return self.fields["regrid_error"]

    # -- per-point ------------------------------------------------------------
    def reconstruct(self, method, v, press=None, vel=None, is_rho=False,
                    is_press=False):
        v = np.ascontiguousarray(v, dtype=np.float64)
        press = np.ones(6) if press is None else np.ascontiguousarray(press, dtype=np.float64)
        vel = np.zeros(6) if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        out = np.zeros(2)
        self.lib.ora_reconstruct(method, _ptr(v), _ptr(press), _ptr(vel),
                                 int(is_rho), int(is_press), _ptr(out))
        return out

    def eigen(self, alp, beta, u, vel, rho, cs2, w, h, bsq):
        inp = np.array([alp, beta, u, *vel, *rho, *cs2, *w, *h, *bsq],
                       dtype=np.float64)
        lam = np.zeros(8)
        self.lib.ora_eigen(_ptr(inp), _ptr(lam))
        return lam

    def riemann(self, flux_type, lam, uL, uR, fL, fR):
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        return self.lib.ora_riemann(flux_type, _ptr(lam), uL, uR, fL, fR)

    def prim2con(self, g6, prim):
        g6 = np.ascontiguousarray(g6, dtype=np.float64)
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        cons = np.zeros(10)
        self.lib.ora_prim2con(_ptr(g6), _ptr(prim), _ptr(cons))
        return cons

    def c2p_point(self, solver, cons, g6, seed, atmo):
        cons = np.array(cons, dtype=np.float64)
        g6 = np.ascontiguousarray(g6, dtype=np.float64)
        seed = np.ascontiguousarray(seed, dtype=np.float64)
        atmo = np.ascontiguousarray(atmo, dtype=np.float64)
        prim = np.zeros(16)
        rep = (C.c_int * 3)()
        self._check(self.lib.ora_c2p_point(solver, _ptr(cons), _ptr(g6),
                                           _ptr(seed), _ptr(atmo), _ptr(prim),
                                           rep))
        return prim, cons, tuple(rep)

    def tab_query(self, which, rho, x, ye):
        e = C.c_double(0.0)
        r = self.lib.ora_eos_tab_query(which, rho, x, ye, C.byref(e))
        return r, e.value


def reference():
    """The reference-compiled checker, or None when it was not built."""
    return Oracle(REFERENCE_SO) if os.path.exists(REFERENCE_SO) else None


def restatement():
    return Oracle(RESTATEMENT_SO)
