"""ctypes mirror of ``include/asterx_b200.h`` (box, grid-function ids,
parameters) and the numpy-side box layout.

The structures here must match the C header field for field;
``tests/test_abi.py`` checks sizes and offsets against the compiled library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

GF_NAMES = [
    # ADMBaseX, vertex-centred
    "gxx", "gxy", "gxz", "gyy", "gyz", "gzz", "alp", "betax", "betay", "betaz",
    "kxx", "kxy", "kxz", "kyy", "kyz", "kzz",
    # HydroBaseX primitives
    "rho", "velx", "vely", "velz", "eps", "press", "temperature", "Ye",
    "entropy", "Bvecx", "Bvecy", "Bvecz",
    # conserved and RHS
    "dens", "momx", "momy", "momz", "tau", "DYe", "DEnt",
    "densrhs", "momxrhs", "momyrhs", "momzrhs", "taurhs", "DYe_rhs", "DEntrhs",
    # vector potential
    "Avec_x", "Avec_y", "Avec_z", "Psi",
    "Avec_x_rhs", "Avec_y_rhs", "Avec_z_rhs", "Psi_rhs",
    # magnetic field
    "dBx_stag", "dBy_stag", "dBz_stag", "dBx", "dBy", "dBz",
    # c2p bookkeeping
    "con2prim_flag", "saved_rho", "saved_velx", "saved_vely", "saved_velz",
    "saved_eps", "saved_Ye",
    "zvec_x", "zvec_y", "zvec_z", "svec_x", "svec_y", "svec_z",
    # scratch
    "Fx", "Fy", "Fz", "Fbetax", "Fbetay", "Fbetaz", "G",
    "fxBy", "fxBz", "fyBx", "fyBz", "fzBx", "fzBy",
    "acc_dens", "acc_momx", "acc_momy", "acc_momz", "acc_tau", "acc_DYe",
    "acc_DEnt",
    # upwind CT face data
    "vtilde_y_xface", "vtilde_z_xface", "vtilde_z_yface", "vtilde_x_yface",
    "vtilde_x_zface", "vtilde_y_zface", "amax_xface", "amin_xface",
    "amax_yface", "amin_yface", "amax_zface", "amin_zface",
]
GF = {n: i for i, n in enumerate(GF_NAMES)}
NUM_GF = len(GF_NAMES)

METRIC = ["gxx", "gxy", "gxz", "gyy", "gyz", "gzz", "alp", "betax", "betay",
          "betaz"]
CURV = ["kxx", "kxy", "kxz", "kyy", "kyz", "kzz"]
PRIMS = ["rho", "velx", "vely", "velz", "eps", "press", "temperature", "Ye",
         "entropy", "Bvecx", "Bvecy", "Bvecz"]
CONS = ["dens", "momx", "momy", "momz", "tau", "DYe", "DEnt"]
HYDRO_RHS = ["densrhs", "momxrhs", "momyrhs", "momzrhs", "taurhs", "DYe_rhs",
             "DEntrhs"]
AVEC = ["Avec_x", "Avec_y", "Avec_z", "Psi"]
AVEC_RHS = ["Avec_x_rhs", "Avec_y_rhs", "Avec_z_rhs", "Psi_rhs"]
SAVED = ["saved_rho", "saved_velx", "saved_vely", "saved_velz", "saved_eps",
         "saved_Ye"]
AUX = ["Fx", "Fy", "Fz", "Fbetax", "Fbetay", "Fbetaz", "G"]
BFLUX = ["fxBy", "fxBz", "fyBx", "fyBz", "fzBx", "fzBy"]
ACC = ["acc_dens", "acc_momx", "acc_momy", "acc_momz", "acc_tau", "acc_DYe",
       "acc_DEnt"]
UCT = ["vtilde_y_xface", "vtilde_z_xface", "amax_xface", "amin_xface",
       "vtilde_z_yface", "vtilde_x_yface", "amax_yface", "amin_yface",
       "vtilde_x_zface", "vtilde_y_zface", "amax_zface", "amin_zface"]
# centring (x, y, z; 1 = cell, 0 = vertex) of the upwind-CT face data
UCT_CENT = {n: {"x": (0, 1, 1), "y": (1, 0, 1), "z": (1, 1, 0)}[n[-5]] for n in UCT}

RECON = {"godunov": 0, "minmod": 1, "monocentral": 2, "ppm": 3, "eppm": 4,
         "wenoz": 5, "mp5": 6}
FLUX = {"lxf": 0, "hlle": 1}
C2P = {"none": 0, "noble": 1, "palenzuela": 2, "entropy": 3}

# c2p cell flags (AsterX/src/con2prim.cxx:27-35)
C2P_INIT, C2P_PRIME, C2P_SECOND, C2P_ENTROPY, C2P_ATMO, C2P_AVG, C2P_FAIL = range(7)
# outer-boundary rules (axb_bc)
BC_PERIODIC, BC_NEUMANN, BC_LINEAR = 0, 1, 2
# regrid error indicators (axb_regrid), by the regrid_method keyword
REGRID = {"first derivative": 0, "second derivative": 1, "second derivative norm": 2,
          "first gradient": 3}
# the stress-energy tensor components, in the order axb_tmunu takes them
TMUNU = ["eTtt", "eTtx", "eTty", "eTtz", "eTxx", "eTxy", "eTxz", "eTyy", "eTyz", "eTzz"]
# device error-word bits (AXB_EW_* in include/asterx_b200.h)
EW_NAN_FLUX, EW_NAN_RHS, EW_C2P_FAIL, EW_ROOT_CAP, EW_QUEUE_TIMEOUT = 1, 2, 4, 8, 16


class Box(C.Structure):
    _fields_ = [("n", C.c_int32 * 3), ("ng", C.c_int32), ("sy", C.c_int64),
                ("sz", C.c_int64), ("dx", C.c_double * 3),
                ("xmin", C.c_double * 3)]


class Fields(C.Structure):
    _fields_ = [("gf", C.c_void_p * NUM_GF)]


class FieldsStrided(C.Structure):
    """axb_fields_strided: one pointer and its own (sy, sz) per grid function."""
    _fields_ = [("gf", C.c_void_p * NUM_GF), ("sy", C.c_int64 * NUM_GF),
                ("sz", C.c_int64 * NUM_GF)]


# independent cells for axb_c2p_cells / axb_mlp_features (axb_cells)
CELL_INPUTS = ["dens", "momx", "momy", "momz", "tau", "DYe", "DEnt", "dBx", "dBy", "dBz",
               "gxx", "gxy", "gxz", "gyy", "gyz", "gzz"]
CELL_SEEDS = ["seed_rho", "seed_eps", "seed_Ye", "seed_velx", "seed_vely", "seed_velz",
              "seed_temperature"]
CELL_OUTPUTS = ["rho", "eps", "press", "velx", "vely", "velz", "w_lorentz", "Ye",
                "temperature", "entropy", "iters", "flag"]


class Cells(C.Structure):
    _fields_ = [("n", C.c_int64), ("dens", C.c_void_p), ("mom", C.c_void_p * 3),
                ("tau", C.c_void_p), ("DYe", C.c_void_p), ("DEnt", C.c_void_p),
                ("dB", C.c_void_p * 3), ("g", C.c_void_p * 6),
                ("seed_rho", C.c_void_p), ("seed_eps", C.c_void_p), ("seed_Ye", C.c_void_p),
                ("seed_vel", C.c_void_p * 3), ("seed_temperature", C.c_void_p),
                ("rho", C.c_void_p), ("eps", C.c_void_p), ("press", C.c_void_p),
                ("vel", C.c_void_p * 3), ("w_lorentz", C.c_void_p), ("Ye", C.c_void_p),
                ("temperature", C.c_void_p), ("entropy", C.c_void_p),
                ("iters", C.c_void_p), ("flag", C.c_void_p), ("guess", C.c_void_p),
                ("fallback", C.c_void_p)]


def cells_struct(n, arrays: dict):
    """axb_cells from a dict of device pointers (ints) keyed by the names of
    CELL_INPUTS / CELL_SEEDS / CELL_OUTPUTS; missing names stay NULL."""
    c = Cells()
    c.n = int(n)
    get = lambda k: arrays.get(k)
    c.dens, c.tau, c.DYe, c.DEnt = get("dens"), get("tau"), get("DYe"), get("DEnt")
    for q, ax in enumerate("xyz"):
        c.mom[q] = get("mom" + ax)
        c.dB[q] = get("dB" + ax)
        c.seed_vel[q] = get("seed_vel" + ax)
        c.vel[q] = get("vel" + ax)
    for q, nm in enumerate(["gxx", "gxy", "gxz", "gyy", "gyz", "gzz"]):
        c.g[q] = get(nm)
    for nm in ("seed_rho", "seed_eps", "seed_Ye", "seed_temperature", "rho", "eps",
               "press", "w_lorentz", "Ye", "temperature", "entropy", "iters", "flag",
               "guess", "fallback"):
        setattr(c, nm, get(nm))
    return c


_PARAM_INTS_1 = ["reconstruction_method", "loworder_method",
                 "reconstruct_with_temperature", "ppm_shock_detection",
                 "ppm_zone_flattening"]
_PARAM_DBL_1 = ["ppm_eta1", "ppm_eta2", "ppm_eps", "ppm_eps_shock", "ppm_small",
                "ppm_omega1", "ppm_omega2", "enhanced_ppm_C2", "weno_eps",
                "mp5_alpha", "poly_k", "poly_gamma"]
_PARAM_INTS_2 = ["flux_type", "recon_type", "vector_potential_gauge",
                 "local_spatial_order", "use_uct", "use_entropy_fix", "excise",
                 "use_mask"]
_PARAM_DBL_2 = ["lorenz_damp_fac"]
_PARAM_INTS_3 = ["c2p_prime", "c2p_second", "max_iter", "thermal_eos_atmo",
                 "use_press_atmo", "use_z", "use_temperature", "Ye_lenient"]
_PARAM_DBL_3 = ["c2p_tol", "rho_abs_min", "atmo_tol", "eps_atmo", "p_atmo",
                "t_atmo", "Ye_atmo", "r_atmo", "n_rho_atmo", "n_press_atmo",
                "n_temp_atmo", "alp_thresh", "rho_BH", "eps_BH", "vwlim_BH",
                "cons_error_limit", "vw_lim", "B_lim"]


class Params(C.Structure):
    _fields_ = ([(n, C.c_int32) for n in _PARAM_INTS_1] +
                [(n, C.c_double) for n in _PARAM_DBL_1] +
                [(n, C.c_int32) for n in _PARAM_INTS_2] +
                [(n, C.c_double) for n in _PARAM_DBL_2] +
                [(n, C.c_int32) for n in _PARAM_INTS_3] +
                [(n, C.c_double) for n in _PARAM_DBL_3])


def default_params(**over) -> Params:
    """The reference's param.ccl defaults (ReconX/param.ccl, AsterX/param.ccl,
    Con2PrimFactory/param.ccl, EOSX/param.ccl), then ``over``."""
    p = Params()
    d = dict(
        reconstruction_method=RECON["godunov"], loworder_method=RECON["godunov"],
        reconstruct_with_temperature=0, ppm_shock_detection=1,
        ppm_zone_flattening=0, ppm_eta1=20.0, ppm_eta2=0.05, ppm_eps=0.33,
        ppm_eps_shock=0.01, ppm_small=1e-7, ppm_omega1=0.75, ppm_omega2=10.0,
        enhanced_ppm_C2=1.25, weno_eps=1e-26, mp5_alpha=4.0, poly_k=100.0,
        poly_gamma=2.0, flux_type=FLUX["lxf"], recon_type=0,
        vector_potential_gauge=1, local_spatial_order=2, use_uct=0,
        use_entropy_fix=0, excise=0, use_mask=0, lorenz_damp_fac=0.0,
        c2p_prime=C2P["noble"], c2p_second=C2P["palenzuela"], max_iter=30,
        thermal_eos_atmo=1, use_press_atmo=0, use_z=0, use_temperature=0,
        Ye_lenient=0, c2p_tol=1e-10, rho_abs_min=1e-13, atmo_tol=1e-3,
        eps_atmo=1e-10, p_atmo=1e-10, t_atmo=1e-2, Ye_atmo=0.5, r_atmo=1e100,
        n_rho_atmo=0.0, n_press_atmo=0.0, n_temp_atmo=0.0, alp_thresh=0.0,
        rho_BH=1e100, eps_BH=1e100, vwlim_BH=1e100, cons_error_limit=-1.0,
        vw_lim=10.0, B_lim=100.0)
    for k, v in over.items():
        if isinstance(v, str):
            v = {"reconstruction_method": RECON, "loworder_method": RECON,
                 "flux_type": FLUX, "c2p_prime": C2P,
                 "c2p_second": C2P}[k][v.lower()]
        d[k] = v
    for k, v in d.items():
        setattr(p, k, v)
    return p


@dataclass
class Layout:
    """Index layout of one box: every grid function is a flat FP64 array
    ``f[i + sy*j + sz*k]`` with ``i, j, k`` in ``[0, n + 2*ng]``."""

    n: tuple
    ng: int
    dx: tuple
    xmin: tuple

    def __post_init__(self):
        self.n = tuple(int(v) for v in self.n)
        self.npts = tuple(v + 2 * self.ng + 1 for v in self.n)
        # rows start on 32-byte boundaries (4 doubles)
        self.sy = (self.npts[0] + 3) // 4 * 4
        self.sz = self.sy * self.npts[1]
        self.size = self.sz * self.npts[2]

    def box(self) -> Box:
        b = Box()
        b.n[:] = self.n
        b.ng = self.ng
        b.sy = self.sy
        b.sz = self.sz
        b.dx[:] = self.dx
        b.xmin[:] = self.xmin
        return b

    def view(self, flat):
        """3-D [k, j, i] view (padding columns included) of a flat array."""
        return flat.reshape(self.npts[2], self.npts[1], self.sy)

    def zeros(self):
        return np.zeros(self.size)

    def coords(self, centring):
        """Coordinates (x, y, z) broadcastable to view() shape, for a
        centring triple such as (1, 1, 1) = cell, (0, 0, 0) = vertex."""
        out = []
        for d in range(3):
            npt = (self.sy, self.npts[1], self.npts[2])[d]
            idx = np.arange(npt, dtype=np.float64)
            x = self.xmin[d] + (idx - self.ng + 0.5 * centring[d]) * self.dx[d]
            shape = [1, 1, 1]
            shape[2 - d] = npt
            out.append(x.reshape(shape))
        return out

    def interior(self, centring=(1, 1, 1), ext=0):
        """Slices (k, j, i) of the interior of a centring, widened by ext."""
        sl = []
        for d in (2, 1, 0):
            lo = self.ng - ext
            hi = self.ng + self.n[d] + (0 if centring[d] else 1) + ext
            sl.append(slice(lo, hi))
        return tuple(sl)
