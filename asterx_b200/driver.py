"""Multi-step evolution of one box on the engine, with the time integrators
and outer-boundary rules of the reference's driver, and the reference's
1-D shock-tube tests.

The reference's scheduled routines run inside CarpetX: ODESolvers advances
the evolved variables with an explicit Runge-Kutta method, calling the RHS
group for every stage and the post-step group (SYNC of the evolved
variables, then AsterX_Con2PrimGroup) after every stage update
(AsterX/schedule.ccl:107-165); every SYNC of a grid function at a physical
outer boundary applies the boundary rule (CarpetX's boundary_x ..
boundary_upper_z).  `Evolution` does the same on the device through the C
ABI: axb_rhs_group_bc, axb_rk_lincomb, axb_fill_boundary and
axb_con2prim_group.

Runge-Kutta methods (ODESolvers::method), stage k of s stages:
  rk2     midpoint rule: y1 = y0 + dt/2 k1;  y = y0 + dt k2
  ssprk3  Shu-Osher:     y1 = y0 + dt k1;  y2 = 3/4 y0 + 1/4 y1 + dt/4 k2;
                         y = 1/3 y0 + 2/3 y2 + 2/3 dt k3
  rk4     classical:     y1 = y0 + dt/2 k1;  y2 = y0 + dt/2 k2;  y3 = y0 + dt k3;
                         y = y0 + dt/6 (k1 + 2 k2 + 2 k3 + k4)

The 1-D tests (AsterX/test/Balsara*_shocktube_*.par, restated in
ONE_D_TESTS): AsterSeeds' Riemann problems (AsterSeeds/src/1D_tests.cxx:
165-481) on [-0.5, 0.5]^3 with 2 cells across the shock, dt = dtfac * the
smallest spacing, the stated boundary rule, RK4.  `one_d_initial` builds the
initial state as AsterSeeds and AsterX_InitialGroup leave it (primitives and
vector potential on every point, dB_stag and the cell field from curl A,
the primitive checks, prim -> con, boundary fills).
"""
from __future__ import annotations

import math
from typing import Dict, List, Sequence

import numpy as np

from . import abi
from .abi import Layout

EVOLVED = abi.CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]
RHS = abi.HYDRO_RHS + abi.AVEC_RHS
PRIMS = ["rho", "velx", "vely", "velz", "eps", "press", "temperature", "Ye", "entropy",
         "Bvecx", "Bvecy", "Bvecz"]
BC_NAMES = {"periodic": abi.BC_PERIODIC, "neumann": abi.BC_NEUMANN,
            "linear extrapolation": abi.BC_LINEAR}

# (left state, right state): rho, vel^i, press, B^i (AsterSeeds/src/1D_tests.cxx:191-280)
BALSARA = {
    "Balsara1": ((1.0, (0.0, 0.0, 0.0), 1.0, (0.5, 1.0, 0.0)),
                 (0.125, (0.0, 0.0, 0.0), 0.1, (0.5, -1.0, 0.0))),
    "Balsara2": ((1.0, (0.0, 0.0, 0.0), 30.0, (5.0, 6.0, 6.0)),
                 (1.0, (0.0, 0.0, 0.0), 1.0, (5.0, 0.7, 0.7))),
    "Balsara3": ((1.0, (0.0, 0.0, 0.0), 1000.0, (10.0, 7.0, 7.0)),
                 (1.0, (0.0, 0.0, 0.0), 0.1, (10.0, 0.7, 0.7))),
    "Balsara4": ((1.0, (0.999, 0.0, 0.0), 0.1, (10.0, 7.0, 7.0)),
                 (1.0, (-0.999, 0.0, 0.0), 0.1, (10.0, -7.0, -7.0))),
    "Balsara5": ((1.08, (0.4, 0.3, 0.2), 0.95, (2.0, 0.3, 0.3)),
                 (1.0, (-0.45, -0.2, 0.2), 1.0, (2.0, -0.7, 0.5))),
}


def _case(test, recon, flux="hlle", bc="neumann", shock_dir="x", n=50, ng=3, gamma=2.0,
          c2p=("noble", "palenzuela"), c2p_tol=1e-8, rho_abs_min=1e-8, eps_min=0.0,
          final_time=0.4):
    return dict(test=test, recon=recon, flux=flux, bc=bc, shock_dir=shock_dir, n=n, ng=ng,
                gamma=gamma, c2p=c2p, c2p_tol=c2p_tol, rho_abs_min=rho_abs_min,
                eps_min=eps_min, final_time=final_time, dtfac=0.25, method="rk4",
                out_every=10)


G53 = 1.66666666666667
# The reference's 1-D regression tests (AsterX/test/<name>.par).
ONE_D_TESTS = {
    "Balsara1_shocktube_xdir_ppm": _case("Balsara1", "ppm", bc="linear extrapolation"),
    "Balsara1_shocktube_xdir_wenoz": _case("Balsara1", "wenoz"),
    "Balsara1_shocktube_xdir_mp5": _case("Balsara1", "mp5"),
    "Balsara1_shocktube_xdir_godunov": _case("Balsara1", "godunov", ng=2),
    "Balsara1_shocktube_xdir_monocentral": _case("Balsara1", "monocentral", ng=2),
    "Balsara1_shocktube_xdir_ppm_PalenzuelaC2P": _case("Balsara1", "ppm",
                                                       c2p=("palenzuela", "none"),
                                                       c2p_tol=1e-14),
    "Balsara1_shocktube_ydir_ppm": _case("Balsara1", "ppm", shock_dir="y"),
    "Balsara1_shocktube_zdir_ppm": _case("Balsara1", "ppm", shock_dir="z"),
    "Balsara2_shocktube_xdir_ppm": _case("Balsara2", "ppm", gamma=G53),
    "Balsara3_shocktube_xdir_minmod_LxF": _case("Balsara3", "minmod", flux="lxf", n=80,
                                                ng=2, gamma=G53, rho_abs_min=1e-6,
                                                eps_min=1e-9),
    "Balsara4_shocktube_xdir_ppm": _case("Balsara4", "ppm", gamma=G53),
    "Balsara5_shocktube_xdir_ppm": _case("Balsara5", "ppm", gamma=G53, final_time=0.55),
}


def _rotations(shock_dir):
    """R and its inverse of AsterSeeds (1D_tests.cxx:285-351): rotation
    angles about x, y, z for the shock direction, R = R_x R_y R_z and
    Rinv = R_z(-tz) R_y(-ty) R_x(-tx)."""
    tx, ty, tz = {"x": (0.0, 0.0, 0.0), "y": (0.5 * math.pi, 0.0, 0.5 * math.pi),
                  "z": (0.0, -0.5 * math.pi, -0.5 * math.pi)}[shock_dir]

    def Rx(t):
        return np.array([[1.0, 0.0, 0.0], [0.0, math.cos(t), math.sin(t)],
                         [0.0, -math.sin(t), math.cos(t)]])

    def Ry(t):
        return np.array([[math.cos(t), 0.0, -math.sin(t)], [0.0, 1.0, 0.0],
                         [math.sin(t), 0.0, math.cos(t)]])

    def Rz(t):
        return np.array([[math.cos(t), math.sin(t), 0.0], [-math.sin(t), math.cos(t), 0.0],
                         [0.0, 0.0, 1.0]])

    return Rx(tx) @ Ry(ty) @ Rz(tz), Rz(-tz) @ Ry(-ty) @ Rx(-tx)


def one_d_layout(case, ng=None):
    """The box of a 1-D test: n cells along the shock, 2 across, on
    [-0.5, 0.5]^3."""
    c = ONE_D_TESTS[case] if isinstance(case, str) else case
    ax = "xyz".index(c["shock_dir"])
    n = [2, 2, 2]
    n[ax] = c["n"]
    return Layout(tuple(n), c["ng"] if ng is None else ng, tuple(1.0 / v for v in n),
                  (-0.5, -0.5, -0.5))


def params_for(case):
    c = ONE_D_TESTS[case] if isinstance(case, str) else case
    prime, second = c["c2p"]
    return abi.default_params(
        reconstruction_method=c["recon"], flux_type=c["flux"], c2p_prime=prime,
        c2p_second=second, c2p_tol=c["c2p_tol"], max_iter=100, rho_abs_min=c["rho_abs_min"],
        B_lim=1e8, vw_lim=1e8, Ye_lenient=1, poly_gamma=c["gamma"])


def eos_kw_for(case):
    """Ideal-gas EOS of the test (EOSX: gl_gamma, rho_max = eps_max = 1e8,
    eps_min)."""
    c = ONE_D_TESTS[case] if isinstance(case, str) else case
    return dict(gamma=c["gamma"], rho=(0.0, 1e8), eps=(c["eps_min"], 1e8), ye=(0.0, 1.0),
                poly_gamma=c["gamma"], poly_k=100.0)


def bc_for(case):
    c = ONE_D_TESTS[case] if isinstance(case, str) else case
    return (BC_NAMES[c["bc"]],) * 6


def dt_for(case, L):
    c = ONE_D_TESTS[case] if isinstance(case, str) else case
    return c["dtfac"] * min(L.dx)


def fill_boundary_np(L: Layout, f: Dict[str, np.ndarray], names: Sequence[str], bc):
    """Host form of axb_fill_boundary (same rules, same order: x, then y,
    then z, each over the full extent of the other two directions)."""
    for name in names:
        cent = CENTRING.get(name, (1, 1, 1))
        v = L.view(f[name])
        for d in range(3):
            ax = 2 - d  # view axes are (k, j, i)
            N = [L.n[e] + 2 * L.ng + (0 if cent[e] else 1) for e in range(3)]
            sl = [slice(0, N[2]), slice(0, N[1]), slice(0, N[0])]
            sub = v[tuple(sl)]
            lo_b = L.ng
            hi_b = L.ng + L.n[d] - (1 if cent[d] else 0)
            for side, typ in ((0, bc[2 * d]), (1, bc[2 * d + 1])):
                for q in range(L.ng):
                    gi = q if side == 0 else hi_b + 1 + q
                    bi = lo_b if side == 0 else hi_b
                    ii = bi + 1 if side == 0 else bi - 1

                    def at(i):
                        idx = [slice(None)] * 3
                        idx[ax] = i
                        return tuple(idx)
                    if typ == abi.BC_PERIODIC:
                        src = L.ng + (gi - L.ng) % L.n[d]
                        sub[at(gi)] = sub[at(src)]
                    elif typ == abi.BC_NEUMANN:
                        sub[at(gi)] = sub[at(bi)]
                    else:
                        k = abs(gi - bi)
                        sub[at(gi)] = sub[at(bi)] + k * (sub[at(bi)] - sub[at(ii)])


CENTRING = {"Avec_x": (1, 0, 0), "Avec_y": (0, 1, 0), "Avec_z": (0, 0, 1), "Psi": (0, 0, 0),
            "Avec_x_rhs": (1, 0, 0), "Avec_y_rhs": (0, 1, 0), "Avec_z_rhs": (0, 0, 1),
            "Psi_rhs": (0, 0, 0), "dBx_stag": (0, 1, 1), "dBy_stag": (1, 0, 1),
            "dBz_stag": (1, 1, 0), "Fx": (0, 0, 0), "Fy": (0, 0, 0), "Fz": (0, 0, 0),
            "Fbetax": (0, 0, 0), "Fbetay": (0, 0, 0), "Fbetaz": (0, 0, 0), "G": (0, 0, 0),
            "fxBy": (0, 1, 1), "fxBz": (0, 1, 1), "fyBx": (1, 0, 1), "fyBz": (1, 0, 1),
            "fzBx": (1, 1, 0), "fzBy": (1, 1, 0)}
for _g in ("gxx", "gxy", "gxz", "gyy", "gyz", "gzz", "alp", "betax", "betay", "betaz",
           "kxx", "kxy", "kxz", "kyy", "kyz", "kzz"):
    CENTRING[_g] = (0, 0, 0)
CENTRING.update(abi.UCT_CENT)


def one_d_initial(case, ng=None, ye=0.5):
    """Initial state of a 1-D test on the host: AsterSeeds' primitives on
    every cell and vector potential on every edge (the rot_off branch of
    1D_tests.cxx:392-427: A_x = B_y z, A_y = B_z x, A_z = B_x y with the
    side's rotated B), Psi = 0, flat metric; then AsterX_InitialGroup
    (AsterX/schedule.ccl:44-104): dB_stag = curl A on the interior faces,
    dB and B on the interior cells, the primitive checks (entropy = kappa,
    saved primitives, zvec / svec) and prim -> con on the interior, each
    followed by its SYNC's boundary fill.  Ye (which the test leaves to
    HydroBaseX's initial value) is `ye`; the ideal gas ignores it except
    for the Ye > 0 test of the low-order fallback."""
    from . import workloads as W
    c = ONE_D_TESTS[case] if isinstance(case, str) else case
    L = one_d_layout(c, ng)
    gamma = c["gamma"]
    bc = bc_for(c)
    (rl, vl, pl, Bl), (rr, vr, pr, Br) = BALSARA[c["test"]]
    R, Rinv = _rotations(c["shock_dir"])
    oBl, oBr = Rinv @ np.array(Bl), Rinv @ np.array(Br)
    ovl, ovr = Rinv @ np.array(vl), Rinv @ np.array(vr)
    f: Dict[str, np.ndarray] = {}
    W.flat_metric(L, f)
    shape = L.view(L.zeros()).shape

    def side_left(cent):
        x, y, z = L.coords(cent)
        X, Y, Z = (np.broadcast_to(a, shape) for a in (x, y, z))
        newx = R[0, 0] * X + R[0, 1] * Y + R[0, 2] * Z
        return newx <= 0.0, X, Y, Z

    left, _, _, _ = side_left((1, 1, 1))
    f["rho"] = np.where(left, rl, rr).ravel().copy()
    for q, nm in enumerate(("velx", "vely", "velz")):
        f[nm] = np.where(left, ovl[q], ovr[q]).ravel().copy()
    f["press"] = np.where(left, pl, pr).ravel().copy()
    f["eps"] = f["press"] / ((gamma - 1.0) * f["rho"])
    f["Ye"] = np.full(L.size, ye)
    # vector potential on every edge (rot_off branch)
    for name, cent, expr in (("Avec_x", (1, 0, 0), lambda B, X, Y, Z: B[1] * Z),
                             ("Avec_y", (0, 1, 0), lambda B, X, Y, Z: B[2] * X),
                             ("Avec_z", (0, 0, 1), lambda B, X, Y, Z: B[0] * Y)):
        lft, X, Y, Z = side_left(cent)
        f[name] = np.where(lft, expr(oBl, X, Y, Z), expr(oBr, X, Y, Z)).ravel().copy()
    f["Psi"] = L.zeros()
    # AsterX_InitialGroup
    f["dBx_stag"], f["dBy_stag"], f["dBz_stag"] = W._curl_stag(L, f["Avec_x"], f["Avec_y"],
                                                               f["Avec_z"])
    fill_boundary_np(L, f, ["dBx_stag", "dBy_stag", "dBz_stag"], bc)
    W._cell_B_from_stag(L, f)
    fill_boundary_np(L, f, ["dBx", "dBy", "dBz", "Bvecx", "Bvecy", "Bvecz"], bc)
    # AsterX_CheckPrims on the interior: no floor or ceiling acts on these
    # states; entropy = kappa(rho, eps), temperature = (Gamma - 1) eps
    f["entropy"] = (gamma - 1.0) * f["eps"] * f["rho"] ** (1.0 - gamma)
    f["temperature"] = (gamma - 1.0) * f["eps"]
    W.saved_from_prims(f)
    W.cons_from_prims(L, f)
    fill_boundary_np(L, f, PRIMS + abi.SAVED + abi.CONS +
                     ["zvec_x", "zvec_y", "zvec_z", "svec_x", "svec_y", "svec_z"], bc)
    for n in abi.GF_NAMES:
        f.setdefault(n, L.zeros())
    return L, f


# The reference's 2-D regression tests (AsterX/test/<name>.par): AsterSeeds'
# 2DTest cases (AsterSeeds/src/2D_tests.cxx:33-190) on a box two cells thick
# in z, Neumann boundaries, RK4, dt = dtfac * the smallest spacing, and the
# settings the hot path reads (the rest are the param.ccl defaults).
TWO_D_TESTS = {
    "Magnetic_rotor": dict(
        test="magnetic rotor", recon="ppm", flux="hlle", n=(40, 40, 2), ng=3,
        xmin=(-0.5, -0.5, -0.004), xmax=(0.5, 0.5, 0.004), bc="neumann",
        gamma=1.66666666666667, c2p=("noble", "palenzuela"), c2p_tol=1e-8, max_iter=30,
        rho_abs_min=1e-13, eps_min=1e-6, B_lim=100.0, vw_lim=10.0, Ye_lenient=0,
        use_uct=0, recon_type=0, use_entropy_fix=0, dtfac=0.35, final_time=0.1,
        method="rk4", out_every=20),
    "Cylindrical_blast": dict(
        test="cylindrical blast", recon="minmod", flux="hlle", n=(50, 50, 2), ng=2,
        xmin=(-6.0, -6.0, -0.06), xmax=(6.0, 6.0, 0.06), bc="neumann",
        gamma=1.3333333333, c2p=("noble", "palenzuela"), c2p_tol=1e-8, max_iter=1000,
        rho_abs_min=1e-6, eps_min=1e-7, B_lim=1e8, vw_lim=1e8, Ye_lenient=1,
        use_uct=1, recon_type=1, use_entropy_fix=1, dtfac=0.35, final_time=2.0,
        method="rk4", out_every=20),
}


def two_d_layout(case, ng=None):
    c = TWO_D_TESTS[case]
    dx = tuple((hi - lo) / n for lo, hi, n in zip(c["xmin"], c["xmax"], c["n"]))
    return Layout(tuple(c["n"]), c["ng"] if ng is None else ng, dx, tuple(c["xmin"]))


def two_d_params(case):
    c = TWO_D_TESTS[case]
    prime, second = c["c2p"]
    return abi.default_params(
        reconstruction_method=c["recon"], flux_type=c["flux"], c2p_prime=prime,
        c2p_second=second, c2p_tol=c["c2p_tol"], max_iter=c["max_iter"],
        rho_abs_min=c["rho_abs_min"], B_lim=c["B_lim"], vw_lim=c["vw_lim"],
        Ye_lenient=c["Ye_lenient"], poly_gamma=c["gamma"], use_uct=c["use_uct"],
        recon_type=c["recon_type"], use_entropy_fix=c["use_entropy_fix"])


def two_d_eos_kw(case):
    c = TWO_D_TESTS[case]
    return dict(gamma=c["gamma"], rho=(0.0, 1e8), eps=(c["eps_min"], 1e8), ye=(0.0, 1.0),
                poly_gamma=c["gamma"], poly_k=100.0)


def two_d_initial(case, ng=None, ye=0.5):
    """Initial state of a 2-D test on the host: AsterSeeds' primitives on
    every cell and vector potential on every edge (2D_tests.cxx:33-73 and
    135-190: A_x = A_y = 0, A_z = a y with a = 1 for the rotor and 0.1 for
    the blast), flat metric, then AsterX_InitialGroup as in one_d_initial."""
    from . import workloads as W
    c = TWO_D_TESTS[case]
    L = two_d_layout(case, ng)
    gamma = c["gamma"]
    bc = (BC_NAMES[c["bc"]],) * 6
    f: Dict[str, np.ndarray] = {}
    W.flat_metric(L, f)
    shape = L.view(L.zeros()).shape
    x, y, _ = (np.broadcast_to(a, shape) for a in L.coords((1, 1, 1)))
    r = np.sqrt(x * x + y * y)
    zero = np.zeros(shape)
    if c["test"] == "magnetic rotor":
        inside = r < 0.1
        omega = 9.95
        rho = np.where(inside, 10.0, 1.0)
        vx = np.where(inside, -omega * y, 0.0)
        vy = np.where(inside, omega * x, 0.0)
        press = np.ones(shape)
        a_z = 1.0
    else:
        r_in, r_out, rho_in, rho_out, p_in, p_out = 0.8, 1.0, 1e-2, 1e-4, 1.0, 3.0e-5
        with np.errstate(divide="ignore", invalid="ignore"):
            rho_mid = np.exp(((r_out - r) * math.log(rho_in) + (r - r_in) * math.log(rho_out))
                             / (r_out - r_in))
            p_mid = np.exp(((r_out - r) * math.log(p_in) + (r - r_in) * math.log(p_out))
                           / (r_out - r_in))
        rho = np.where(r < r_in, rho_in, np.where(r > r_out, rho_out, rho_mid))
        press = np.where(r < r_in, p_in, np.where(r > r_out, p_out, p_mid))
        vx = vy = zero
        a_z = 0.1
    f["rho"] = rho.ravel().copy()
    f["velx"] = np.asarray(vx).ravel().copy()
    f["vely"] = np.asarray(vy).ravel().copy()
    f["velz"] = zero.ravel().copy()
    f["press"] = press.ravel().copy()
    f["eps"] = f["press"] / ((gamma - 1.0) * f["rho"])
    f["Ye"] = np.full(L.size, ye)
    f["Avec_x"] = L.zeros()
    f["Avec_y"] = L.zeros()
    _, ye_z, _ = (np.broadcast_to(a, shape) for a in L.coords((0, 0, 1)))
    f["Avec_z"] = (a_z * ye_z).ravel().copy()
    f["Psi"] = L.zeros()
    f["dBx_stag"], f["dBy_stag"], f["dBz_stag"] = W._curl_stag(L, f["Avec_x"], f["Avec_y"],
                                                               f["Avec_z"])
    fill_boundary_np(L, f, ["dBx_stag", "dBy_stag", "dBz_stag"], bc)
    W._cell_B_from_stag(L, f)
    fill_boundary_np(L, f, ["dBx", "dBy", "dBz", "Bvecx", "Bvecy", "Bvecz"], bc)
    f["entropy"] = (gamma - 1.0) * f["eps"] * f["rho"] ** (1.0 - gamma)
    f["temperature"] = (gamma - 1.0) * f["eps"]
    W.saved_from_prims(f)
    W.cons_from_prims(L, f)
    fill_boundary_np(L, f, PRIMS + abi.SAVED + abi.CONS +
                     ["zvec_x", "zvec_y", "zvec_z", "svec_x", "svec_y", "svec_z"], bc)
    for n in abi.GF_NAMES:
        f.setdefault(n, L.zeros())
    return L, f


def cut_at(L: Layout, f, name, axis, fixed):
    """Values of `name` along `axis` (ghosts included) through the point whose
    other two interior indices are `fixed` (the reference's TSV output)."""
    v = L.view(f[name])
    ax = "xyz".index(axis)
    others = [d for d in range(3) if d != ax]
    idx = [0, 0, 0]
    for d, q in zip(others, fixed):
        idx[d] = L.ng + int(q)
    idx[ax] = slice(0, L.n[ax] + 2 * L.ng)
    return np.asarray(v[idx[2], idx[1], idx[0]])


# Runge-Kutta methods: per stage, the combination that forms the next state
# from the initial state y0, the stored stage RHS k1 .. k(s-1) and this
# stage's RHS: (coefficients of [y0, y_current], coefficients of the stored
# stages, coefficient of this stage's RHS), all in units of dt for RHS terms.
RK_METHODS = {
    "rk2": [((1.0, 0.0), (), 0.5), ((1.0, 0.0), (), 1.0)],
    "ssprk3": [((1.0, 0.0), (), 1.0), ((0.75, 0.25), (), 0.25),
               ((1.0 / 3.0, 2.0 / 3.0), (), 2.0 / 3.0)],
    "rk4": [((1.0, 0.0), (), 0.5), ((1.0, 0.0), (), 0.5), ((1.0, 0.0), (), 1.0),
            ((1.0, 0.0), (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0), 1.0 / 6.0)],
}


class Evolution:
    """Multi-step evolution of one box on the engine: for every stage the
    RHS group with the outer-boundary rules, the stage combination, the
    boundary fill of the evolved variables, the post-step group and the
    boundary fill of the primitives (and of the face and cell fields the
    reference SYNCs there), as ODESolvers and AsterX's schedule order them."""

    def __init__(self, eng, L: Layout, fields, params, eos, method="rk4", bc=None):
        self.eng, self.L, self.f, self.p, self.eos = eng, L, fields, params, eos
        self.method = RK_METHODS[method]
        self.bc = bc if bc is not None else (abi.BC_PERIODIC,) * 6
        t = eng.torch
        mk = lambda: {n: t.empty_like(fields[n]) for n in EVOLVED}
        self.y0 = mk()
        nstore = max(len(s[1]) for s in self.method)
        # stored stage RHS under the evolved variables' names (the combination
        # reads states by those names)
        self.k = [{n: t.empty_like(fields[n]) for n in EVOLVED} for _ in range(nstore)]
        self.rhs = {r: fields[r] for r in RHS}
        self.post = PRIMS + [{1: "zvec_", 2: "svec_"}.get(int(params.recon_type), "")
                             + a for a in "xyz" if int(params.recon_type) in (1, 2)]
        self.iteration = 0

    def step(self, dt):
        eng, L, f = self.eng, self.L, self.f
        for n in EVOLVED:
            self.y0[n].copy_(f[n])
        for s, (yc, kc, rc) in enumerate(self.method):
            eng.rhs_group_bc(L, f, self.p, self.eos, self.bc)
            states, coef = [self.y0], [yc[0]]
            if yc[1]:
                states.append({n: f[n] for n in EVOLVED})
                coef.append(yc[1])
            for q, c in enumerate(kc):
                states.append(self.k[q])
                coef.append(c * dt)
            if s < len(self.k):
                for n, r in zip(EVOLVED, RHS):
                    self.k[s][n].copy_(f[r])
            eng.rk_lincomb(L, {n: f[n] for n in EVOLVED}, states, coef, rc * dt, self.rhs)
            eng.fill_boundary(L, f, EVOLVED, self.bc)
            eng.con2prim_group(L, f, self.p, self.eos)
            eng.fill_boundary(L, f, self.post + ["dBx_stag", "dBy_stag", "dBz_stag"] +
                              abi.CONS + abi.SAVED, self.bc)
        self.iteration += 1


def cut(L: Layout, f, name, axis="x"):
    """Values of `name` on the line through the first interior cell across
    the shock, ghosts included (the reference's TSV 1-D output)."""
    v = L.view(f[name])
    ax = "xyz".index(axis)
    n = L.n[ax] + 2 * L.ng
    sl = [L.ng, L.ng, L.ng]
    sl[ax] = slice(0, n)
    return np.asarray(v[sl[2], sl[1], sl[0]])
