"""The per-point entry points of include/asterx_b200_point.hxx (the
reference's per-point signatures over the engine's device functions),
compiled by nvcc as host code, against the reference's own functors
compiled from the reference sources (oracle/_ref):

  reconstruct   ReconX::reconstruct       ReconX/src/reconstruct.hxx:36-42
  eigenvalues   AsterX::eigenvalues       AsterX/src/eigenvalues.hxx:19-24
  hlle, laxf    AsterX::hlle, laxf        AsterX/src/fluxes.hxx:20-49
  prim2con      AsterX::prim2con          AsterX/src/prim2con.hxx:38-83
  c2p_2DNoble::solve, c2p_1DPalenzuela::solve
                Con2PrimFactory/src/c2p_2DNoble.hxx:275-279,
                c2p_1DPalenzuela.hxx:306-309

Tolerances: the engine's arithmetic keeps the reference's operation order
except where it replaces a division by a reciprocal product or 1/sqrt by
rsqrt, which moves the last few ulps: 1e-13 relative (with an absolute
floor scaled to the inputs) for the pointwise functions; for the recovery
the same status and Noble iteration count and primitives within 1e-10
relative, as the GPU parity tests use.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from asterx_b200 import abi
from asterx_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SRC = os.path.join(HERE, "point_api_host.cu")
OUT = os.path.join(HERE, "_build", "libpoint_api.so")
_dp = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _deps():
    inc = [os.path.join(REPO, "include", "asterx_b200_point.hxx"),
           os.path.join(REPO, "include", "asterx_b200.h")]
    csrc = os.path.join(REPO, "asterx_b200", "csrc")
    inc += [os.path.join(csrc, f) for f in os.listdir(csrc) if f.endswith(".cuh")]
    return [SRC] + inc


@pytest.fixture(scope="module")
def pt():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    stale = (not os.path.exists(OUT) or
             any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in _deps()))
    if stale:
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-O2", "-shared",
                        "-gencode", "arch=compute_100a,code=sm_100a",
                        "-Xcompiler", "-fPIC,-ffp-contract=off", SRC, "-o", OUT],
                       check=True)
    L = C.CDLL(OUT)
    L.pt_reconstruct.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_int, _dp, _dp]
    L.pt_eigen.argtypes = [_dp, _dp]
    L.pt_riemann.argtypes = [C.c_int, _dp] + [C.c_double] * 4
    L.pt_riemann.restype = C.c_double
    L.pt_prim2con.argtypes = [_dp, _dp, _dp]
    L.pt_c2p.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_int)]
    return L


def close(a, b, rtol, floor):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= rtol * np.maximum(np.abs(b), floor))


def recon_params(p):
    return np.array([p.ppm_shock_detection, p.ppm_zone_flattening, p.poly_k, p.poly_gamma,
                     p.ppm_eta1, p.ppm_eta2, p.ppm_eps, p.ppm_eps_shock, p.ppm_small,
                     p.ppm_omega1, p.ppm_omega2, p.weno_eps, p.mp5_alpha], dtype=np.float64)


@pytest.mark.parametrize("flattening", [0, 1])
def test_reconstruct(ref, pt, flattening):
    rng = np.random.default_rng(21)
    p = abi.default_params(ppm_zone_flattening=flattening)
    ref.setup(W.Layout((4, 4, 4), 3, (1, 1, 1), (0, 0, 0)), p, {})
    rp = recon_params(p)
    exact = 0
    total = 0
    for trial in range(300):
        v = rng.normal(size=6) * 10 ** rng.uniform(-3, 1)
        if trial % 5 == 0:
            v = np.cumsum(np.abs(v))  # monotone stencils
        if trial % 7 == 0:
            v[3:] *= 5.0  # a jump
        pr = np.abs(rng.normal(size=6)) + 0.1
        vel = rng.uniform(-0.9, 0.9, 6)
        for m in (0, 1, 2, 3, 5, 6):
            for is_rho in (False, True):
                want = ref.reconstruct(m, v, pr, vel, is_rho)
                got = np.zeros(2)
                pt.pt_reconstruct(m, _ptr(v), _ptr(pr), _ptr(vel), int(is_rho), 0,
                                  _ptr(rp), _ptr(got))
                scale = np.abs(v).max()
                assert close(got, want, 1e-13, scale), (m, is_rho, v, got, want)
                exact += int(np.array_equal(got, want))
                total += 1
    # most faces agree to the bit; WENO-Z's one division moves a few ulps
    assert exact > 0.5 * total


def test_eigenvalues_and_riemann(ref, pt):
    rng = np.random.default_rng(22)
    for _ in range(300):
        alp, beta, u = rng.uniform(0.8, 1.2), rng.uniform(-0.1, 0.1), rng.uniform(0.8, 1.2)
        pairs = [rng.uniform(-0.9, 0.9, 2), rng.uniform(0.1, 1, 2), rng.uniform(0, 0.3, 2),
                 rng.uniform(1, 3, 2), rng.uniform(1, 2, 2), rng.uniform(0, 1, 2)]
        want = ref.eigen(alp, beta, u, *pairs)
        inp = np.array([alp, beta, u, *np.concatenate(pairs)], dtype=np.float64)
        got = np.zeros(8)
        pt.pt_eigen(_ptr(inp), _ptr(got))
        assert close(got, want, 1e-13, 1e-12), (got, want)
        uL, uR, fL, fR = rng.normal(size=4)
        for ft in (abi.FLUX["lxf"], abi.FLUX["hlle"]):
            w = ref.riemann(ft, want, uL, uR, fL, fR)
            g = pt.pt_riemann(ft, _ptr(want), uL, uR, fL, fR)
            assert close(g, w, 1e-13, max(abs(uL), abs(uR), abs(fL), abs(fR))), (ft, g, w)


def test_prim2con(ref, pt):
    rng = np.random.default_rng(23)
    for _ in range(300):
        g6 = np.array([1, 0, 0, 1, 0, 1.0]) + 0.05 * rng.uniform(-1, 1, 6)
        prim = np.concatenate([[10 ** rng.uniform(-6, 0)], rng.uniform(-0.4, 0.4, 3),
                               [10 ** rng.uniform(-3, 1)], [rng.uniform(0.01, 1)],
                               [rng.uniform(0, 1)], [rng.uniform(0.05, 0.5)],
                               rng.normal(size=3)])
        want = ref.prim2con(g6, prim)
        got = np.zeros(10)
        pt.pt_prim2con(_ptr(g6), _ptr(prim), _ptr(got))
        assert close(got, want, 1e-14, 1e-300), (got, want)


@pytest.mark.parametrize("solver", ["noble", "palenzuela"])
def test_c2p_solve(ref, pt, solver):
    gamma = 5.0 / 3.0
    n = 400
    cells = W.c2p_cells(n, seed=24, gamma=gamma, w_range=(1.0, 20.0))
    tol = 1e-12 if solver == "noble" else 1e-14
    p = abi.default_params(c2p_prime=solver, c2p_second="none", c2p_tol=tol, max_iter=100,
                           vw_lim=60.0, B_lim=1e8, rho_abs_min=1e-20)
    eos_kw = dict(rho=(1e-40, 1e10), eps=(0.0, 1e10), ye=(0.0, 1.0))
    ref.setup(W.Layout((4, 4, 4), 3, (1, 1, 1), (0, 0, 0)), p, {})
    ref.eos_idealgas(gamma, **eos_kw)
    eos8 = np.array([gamma, 1.0, *eos_kw["eps"], *eos_kw["rho"], *eos_kw["ye"]])
    c2p14 = np.array([p.max_iter, p.c2p_tol, p.alp_thresh, p.cons_error_limit, p.vw_lim,
                      p.B_lim, p.rho_BH, p.eps_BH, p.vwlim_BH, p.Ye_lenient, p.use_z,
                      p.use_temperature, p.use_press_atmo, 0.0])
    rho_atm = 1e-20
    eps_atm = p.t_atmo / (gamma - 1.0)
    atmo = np.array([rho_atm, eps_atm, p.Ye_atmo, (gamma - 1.0) * rho_atm * eps_atm, p.t_atmo,
                     (gamma - 1.0) * eps_atm * rho_atm ** (1.0 - gamma),
                     rho_atm * (1 + p.atmo_tol)])
    code = abi.C2P[solver]
    ok = 0
    for i in range(n):
        cons = np.array([cells[k][i] for k in ("dens", "momx", "momy", "momz", "tau", "DYe",
                                               "DEnt", "dBx", "dBy", "dBz")])
        g6 = np.array([cells[k][i] for k in ("gxx", "gxy", "gxz", "gyy", "gyz", "gzz")])
        sq = np.sqrt(np.linalg.det(np.array([[g6[0], g6[1], g6[2]], [g6[1], g6[3], g6[4]],
                                             [g6[2], g6[4], g6[5]]])))
        seed = np.array([cons[0] / sq, eps_atm, cons[5] / cons[0], 0.0, p.t_atmo, 0.0, 0.0,
                         0.0, 0.0])
        wprim, wcons, wrep = ref.c2p_point(code, cons, g6, seed, atmo)
        gcons = cons.copy()
        gprim = np.zeros(16)
        grep = (C.c_int * 3)()
        pt.pt_c2p(code, _ptr(gcons), _ptr(g6), _ptr(seed), _ptr(atmo), _ptr(eos8),
                  _ptr(c2p14), _ptr(gprim), grep)
        assert grep[0] == wrep[0], (i, tuple(grep), wrep)
        if solver == "noble":
            assert grep[1] == wrep[1], (i, tuple(grep), wrep)
        if wrep[0] == 0:
            ok += 1
            for j in (0, 1, 3, 6, 7, 8, 9):  # rho eps press vel W
                # 1e-10 relative, 1e-14 absolute for components near zero
                assert close(gprim[j], wprim[j], 1e-10, 1e-4), (i, j, gprim[j], wprim[j])
    assert ok > 0.9 * n
