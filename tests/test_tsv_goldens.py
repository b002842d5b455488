"""The reference's own regression goldens: the 1-D shock tubes of AsterX/test
(Balsara 1-5; PPM, WENO-Z, MP5, Godunov, monocentral, minmod; HLLE and LxF;
Noble with Palenzuela backup and Palenzuela alone; x, y and z shock
directions; Neumann and linear-extrapolation boundaries; RK4), compared as
AsterX/test/test.ccl compares them: every value of rho, vel, eps, press and
Bvec on the output cut, ghosts included, at every output iteration, within
1e-8 absolute or 1e-8 relative.  Fixtures: tests/golden/tsv_<case>.npz
(made by tests/golden/make_tsv_golden.py from the reference's TSV files).

* test_reference_build_reproduces_goldens (CPU): the reference's own
  routines (oracle/_ref) driven with the driver semantics of
  asterx_b200/driver.py -- this pins the checker and those semantics
  (RK4, boundary fills, initial data) to the reference's published results.
* test_engine_reproduces_goldens (GPU): the same evolutions on the engine
  through the C ABI (driver.Evolution: axb_rhs_group_bc, axb_rk_lincomb,
  axb_fill_boundary, axb_con2prim_group).
"""
import os

import numpy as np
import pytest

from asterx_b200 import driver as D

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = sorted(D.ONE_D_TESTS)
FIELDS = ["rho", "velx", "vely", "velz", "eps", "press", "Bvecx", "Bvecy", "Bvecz"]
TOL = 1e-8


def golden(case):
    return np.load(os.path.join(HERE, "golden", f"tsv_{case}.npz"))


def check_against(case, cuts, ng_run):
    """cuts: {iteration: {name: values on [-ng_run, n + ng_run)}}; the
    golden's points are [-ng, n + ng) of the test's own ghost count."""
    g = golden(case)
    idx = g["index"]
    checked = 0
    worst = 0.0
    for q, it in enumerate(g["iterations"]):
        it = int(it)
        assert it in cuts, f"{case}: no output at iteration {it}"
        for n in FIELDS:
            want = g[n][q]
            got = cuts[it][n][idx + ng_run]
            d = np.abs(got - want)
            bad = (d > TOL) & (d > TOL * np.abs(want))
            assert not bad.any(), (case, it, n, int(np.argmax(d)), float(d.max()))
            worst = max(worst, float(d.max()))
            checked += d.size
    return checked, worst


@pytest.mark.parametrize("case", CASES)
def test_reference_build_reproduces_goldens(ref, case):
    from tests.tsv_reference import run_reference
    c = D.ONE_D_TESTS[case]
    cuts = run_reference(ref, case)
    check_against(case, cuts, c["ng"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_engine_reproduces_goldens(engine, case):
    c = D.ONE_D_TESTS[case]
    ng = max(3, c["ng"])  # the engine's stencils need 3 ghost layers
    L, f = D.one_d_initial(case, ng=ng)
    p = D.params_for(case)
    eos = engine.eos_idealgas(**D.eos_kw_for(case))
    dev = engine.upload(L, f)
    ev = D.Evolution(engine, L, dev, p, eos, method=c["method"], bc=D.bc_for(case))
    dt = D.dt_for(case, L)
    nit = int(round(c["final_time"] / dt))
    axis = c["shock_dir"]
    cuts = {}

    def snap(it):
        host = {n: dev[n].cpu().numpy() for n in D.PRIMS}
        cuts[it] = {n: D.cut(L, host, n, axis) for n in D.PRIMS}

    snap(0)
    for it in range(1, nit + 1):
        ev.step(dt)
        if it % c["out_every"] == 0:
            snap(it)
    checked, worst = check_against(case, cuts, ng)
    print(f"{case}: {checked} values within 1e-8, largest difference {worst:.2e}")


# ---------------------------------------------------------------------------
# 2-D tests: the magnetic rotor (PPM, flux CT) and the cylindrical blast
# (minmod, upwind CT, z_vec reconstruction, entropy backup), compared on
# their x and y cuts
# ---------------------------------------------------------------------------
CASES_2D = sorted(D.TWO_D_TESTS)


def check_against_2d(case, cuts, ng_run):
    g = golden(case)
    checked = 0
    worst = 0.0
    for q, it in enumerate(g["iterations"]):
        it = int(it)
        assert it in cuts, f"{case}: no output at iteration {it}"
        for ax in ("x", "y"):
            idx = g[ax + "_index"]
            for n in FIELDS:
                want = g[ax + "_" + n][q]
                got = cuts[it][ax][n][idx + ng_run]
                d = np.abs(got - want)
                bad = (d > TOL) & (d > TOL * np.abs(want))
                assert not bad.any(), (case, it, ax, n, int(np.argmax(d)), float(d.max()))
                worst = max(worst, float(d.max()))
                checked += d.size
    return checked, worst


def fixed_points(case):
    g = golden(case)
    return {ax: tuple(int(v) for v in g[ax + "_fixed"]) for ax in ("x", "y")}


@pytest.mark.parametrize("case", CASES_2D)
def test_reference_build_reproduces_goldens_2d(ref, case):
    from tests.tsv_reference import run_reference_2d
    c = D.TWO_D_TESTS[case]
    ng = max(3, c["ng"])
    cuts = run_reference_2d(ref, case, fixed_points(case), ng=ng)
    checked, worst = check_against_2d(case, cuts, ng)
    print(f"{case}: {checked} values within 1e-8, largest difference {worst:.2e}")


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES_2D)
def test_engine_reproduces_goldens_2d(engine, case):
    c = D.TWO_D_TESTS[case]
    ng = max(3, c["ng"])  # the engine's stencils need 3 ghost layers
    L, f = D.two_d_initial(case, ng=ng)
    p = D.two_d_params(case)
    eos = engine.eos_idealgas(**D.two_d_eos_kw(case))
    dev = engine.upload(L, f)
    bc = (D.BC_NAMES[c["bc"]],) * 6
    ev = D.Evolution(engine, L, dev, p, eos, method=c["method"], bc=bc)
    dt = c["dtfac"] * min(L.dx)
    nit = int(c["final_time"] / dt + 1e-9)
    fixed = fixed_points(case)
    cuts = {}

    def snap(it):
        host = {n: dev[n].cpu().numpy() for n in D.PRIMS}
        cuts[it] = {ax: {n: D.cut_at(L, host, n, ax, fixed[ax]) for n in D.PRIMS}
                    for ax in ("x", "y")}

    snap(0)
    for it in range(1, nit + 1):
        ev.step(dt)
        if it % c["out_every"] == 0:
            snap(it)
    checked, worst = check_against_2d(case, cuts, ng)
    print(f"{case}: {checked} values within 1e-8, largest difference {worst:.2e}")
