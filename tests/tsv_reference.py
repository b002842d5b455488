"""The reference's own routines (oracle/_ref, compiled from the reference
sources) driven through a 1-D test of AsterX/test with the driver semantics
of asterx_b200/driver.py: the RHS group on the interior with the SYNC'd face
fluxes and vertex auxiliaries filled by the boundary rule, the Runge-Kutta
stage combination, the boundary fills after every stage, the post-step group.
Test infrastructure: the CPU counterpart of driver.Evolution, used to pin
the driver semantics against the reference's TSV goldens without a GPU."""
import numpy as np

from asterx_b200 import abi
from asterx_b200 import driver as D

FACE_FLUX = [f"f{d}{v}" for d in "xyz" for v in
             ("dens", "momx", "momy", "momz", "tau", "DYe", "DEnt", "Bx", "By", "Bz")]
FLUX_CENT = {f"f{d}{v}": {"x": (0, 1, 1), "y": (1, 0, 1), "z": (1, 1, 0)}[d]
             for d in "xyz" for v in ("dens", "momx", "momy", "momz", "tau", "DYe", "DEnt",
                                      "Bx", "By", "Bz")}
AUX = ["Fx", "Fy", "Fz", "Fbetax", "Fbetay", "Fbetaz", "G"]


def evolve_reference(ref, L, f, p, bc, eos_kw, dt, nit, method, snaps, snap):
    """Evolve the host state `f` with the reference build for `nit` steps of
    `dt`; snap(it, host) at the iterations in `snaps`."""
    D.CENTRING.update(FLUX_CENT)
    host = {k: v.copy() for k, v in f.items()}
    ref.setup(L, p, host)
    ref.eos_idealgas(**eos_kw)
    method = D.RK_METHODS[method]
    faces = FACE_FLUX + AUX + (abi.UCT if p.use_uct else [])
    if 0 in snaps:
        snap(0, host)
    for it in range(1, nit + 1):
        y0 = {n: host[n].copy() for n in D.EVOLVED}
        ks = []
        for s, (yc, kc, rc) in enumerate(method):
            ref.run("fluxes")
            D.fill_boundary_np(L, ref.fields, faces, bc)
            ref.run("sources")
            ref.run("rhs")
            k = {n: host[r].copy() for n, r in zip(D.EVOLVED, D.RHS)}
            for n in D.EVOLVED:
                sl = L.interior(D.CENTRING.get(n, (1, 1, 1)))
                v = L.view(host[n])
                acc = yc[0] * L.view(y0[n])[sl]
                if yc[1]:
                    acc = acc + yc[1] * v[sl]
                for q, cq in enumerate(kc):
                    acc = acc + (cq * dt) * L.view(ks[q][n])[sl]
                v[sl] = acc + (rc * dt) * L.view(k[n])[sl]
            ks.append(k)
            D.fill_boundary_np(L, host, D.EVOLVED, bc)
            ref.run("bstag")
            D.fill_boundary_np(L, host, ["dBx_stag", "dBy_stag", "dBz_stag"], bc)
            ref.run("dB")
            ref.run("c2p")
            D.fill_boundary_np(L, host, D.PRIMS + ["dBx", "dBy", "dBz"] + abi.CONS +
                               abi.SAVED + ["zvec_x", "zvec_y", "zvec_z"], bc)
        if it in snaps:
            snap(it, host)


def run_reference(ref, case, snapshots=None, ng=None):
    """Evolve `case` with the reference build; returns {iteration: {name:
    cut}} at the iterations in `snapshots` (default every out_every)."""
    c = D.ONE_D_TESTS[case]
    L, f = D.one_d_initial(case, ng=ng)
    dt = D.dt_for(case, L)
    nit = int(round(c["final_time"] / dt))
    snaps = snapshots if snapshots is not None else list(range(0, nit + 1, c["out_every"]))
    out = {}

    def snap(it, host):
        out[it] = {n: D.cut(L, host, n, c["shock_dir"]).copy() for n in D.PRIMS}

    evolve_reference(ref, L, f, D.params_for(case), D.bc_for(case), D.eos_kw_for(case), dt,
                     nit, c["method"], snaps, snap)
    return out


def run_reference_2d(ref, case, fixed, ng=None):
    """Evolve the 2-D test `case` with the reference build; returns
    {iteration: {axis: {name: cut}}} for the x and y cuts through the
    points `fixed` = {axis: (the other two interior indices)}."""
    c = D.TWO_D_TESTS[case]
    L, f = D.two_d_initial(case, ng=ng)
    dt = c["dtfac"] * min(L.dx)
    nit = int(c["final_time"] / dt + 1e-9)
    snaps = list(range(0, nit + 1, c["out_every"]))
    out = {}

    def snap(it, host):
        out[it] = {ax: {n: D.cut_at(L, host, n, ax, fixed[ax]).copy() for n in D.PRIMS}
                   for ax in ("x", "y")}

    evolve_reference(ref, L, f, D.two_d_params(case), (D.BC_NAMES[c["bc"]],) * 6,
                     D.two_d_eos_kw(case), dt, nit, c["method"], snaps, snap)
    return out
