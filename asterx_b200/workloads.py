"""Seeded synthetic inputs for the hot path (numpy, host side).

There is no public dataset for this path: every workload is generated here
from a seed, with the shapes and value ranges of the configurations it stands
for.  Nothing here calls the engine; ``bench.py`` and the tests upload the
arrays themselves.

* ``balsara_box`` -- a uniform patch with the Balsara-1 planar discontinuity
  (left rho=1, p=1, B=(0.5, 1, 0); right rho=0.125, p=0.1, B=(0.5, -1, 0)),
  flat metric, seeded relative perturbations of rho and p; B is set through
  the staggered vector potential A = (0, -Bx z, |x|) whose discrete curl is
  exactly (Bx, sign, 0).
* ``curved_box`` -- a periodic patch with a static curved metric
  (gamma_ij = delta_ij + 0.05 * four seeded symmetric sine modes with
  wavenumbers 1-4, lapse 1 - 0.05 sin, shift amplitude 0.01, extrinsic
  curvature from a further sine mode), smooth seeded primitives plus three
  planar jumps, Lorentz factors up to 10, rho log-uniform in [1e-8, 1],
  magnetisation b^2/rho roughly log-uniform in [1e-3, 10]; B from the curl
  of a seeded periodic vector potential.
* ``c2p_cells`` -- independent cells for the primitive-recovery benchmark.
"""
from __future__ import annotations

import math

import numpy as np

from .abi import Layout


class _XP:
    """Minimal array namespace over numpy or torch (CPU or CUDA), so the same
    generator builds small host boxes for the tests and 256^3 boxes directly
    in device memory for the benchmark."""

    def __init__(self, mod=np, device=None):
        self.mod = mod
        self.torch = mod is not np
        self.device = device

    def __getattr__(self, name):
        return getattr(self.mod, name)

    def asarray(self, a):
        if self.torch:
            return self.mod.as_tensor(np.asarray(a), dtype=self.mod.float64,
                                      device=self.device)
        return np.asarray(a, dtype=np.float64)

    def zeros(self, n):
        if self.torch:
            return self.mod.zeros(n, dtype=self.mod.float64, device=self.device)
        return np.zeros(n)

    def full(self, n, v):
        if self.torch:
            return self.mod.full((n,), float(v), dtype=self.mod.float64,
                                 device=self.device)
        return np.full(n, float(v))

    def copy(self, a):
        return a.clone() if self.torch else a.copy()

    def bcast(self, a, shape):
        """broadcast to shape and flatten to a fresh contiguous array"""
        if self.torch:
            if not hasattr(a, "shape") or a.dim() == 0:
                a = self.mod.as_tensor(a, dtype=self.mod.float64, device=self.device)
            return self.mod.broadcast_to(a, shape).reshape(-1).clone()
        return np.broadcast_to(a, shape).ravel().copy()

    def coords(self, L, centring):
        return [self.asarray(c) for c in L.coords(centring)]

    def uniform(self, rng, lo, hi, n):
        u = rng.uniform(lo, hi, n)
        return self.asarray(u)


_NP = _XP(np)


def _modes(rng, coords, kmax=4, nmodes=4, xp=_NP):
    """Sum of seeded sine modes, periodic on the unit cube."""
    x, y, z = coords
    f = 0.0
    for _ in range(nmodes):
        k = rng.integers(1, kmax + 1, size=3) * rng.choice([-1, 1], size=3)
        ph = rng.uniform(0, 2 * np.pi)
        f = f + xp.sin(2 * math.pi * (float(k[0]) * x + float(k[1]) * y
                                      + float(k[2]) * z) + ph)
    return f / nmodes


def _shape(L):
    return (L.npts[2], L.npts[1], L.sy)


def flat_metric(L: Layout, f: dict, xp=_NP):
    for n in ("gxy", "gxz", "gyz", "betax", "betay", "betaz", "kxx", "kxy",
              "kxz", "kyy", "kyz", "kzz"):
        f[n] = xp.zeros(L.size)
    for n in ("gxx", "gyy", "gzz", "alp"):
        f[n] = xp.full(L.size, 1.0)


def curved_metric(L: Layout, f: dict, rng, amp=0.05, shift_amp=0.01,
                  curv_amp=0.02, xp=_NP):
    cv = xp.coords(L, (0, 0, 0))
    shape = _shape(L)
    diag = {"gxx": 1.0, "gyy": 1.0, "gzz": 1.0, "gxy": 0.0, "gxz": 0.0,
            "gyz": 0.0}
    for n, d in diag.items():
        f[n] = xp.bcast(d + amp * _modes(rng, cv, xp=xp), shape)
    g = [f[n] for n in ("gxx", "gxy", "gxz", "gyy", "gyz", "gzz")]
    m1 = g[0]
    m2 = g[0] * g[3] - g[1] ** 2
    det = (g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] * (g[1] * g[5] - g[4] * g[2])
           + g[2] * (g[1] * g[4] - g[3] * g[2]))
    assert bool((m1 > 0).all()) and bool((m2 > 0).all()) and bool((det > 0).all()), \
        "metric not positive definite"
    f["alp"] = xp.bcast(1.0 - amp * _modes(rng, cv, xp=xp), shape)
    for n in ("betax", "betay", "betaz"):
        f[n] = xp.bcast(shift_amp * _modes(rng, cv, xp=xp), shape)
    for n in ("kxx", "kxy", "kxz", "kyy", "kyz", "kzz"):
        f[n] = xp.bcast(curv_amp * _modes(rng, cv, xp=xp), shape)


def _curl_stag(L: Layout, Ax, Ay, Az, xp=_NP):
    """Face curl of edge A exactly as AsterX/src/computeBfromA.cxx:32-55, on
    every face whose neighbours exist."""
    v = L.view
    ax, ay, az = v(Ax), v(Ay), v(Az)
    idx = [1.0 / d for d in L.dx]
    bx, by, bz = (v(xp.zeros(L.size)) for _ in range(3))
    bx[:-1, :-1, :] = (idx[1] * (az[:-1, 1:, :] - az[:-1, :-1, :])
                       - idx[2] * (ay[1:, :-1, :] - ay[:-1, :-1, :]))
    by[:-1, :, :-1] = (idx[2] * (ax[1:, :, :-1] - ax[:-1, :, :-1])
                       - idx[0] * (az[:-1, :, 1:] - az[:-1, :, :-1]))
    bz[:, :-1, :-1] = (idx[0] * (ay[:, :-1, 1:] - ay[:, :-1, :-1])
                       - idx[1] * (ax[:, 1:, :-1] - ax[:, :-1, :-1]))
    return bx.reshape(-1), by.reshape(-1), bz.reshape(-1)


def _v2c(L: Layout, a, xp=_NP):
    """Vertex-to-cell average (the 8 corners, AsterUtils aster_interp.hxx:
    23-36), defined on every cell whose corners exist."""
    v = L.view(a)
    out = L.view(xp.zeros(L.size))
    out[:-1, :-1, :-1] = (v[:-1, :-1, :-1] + v[:-1, :-1, 1:] + v[:-1, 1:, :-1]
                          + v[:-1, 1:, 1:] + v[1:, :-1, :-1] + v[1:, :-1, 1:]
                          + v[1:, 1:, :-1] + v[1:, 1:, 1:]) / 8.0
    return out.reshape(-1)


def _sqrt_detg_cell(L: Layout, f, xp=_NP):
    g = [_v2c(L, f[n], xp) for n in ("gxx", "gxy", "gxz", "gyy", "gyz", "gzz")]
    det = (g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] * (g[1] * g[5] - g[4] * g[2])
           + g[2] * (g[1] * g[4] - g[3] * g[2]))
    return xp.sqrt(xp.where(det > 0, det, det * 0 + 1.0)), g


def _finish_prims(L, f, gamma, ye=None, xp=_NP):
    """eps, temperature, entropy (kappa) and Ye from rho and press for an
    ideal gas (EOSX/src/eos_3p_idealgas/eos_3p_idealgas.hxx:115-229)."""
    rho, press = f["rho"], f["press"]
    f["eps"] = press / (rho * (gamma - 1.0))
    f["temperature"] = (gamma - 1.0) * f["eps"]
    f["entropy"] = (gamma - 1.0) * f["eps"] * rho ** (1.0 - gamma)
    f["Ye"] = xp.full(L.size, 0.5) if ye is None else ye


def _cell_B_from_stag(L, f, xp=_NP):
    v = L.view
    dB = []
    for n, ax in (("dBx_stag", 2), ("dBy_stag", 1), ("dBz_stag", 0)):
        s = v(f[n])
        c = v(xp.zeros(L.size))
        if ax == 2:
            c[:, :, :-1] = 0.5 * (s[:, :, :-1] + s[:, :, 1:])
        elif ax == 1:
            c[:, :-1, :] = 0.5 * (s[:, :-1, :] + s[:, 1:, :])
        else:
            c[:-1, :, :] = 0.5 * (s[:-1, :, :] + s[1:, :, :])
        dB.append(c.reshape(-1))
    sq, _ = _sqrt_detg_cell(L, f, xp)
    f["dBx"], f["dBy"], f["dBz"] = dB
    f["Bvecx"], f["Bvecy"], f["Bvecz"] = (d / sq for d in dB)


def balsara_box(n=64, ng=3, gamma=5.0 / 3.0, seed=1, pert=1e-3):
    """Config-1 patch: Balsara-1 discontinuity at x = 0 on [-0.5, 0.5]^3."""
    if isinstance(n, int):
        n = (n, n, n)
    L = Layout(n, ng, tuple(1.0 / v for v in n), (-0.5, -0.5, -0.5))
    rng = np.random.default_rng(seed)
    f = {}
    flat_metric(L, f)
    xc, _, _ = L.coords((1, 1, 1))
    shape = L.view(L.zeros()).shape
    left = np.broadcast_to(xc < 0, shape).ravel()
    f["rho"] = np.where(left, 1.0, 0.125) * (1 + pert * rng.uniform(-1, 1, L.size))
    f["press"] = np.where(left, 1.0, 0.1) * (1 + pert * rng.uniform(-1, 1, L.size))
    for nm in ("velx", "vely", "velz"):
        f[nm] = L.zeros()
    _finish_prims(L, f, gamma)
    # vector potential: A_x = 0, A_y = -Bx z (y-edges: z at vertices),
    # A_z = |x| (z-edges: x at vertices) -> B = (0.5, +1 for x<0 / -1, 0)
    xv, yv, zv = L.coords((0, 0, 0))
    f["Avec_x"] = L.zeros()
    f["Avec_y"] = np.broadcast_to(-0.5 * zv, shape).ravel().copy()
    f["Avec_z"] = np.broadcast_to(np.abs(xv), shape).ravel().copy()
    f["Psi"] = L.zeros()
    f["dBx_stag"], f["dBy_stag"], f["dBz_stag"] = _curl_stag(
        L, f["Avec_x"], f["Avec_y"], f["Avec_z"])
    _cell_B_from_stag(L, f)
    return L, f


def curved_box(n=24, ng=3, gamma=4.0 / 3.0, seed=2, wmax=10.0, njumps=3,
               with_ye=False, sigma=(1e-3, 10.0), jump=(2.0, 8.0),
               rho_min=1e-8, theta=(1e-2, 1.0), xp=None, a_amp=0.05, rho_max=1.0):
    """Config-2-like periodic patch on [0, 1]^3 with a curved static metric.
    ``xp`` selects the array library: None/numpy for host arrays, or an
    ``_XP(torch, device)`` to build the box in device memory."""
    xp = xp or _NP
    if isinstance(n, int):
        n = (n, n, n)
    L = Layout(n, ng, tuple(1.0 / v for v in n), (0.0, 0.0, 0.0))
    rng = np.random.default_rng(seed)
    shape = _shape(L)
    f = {}
    curved_metric(L, f, rng, xp=xp)
    cc = xp.coords(L, (1, 1, 1))

    def smooth(lo, hi, kmax=3, nmodes=3):
        u = 0.5 * (1 + _modes(rng, cc, kmax=kmax, nmodes=nmodes, xp=xp))
        return xp.bcast(lo + (hi - lo) * u, shape)

    # vector potential on edges, B from its curl
    ev = {"Avec_x": (1, 0, 0), "Avec_y": (0, 1, 0), "Avec_z": (0, 0, 1)}
    for nm, cent in ev.items():
        c = xp.coords(L, cent)
        f[nm] = xp.bcast(a_amp * _modes(rng, c, kmax=3, xp=xp), shape)
    f["Psi"] = xp.bcast(1e-3 * _modes(rng, xp.coords(L, (0, 0, 0)), xp=xp), shape)
    f["dBx_stag"], f["dBy_stag"], f["dBz_stag"] = _curl_stag(
        L, f["Avec_x"], f["Avec_y"], f["Avec_z"], xp)
    _cell_B_from_stag(L, f, xp)
    _, g = _sqrt_detg_cell(L, f, xp)

    # velocity: Lorentz factor in [1, wmax] along a smooth unit direction
    W = smooth(1.0, wmax, kmax=1, nmodes=2)
    th = smooth(0.3 * np.pi, 0.7 * np.pi, kmax=1, nmodes=2)
    ph0 = rng.uniform(0, 2 * np.pi)
    ph = smooth(ph0, ph0 + 0.5 * np.pi, kmax=1, nmodes=2)
    d = [xp.sin(th) * xp.cos(ph), xp.sin(th) * xp.sin(ph), xp.cos(th)]
    gd = [[g[0], g[1], g[2]], [g[1], g[3], g[4]], [g[2], g[4], g[5]]]

    def lower(v):
        return [gd[i][0] * v[0] + gd[i][1] * v[1] + gd[i][2] * v[2] for i in range(3)]

    def dot(a, b):
        return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]

    nrm = dot(d, lower(d))
    nrm = xp.where(nrm > 1e-12, nrm, nrm * 0 + 1.0)
    vmag = xp.sqrt(1.0 - 1.0 / W ** 2)
    vel = [di * (vmag / xp.sqrt(nrm)) for di in d]
    f["velx"], f["vely"], f["velz"] = vel
    # density from the magnetisation, then planar jumps
    B = [f["Bvecx"], f["Bvecy"], f["Bvecz"]]
    vlow = lower(vel)
    Bsq = dot(B, lower(B))
    vB = dot(vlow, B)
    bsq = Bsq / W ** 2 + vB ** 2
    sigma_f = 10 ** smooth(np.log10(sigma[0]), np.log10(sigma[1]))
    rho = xp.clip(bsq / sigma_f, rho_min, rho_max)
    theta_f = 10 ** smooth(np.log10(theta[0]), np.log10(theta[1]))
    xyz = [xp.bcast(c, shape) for c in cc]
    for _ in range(njumps):
        nv = rng.normal(size=3)
        nv /= np.linalg.norm(nv)
        x0 = rng.uniform(0.2, 0.8)
        side = (float(nv[0]) * (xyz[0] - x0) + float(nv[1]) * (xyz[1] - 0.5)
                + float(nv[2]) * (xyz[2] - 0.5)) > 0
        rho = xp.where(side, rho * float(rng.uniform(*jump)), rho)
        theta_f = xp.where(side, theta_f / float(rng.uniform(1.5, 4)), theta_f)
    f["rho"] = xp.clip(rho, rho_min, rho_max)
    f["press"] = f["rho"] * theta_f
    ye = smooth(0.05, 0.5) if with_ye else None
    _finish_prims(L, f, gamma, ye, xp)
    return L, f


# ---------------------------------------------------------------------------
# Synthetic tabulated equation of state
# ---------------------------------------------------------------------------
TAB_NV = 19  # variables per node of the EOSX table layout
TAB_LOGPRESS, TAB_LOGENERGY, TAB_ENTROPY, TAB_CS2 = 0, 1, 2, 4


def tab_thermo(rho, temp, ye, xp=_NP):
    """Closed-form thermodynamics of the synthetic table:
    P = rho T (1 + Ye) + T^4 / 3 + 100 rho^2 (ideal gas + radiation + cold
    part), with the specific energy and entropy that satisfy the first law
    for that pressure,
        eps = 1.5 T (1 + Ye) + T^4 / rho + 100 rho,
        s   = (1 + Ye) (1.5 ln T - ln rho) + 4 T^3 / (3 rho),
    and the relativistic sound speed cs^2 = (dP/drho)_s / h, h = 1 + eps + P/rho.
    Returns (press, eps, entropy, cs2)."""
    y1 = 1.0 + ye
    press = rho * temp * y1 + temp ** 4 / 3.0 + 100.0 * rho ** 2
    eps = 1.5 * temp * y1 + temp ** 4 / rho + 100.0 * rho
    ent = y1 * (1.5 * xp.log(temp) - xp.log(rho)) + 4.0 * temp ** 3 / (3.0 * rho)
    p_rho = temp * y1 + 200.0 * rho
    p_t = rho * y1 + 4.0 * temp ** 3 / 3.0
    s_rho = -(y1 / rho + 4.0 * temp ** 3 / (3.0 * rho ** 2))
    s_t = 1.5 * y1 / temp + 4.0 * temp ** 2 / rho
    dp_rho_s = p_rho - p_t * s_rho / s_t
    h = 1.0 + eps + press / rho
    return press, eps, ent, dp_rho_s / h


def synthetic_table(nrho=200, ntemp=100, nye=60, rho=(1e-14, 1e-2), temp=(0.01, 100.0),
                    ye=(0.05, 0.6)):
    """Uniform table on (ln rho, ln T, Ye) in the EOSX layout: 19 variables
    per node, variable fastest, node = i_rho + nrho (i_T + ntemp i_Ye);
    variable 0 ln P, 1 ln eps (energy shift 0, eps > 0 everywhere), 2 entropy,
    4 cs^2, the others zero.  Returns (logrho, logtemp, ye, table)."""
    lr = np.linspace(math.log(rho[0]), math.log(rho[1]), nrho)
    lt = np.linspace(math.log(temp[0]), math.log(temp[1]), ntemp)
    ys = np.linspace(ye[0], ye[1], nye)
    Y, T, R = np.meshgrid(ys, np.exp(lt), np.exp(lr), indexing="ij")
    press, eps, ent, cs2 = tab_thermo(R, T, Y)
    table = np.zeros((nye, ntemp, nrho, TAB_NV))
    table[..., TAB_LOGPRESS] = np.log(press)
    table[..., TAB_LOGENERGY] = np.log(eps)
    table[..., TAB_ENTROPY] = ent
    table[..., TAB_CS2] = cs2
    return lr, lt, ys, table.reshape(-1)


def tabulated_box(n=24, ng=3, seed=5, wmax=10.0, sigma=(1e-3, 10.0), theta=(1e-2, 1.0),
                  temp_scale=0.5, xp=None, **kw):
    """Config-5 patch: the curved-metric box with Ye smooth in [0.05, 0.5],
    densities brought inside the table (vector potential scaled by 10^-1.5, so
    b^2 and rho drop by 10^-3; rho in [1e-10, 5e-3]) and the thermodynamics
    of the synthetic table: T = temp_scale * (p/rho of the ideal-gas box),
    clipped to [0.011, 90], then P, eps and entropy in closed form."""
    xp = xp or _NP
    L, f = curved_box(n=n, ng=ng, seed=seed, wmax=wmax, with_ye=True, sigma=sigma,
                      theta=theta, xp=xp, a_amp=0.05 * 10 ** -1.5, rho_min=1e-10,
                      rho_max=5e-3, **kw)
    rho, ye = f["rho"], f["Ye"]
    temp = xp.clip(temp_scale * f["press"] / rho, 0.011, 90.0)
    press, eps, ent, _ = tab_thermo(rho, temp, ye, xp)
    f["temperature"], f["press"], f["eps"], f["entropy"] = temp, press, eps, ent
    return L, f


def saved_from_prims(f, xp=None):
    xp = xp or _NP
    for n, s in (("rho", "saved_rho"), ("velx", "saved_velx"), ("vely", "saved_vely"),
                 ("velz", "saved_velz"), ("eps", "saved_eps"), ("Ye", "saved_Ye")):
        f[s] = xp.copy(f[n])


def c2p_cells(ncells, seed=4, gamma=5.0 / 3.0, rho_range=(1e-12, 1e-2),
              eps_range=(1e-6, 10.0), w_range=(1.0, 50.0),
              sigma_range=(1e-4, 100.0), metric_amp=0.05, device=None, ye=None):
    """Independent cells of the recovery microbenchmark: rho and eps
    log-uniform, W uniform, magnetisation b^2/rho log-uniform, isotropic
    velocity and field directions, a random metric gamma_ij = delta_ij +
    metric_amp * U(-1, 1) per component; ideal-gas pressure (Gamma `gamma`),
    or the synthetic table's when `ye` = (lo, hi) gives a Ye range (then the
    temperature is found from eps by bisection on the closed form).
    Generated with torch on `device` (a torch.Generator seeded with `seed`)
    when given, else with numpy.  Returns a dict of 1-D float64 arrays:
    the primitives (rho, eps, press, velx.., Bvecx.., W, Ye, temperature,
    entropy), the metric (gxx..gzz) and the densitised conserved variables
    (dens, momx.., tau, DYe, DEnt, dBx..) from the exact Valencia map
    (AsterX/src/prim2con.hxx:38-83), plus the learned-guess targets: the
    position t_u of x = h W in the Palenzuela bracket, and ln W (t_lnw);
    also ln(h W) (t_lnx)."""
    N = int(ncells)
    if device is None:
        rng = np.random.default_rng(seed)
        xp = np
        uni = lambda lo, hi: rng.uniform(lo, hi, N)
        nrm = lambda: rng.normal(size=(3, N))
        stack = np.stack
    else:
        import torch
        gen = torch.Generator(device=device)
        gen.manual_seed(int(seed))
        xp = torch
        uni = lambda lo, hi: lo + (hi - lo) * torch.rand(N, generator=gen, device=device,
                                                           dtype=torch.float64)
        nrm = lambda: torch.randn((3, N), generator=gen, device=device, dtype=torch.float64)
        stack = torch.stack
    lu = lambda a, b: xp.exp(uni(math.log(a), math.log(b)))
    rho = lu(*rho_range)
    eps = lu(*eps_range)
    W = uni(*w_range)
    sigma = lu(*sigma_range)
    g = [1.0 + metric_amp * uni(-1, 1), metric_amp * uni(-1, 1), metric_amp * uni(-1, 1),
         1.0 + metric_amp * uni(-1, 1), metric_amp * uni(-1, 1), 1.0 + metric_amp * uni(-1, 1)]
    gd = [[g[0], g[1], g[2]], [g[1], g[3], g[4]], [g[2], g[4], g[5]]]

    def lower(v):
        return [gd[i][0] * v[0] + gd[i][1] * v[1] + gd[i][2] * v[2] for i in range(3)]

    def dot(a, b):
        return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]

    def unit():
        v = nrm()
        n = xp.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
        return [v[0] / n, v[1] / n, v[2] / n]

    dv = unit()
    nn = dot(dv, lower(dv))
    vmag = xp.sqrt(1.0 - 1.0 / W ** 2) / xp.sqrt(nn)
    vel = [d * vmag for d in dv]
    db = unit()
    vlow = lower(vel)
    b2_per = dot(db, lower(db)) / W ** 2 + dot(vlow, db) ** 2
    bmag = xp.sqrt(sigma * rho / b2_per)
    B = [d * bmag for d in db]
    if ye is None:
        Ye = rho * 0 + 0.5
        press = (gamma - 1.0) * rho * eps
        temp = (gamma - 1.0) * eps
        ent = (gamma - 1.0) * eps * rho ** (1.0 - gamma)
    else:
        Ye = uni(*ye)
        # invert eps(rho, T, Ye) of the synthetic table by bisection in ln T
        lo = rho * 0 + math.log(0.01)
        hi = rho * 0 + math.log(100.0)
        for _ in range(80):
            mid = 0.5 * (lo + hi)
            e_mid = tab_thermo(rho, xp.exp(mid), Ye, xp)[1]
            up = e_mid > eps
            hi = xp.where(up, mid, hi)
            lo = xp.where(up, lo, mid)
        temp = xp.exp(0.5 * (lo + hi))
        press, eps, ent, _ = tab_thermo(rho, temp, Ye, xp)
    det = (g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] * (g[1] * g[5] - g[4] * g[2])
           + g[2] * (g[1] * g[4] - g[3] * g[2]))
    sq = xp.sqrt(det)
    Bl = lower(B)
    Wc = 1.0 / xp.sqrt(1.0 - dot(vlow, vel))
    bst = Wc * dot(B, vlow)
    bl = [Bl[i] / Wc + bst * vlow[i] for i in range(3)]
    bs2 = (dot(B, Bl) + bst * bst) / (Wc * Wc)
    hW2 = Wc * Wc * (rho * (1.0 + eps) + press + bs2)
    out = dict(rho=rho, eps=eps, press=press, W=Wc, Ye=Ye, temperature=temp, entropy=ent)
    for q, ax in enumerate("xyz"):
        out["vel" + ax] = vel[q]
        out["Bvec" + ax] = B[q]
        out["mom" + ax] = sq * (hW2 * vlow[q] - bst * bl[q])
        out["dB" + ax] = sq * B[q]
    for q, nm in enumerate(["gxx", "gxy", "gxz", "gyy", "gyz", "gzz"]):
        out[nm] = g[q]
    out["dens"] = sq * rho * Wc
    out["tau"] = sq * (hW2 - (press + 0.5 * bs2) - bst * bst) - out["dens"]
    out["DYe"] = out["dens"] * Ye
    out["DEnt"] = out["dens"] * ent
    h = 1.0 + eps + press / rho
    x = h * Wc
    # position of x = h W in the Palenzuela scheme's initial bracket
    # [max(1e-10, 1 + q - s), 2 + 2 q - s] (c2p_1DPalenzuela.hxx:395-398),
    # q = tau / D, s = B^2 / D with undensitised D, tau, B
    D = rho * Wc
    q = (out["tau"] / sq) / D
    s_ = dot(B, Bl) / D
    lo = xp.maximum(q * 0 + 1e-10, 1.0 + q - s_)
    hi = 2.0 + 2.0 * q - s_
    out["t_u"] = (x - lo) / (hi - lo)
    out["t_lnx"] = xp.log(x)
    out["t_lnw"] = xp.log(Wc)
    return out


def cons_from_prims(L: Layout, f: dict, xp=None):
    """Densitised conserved variables of every cell from its primitives and
    the vertex-to-cell metric (the Valencia prim->cons map of
    AsterX/src/prim2con.hxx:38-83), written into f, together with
    zvec^i = W v^i and svec^i = rho h W^2 v^i."""
    xp = xp or _NP
    sq, g = _sqrt_detg_cell(L, f, xp)
    gd = [[g[0], g[1], g[2]], [g[1], g[3], g[4]], [g[2], g[4], g[5]]]

    def lower(v):
        return [gd[i][0] * v[0] + gd[i][1] * v[1] + gd[i][2] * v[2] for i in range(3)]

    def dot(a, b):
        return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]

    v = [f["velx"], f["vely"], f["velz"]]
    B = [f["Bvecx"], f["Bvecy"], f["Bvecz"]]
    vl = lower(v)
    Bl = lower(B)
    v2 = xp.clip(dot(vl, v), 0.0, 1 - 1e-15)
    W = 1.0 / xp.sqrt(1.0 - v2)
    bst = W * dot(B, vl)
    bl = [Bl[i] / W + bst * vl[i] for i in range(3)]
    bs2 = (dot(B, Bl) + bst * bst) / (W * W)
    rho, eps, press = f["rho"], f["eps"], f["press"]
    hW2 = W * W * (rho * (1.0 + eps) + press + bs2)
    f["dens"] = sq * rho * W
    f["momx"], f["momy"], f["momz"] = [sq * (hW2 * vl[i] - bst * bl[i]) for i in range(3)]
    f["tau"] = sq * (hW2 - (press + 0.5 * bs2) - bst * bst) - f["dens"]
    f["DYe"] = f["dens"] * f["Ye"]
    f["DEnt"] = f["dens"] * f["entropy"]
    # the velocity-like variables the fluxes reconstruct with recon_type
    # z_vec / s_vec, as the recovery writes them back (con2prim.cxx:432-441)
    rhoh = rho + rho * eps + press
    for i, ax in enumerate("xyz"):
        f["zvec_" + ax] = W * v[i]
        f["svec_" + ax] = rhoh * W * W * v[i]


def perturbed_saved(f: dict, seed=7, amp=1e-2):
    """Saved primitives (the recovery seeds) as the primitives times
    (1 + amp * U(-1, 1)), as a time step leaves them."""
    rng = np.random.default_rng(seed)
    for n, s in (("rho", "saved_rho"), ("velx", "saved_velx"), ("vely", "saved_vely"),
                 ("velz", "saved_velz"), ("eps", "saved_eps"), ("Ye", "saved_Ye")):
        f[s] = f[n] * (1 + amp * rng.uniform(-1, 1, f[n].shape))
