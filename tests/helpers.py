"""Shared helpers for the parity tests."""
import numpy as np

from asterx_b200 import abi


def errors(got, want):
    """(normalised max error, L2 relative error) of two arrays: the max
    absolute difference divided by the max |want|, and ||got-want||/||want||."""
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    scale = np.max(np.abs(want))
    if scale == 0:
        scale = 1.0
    d = np.abs(got - want)
    l2 = np.linalg.norm(want)
    return float(np.max(d) / scale), float(np.linalg.norm(got - want) / (l2 if l2 else 1.0))


EDGE_CENTRING = {"Avec_x_rhs": (1, 0, 0), "Avec_y_rhs": (0, 1, 0),
                 "Avec_z_rhs": (0, 0, 1), "Psi_rhs": (0, 0, 0)}


def interior(L, name, arr):
    c = EDGE_CENTRING.get(name, (1, 1, 1))
    return L.view(arr)[L.interior(c)]


def full_fields(L, f):
    """Every grid function the engine and the checker know, zero-filled where
    the workload does not set it."""
    out = dict(f)
    for n in abi.GF_NAMES:
        if n not in out:
            out[n] = L.zeros()
    return out


CENTRING = {"Avec_x": (1, 0, 0), "Avec_y": (0, 1, 0), "Avec_z": (0, 0, 1),
            "Psi": (0, 0, 0), "dBx_stag": (0, 1, 1), "dBy_stag": (1, 0, 1),
            "dBz_stag": (1, 1, 0)}
CENTRING.update(EDGE_CENTRING)
EVOLVED = abi.CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]
EVOLVED_RHS = abi.HYDRO_RHS + ["Avec_x_rhs", "Avec_y_rhs", "Avec_z_rhs", "Psi_rhs"]
PRIMS_SYNC = ["rho", "velx", "vely", "velz", "eps", "press", "temperature", "Ye",
              "entropy", "Bvecx", "Bvecy", "Bvecz"]


def periodic_sync(L, f, names):
    """Host periodic ghost fill with the same semantics as axb_sync_periodic:
    every point outside the interior of its centring takes the value of its
    periodic image."""
    import numpy as np
    for n in names:
        c = CENTRING.get(n, (1, 1, 1))
        idx = []
        for d in (2, 1, 0):
            npts = L.n[d] + 2 * L.ng + (0 if c[d] else 1)
            hi = L.ng + L.n[d] + (0 if c[d] else 1)
            ii = np.arange(npts)
            out = ii.copy()
            ghost = (ii < L.ng) | (ii >= hi)
            out[ghost] = L.ng + (ii[ghost] - L.ng) % L.n[d]
            idx.append(out)
        v = L.view(f[n])
        k, j, i = idx
        sub = v[:len(k), :len(j), :len(i)]
        sub[...] = sub[np.ix_(k, j, i)]


def ref_stage(L, f, fn, alpha, beta, gamma, dt):
    for u, r in zip(EVOLVED, EVOLVED_RHS):
        c = CENTRING.get(u, (1, 1, 1))
        sl = L.interior(c)
        vu, vn, vr = L.view(f[u]), L.view(fn[u]), L.view(f[r])
        vu[sl] = alpha * vn[sl] + beta * vu[sl] + (gamma * dt) * vr[sl]
