"""Generate the golden fixtures of tests/golden/ from the reference's own
sources (oracle/_ref/libaxref.so, compiled from the reference checkout
through oracle/refshim).  Each fixture stores the seeded inputs' recipe
(generator arguments and parameters) and the reference's interior outputs of
one routine group; tests/test_golden.py regenerates the inputs with the same
seeded generator and checks the oracle restatement against the stored
outputs bit for bit.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from asterx_b200 import abi  # noqa: E402
from asterx_b200 import workloads as W  # noqa: E402
from oracle.oracle import reference  # noqa: E402

CASES = [
    dict(name="rhs_ppm_hlle", group="rhs_group", box=dict(n=6, ng=5, seed=41),
         params=dict(reconstruction_method="ppm", flux_type="hlle")),
    dict(name="rhs_wenoz_hlle_fd4", group="rhs_group", box=dict(n=6, ng=5, seed=42),
         params=dict(reconstruction_method="wenoz", flux_type="hlle", local_spatial_order=4)),
    dict(name="rhs_mp5_lxf", group="rhs_group", box=dict(n=6, ng=5, seed=43),
         params=dict(reconstruction_method="mp5", flux_type="lxf")),
    dict(name="c2p_noble_pal", group="con2prim_group", box=dict(n=6, ng=5, seed=44, c2p=1),
         params=dict(c2p_prime="noble", c2p_second="palenzuela", c2p_tol=1e-12, max_iter=60)),
    dict(name="c2p_pal_noble", group="con2prim_group", box=dict(n=6, ng=5, seed=45, c2p=1),
         params=dict(c2p_prime="palenzuela", c2p_second="noble", c2p_tol=1e-12, max_iter=60)),
]
GAMMA = 4.0 / 3.0
EOS_KW = dict(rho=(1e-40, 1e10), eps=(0.0, 1e10))
OUTPUTS = {"rhs_group": abi.HYDRO_RHS + abi.AVEC_RHS,
           "con2prim_group": ["rho", "eps", "press", "velx", "vely", "velz", "Bvecx",
                              "Bvecy", "Bvecz", "temperature", "entropy", "Ye",
                              "con2prim_flag"] + abi.CONS + abi.SAVED}
CENT = {"Avec_x_rhs": (1, 0, 0), "Avec_y_rhs": (0, 1, 0), "Avec_z_rhs": (0, 0, 1),
        "Psi_rhs": (0, 0, 0)}


def build_inputs(box):
    L, f = W.curved_box(n=box["n"], ng=box["ng"], seed=box["seed"], wmax=2.0,
                        sigma=(1e-3, 0.3), theta=(0.1, 1.0))
    if box.get("c2p"):
        W.cons_from_prims(L, f)
        W.perturbed_saved(f, seed=box["seed"] + 1)
    for n in abi.GF_NAMES:
        f.setdefault(n, L.zeros())
    return L, f


def run_case(lib, case):
    L, f = build_inputs(case["box"])
    p = abi.default_params(**case["params"])
    host = {n: a.copy() for n, a in f.items()}
    lib.setup(L, p, host)
    lib.eos_idealgas(GAMMA, **EOS_KW)
    getattr(lib, case["group"])()
    return {n: L.view(host[n])[L.interior(CENT.get(n, (1, 1, 1)))].copy()
            for n in OUTPUTS[case["group"]]}


def main():
    ref = reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libaxref.so is not built")
    for case in CASES:
        out = run_case(ref, case)
        np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **out)
        with open(os.path.join(HERE, case["name"] + ".json"), "w") as fh:
            json.dump({k: case[k] for k in ("name", "group", "box", "params")}, fh,
                      indent=1)
        print("wrote", case["name"])


if __name__ == "__main__":
    main()
