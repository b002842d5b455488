"""Convert the reference's own regression outputs (the TSV 1-D cuts under
AsterX/test/<case>/ of the reference checkout, compared there at 1e-8 by
AsterX/test/test.ccl) into compact fixtures, tests/golden/tsv_<case>.npz.

Each fixture of a 1-D test holds, for the cut along the shock direction, the
iterations 0, 10, ..., 80, the point indices (ghosts included) and
coordinates, and the values of rho, velx/y/z, eps, press and Bvecx/y/z.  A
2-D test's fixture holds the same for its x and y cuts, with the keys
prefixed by the axis ("x_rho", "y_index", ...) and the indices of the point
the cut passes through ("x_fixed" = (j, k) of the x cut, "y_fixed" = (i, k)).
The case's parameters (the .par file's settings the hot path reads) are
restated in asterx_b200/driver.py (ONE_D_TESTS, TWO_D_TESTS); this script
copies numbers only.

Run from the repository root with the reference checkout named by
AXB_REFERENCE_ROOT (or as the first argument):
    python tests/golden/make_tsv_golden.py <reference root>
"""
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["Balsara1_shocktube_xdir_ppm", "Balsara1_shocktube_xdir_wenoz",
         "Balsara1_shocktube_xdir_mp5", "Balsara1_shocktube_xdir_godunov",
         "Balsara1_shocktube_xdir_monocentral", "Balsara1_shocktube_xdir_ppm_PalenzuelaC2P",
         "Balsara1_shocktube_ydir_ppm", "Balsara1_shocktube_zdir_ppm",
         "Balsara2_shocktube_xdir_ppm", "Balsara3_shocktube_xdir_minmod_LxF",
         "Balsara4_shocktube_xdir_ppm", "Balsara5_shocktube_xdir_ppm"]
CASES_2D = ["Magnetic_rotor", "Cylindrical_blast"]
VARS = {"rho": ["rho"], "vel": ["velx", "vely", "velz"], "eps": ["eps"],
        "press": ["press"], "bvec": ["Bvecx", "Bvecy", "Bvecz"]}


def read_tsv(path):
    with open(path) as fh:
        header = fh.readline().lstrip("#").split()
        cols = [h.split(":", 1)[1] for h in header]
        rows = [line.split() for line in fh if line.strip()]
    data = np.array([[float(v) for v in r] for r in rows])
    return cols, data


def convert(root, case):
    d = os.path.join(root, "AsterX", "test", case)
    axis = "y" if "_ydir_" in case else "z" if "_zdir_" in case else "x"
    col_idx = {"x": "i", "y": "j", "z": "k"}[axis]
    out = {}
    its = sorted({int(os.path.basename(p).split(".it")[1][:6])
                  for p in glob.glob(os.path.join(d, "hydrobasex-rho.it*.%s.tsv" % axis))})
    out["iterations"] = np.array(its)
    for group, names in VARS.items():
        per = {n: [] for n in names}
        for it in its:
            cols, data = read_tsv(os.path.join(d, "hydrobasex-%s.it%06d.%s.tsv" % (group, it, axis)))
            if "index" not in out:
                out["index"] = data[:, cols.index(col_idx)].astype(np.int64)
                out["coord"] = data[:, cols.index(axis)]
                out["time"] = []
            if group == "rho":
                out["time"].append(data[0, cols.index("time")])
            for n in names:
                per[n].append(data[:, cols.index(n)])
        for n in names:
            out[n] = np.array(per[n])
    out["time"] = np.array(out["time"])
    out["axis"] = np.array(axis)
    np.savez_compressed(os.path.join(HERE, "tsv_%s.npz" % case), **out)
    return out


def convert_2d(root, case):
    d = os.path.join(root, "AsterX", "test", case)
    out = {}
    for axis in ("x", "y"):
        col_idx = {"x": "i", "y": "j"}[axis]
        fixed_cols = {"x": ("j", "k"), "y": ("i", "k")}[axis]
        its = sorted({int(os.path.basename(p).split(".it")[1][:6])
                      for p in glob.glob(os.path.join(d, "hydrobasex-rho.it*.%s.tsv" % axis))})
        out["iterations"] = np.array(its)
        times = []
        for group, names in VARS.items():
            per = {n: [] for n in names}
            for it in its:
                cols, data = read_tsv(os.path.join(d, "hydrobasex-%s.it%06d.%s.tsv"
                                                   % (group, it, axis)))
                key = axis + "_index"
                if key not in out:
                    out[key] = data[:, cols.index(col_idx)].astype(np.int64)
                    out[axis + "_coord"] = data[:, cols.index(axis)]
                    out[axis + "_fixed"] = np.array(
                        [int(data[0, cols.index(c)]) for c in fixed_cols])
                if group == "rho":
                    times.append(data[0, cols.index("time")])
                for n in names:
                    per[n].append(data[:, cols.index(n)])
            for n in names:
                out[axis + "_" + n] = np.array(per[n])
        out["time"] = np.array(times)
    np.savez_compressed(os.path.join(HERE, "tsv_%s.npz" % case), **out)
    return out


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AXB_REFERENCE_ROOT", "")
    if not root or not os.path.isdir(os.path.join(root, "AsterX", "test")):
        sys.exit("usage: make_tsv_golden.py <reference root>")
    for c in CASES:
        o = convert(root, c)
        print(c, o["rho"].shape, o["iterations"].tolist())
    for c in CASES_2D:
        o = convert_2d(root, c)
        print(c, o["x_rho"].shape, o["y_rho"].shape, o["iterations"].tolist(),
              o["x_fixed"].tolist(), o["y_fixed"].tolist())
