"""Regenerate the golden fixtures of this directory from mdelast's own test data.

Run where an mdelast checkout is available (``--ref``, else ``$MDELAST_REFERENCE``, else a
checkout called ``reference`` beside this repository):

    python tests/golden/make_golden.py [--ref PATH]

Writes
* ``smoke_static.json``: benchmark S Part A6 expected values per table interpolation
  (``benchmarks/expected/smoke.json:34-88``, rel tol 1e-7), the Part A and C bounds
  (``smoke.json:6-33, 90-113``) and the Part B dynamics bounds (``smoke.json:114-170``);
* ``nialco_lammps.npz``: the fixed 500-atom Ni-Al-Co cell and the LAMMPS values it is checked
  against (``benchmarks/smoke/reference/``), converted as ``run_smoke.py:281-328`` does:
  positions [A] wrapped into the box, 0-based types, forces [eV/A], energy [eV/atom],
  virial [GPa, + = compressive, Voigt order], Born matrix [GPa, LAMMPS order].

The data come from the MIT-licensed mdelast repository (Copyright (c) 2026 R. Shikler,
M. Krief, Y. Ashkenazy); the LAMMPS values were produced by its authors.
"""

import argparse
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NKTV2P = 1.6021765e6  # LAMMPS metal units: eV/A^3 -> bar


def read_lammps_data(path):
    lines = open(path).read().splitlines()
    lo, hi = (float(x) for x in next(l for l in lines if l.endswith("xlo xhi")).split()[:2])
    start = next(i for i, l in enumerate(lines) if l.startswith("Atoms")) + 2
    rows = np.array([[float(x) for x in l.split()] for l in lines[start:] if l.strip()])
    rows = rows[np.argsort(rows[:, 0])]
    return hi - lo, rows[:, 1].astype(int) - 1, rows[:, 2:5]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    a = ap.parse_args()
    from refroot import reference_root
    a.ref = reference_root(a.ref)
    smoke = json.load(open(os.path.join(a.ref, "benchmarks", "expected", "smoke.json")))
    checks = smoke["checks"]
    out = {"source": "mdelast benchmarks/expected/smoke.json (MIT)", "rel_tol": 1e-7,
           "quintic": {}, "bspline": {}, "bounds": {}}
    for k, v in checks.items():
        if k.startswith("static.") and "expected_by_interpolation" in v:
            for interp in ("quintic", "bspline"):
                out[interp][k[len("static."):]] = v["expected_by_interpolation"][interp]
        elif k.startswith("ternary.") or k.startswith("static."):
            out["bounds"][k] = v.get("max")
        elif k.startswith("dynamics."):
            out.setdefault("dynamics_bounds", {})[k] = {b: v[b] for b in ("min", "max") if b in v}
    json.dump(out, open(os.path.join(HERE, "smoke_static.json"), "w"), indent=1, sort_keys=True)

    refdir = os.path.join(a.ref, "benchmarks", "smoke", "reference")
    lv = json.load(open(os.path.join(refdir, "lammps_values.json")))["systems"]["NiAlCo"]
    L, types, pos = read_lammps_data(os.path.join(refdir, "NiAlCo.data"))
    F = np.loadtxt(os.path.join(refdir, "NiAlCo_forces.dump"), skiprows=9)
    F = F[np.argsort(F[:, 0])][:, 1:]
    vir = np.array(lv["virial_bar_lammps_order_xx_yy_zz_xy_xz_yz"])[[0, 1, 2, 5, 4, 3]] / 1e4
    born = np.array(lv["born_matrix_eV_lammps_order"]) * NKTV2P / L**3 / 1e4
    np.savez_compressed(
        os.path.join(HERE, "nialco_lammps.npz"),
        L=L, types=types.astype(np.uint32), positions=np.mod(pos + L / 2, L) - L / 2,
        forces=F, epot=lv["epot_eV_per_atom"], virial=vir, born=born,
        elements=np.array(lv["elements"]), potential=lv["potential"])
    print("wrote", os.path.join(HERE, "smoke_static.json"), os.path.join(HERE, "nialco_lammps.npz"))


if __name__ == "__main__":
    main()
