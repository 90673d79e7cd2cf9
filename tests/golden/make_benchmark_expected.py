"""Writes tests/golden/benchmarks_expected.json: the expected values and tolerances of the
reference's two statistical benchmarks, read as data from its published expectation
files (benchmarks/expected/zn06_300K.json and l12_cuzn3_5K.json): Z1, Cu-6 at.% Zn at
300 K, and L1, L1_2 CuZn3 at 5 K, each an NPT stage then an NVT stage of 50,000 + 100,000
steps. Per quantity it keeps the check itself ("expected" with "tol", or the one-sided
"max" / "min", or "info" for report-only values), the unit, and the reference run's own
standard error and velocity-replica spread where given. The reference checkout is
``$MDELAST_REFERENCE`` or a checkout called ``reference`` beside this repository."""

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
KEEP = ("expected", "tol", "max", "min", "info", "unit", "se_run", "s_vel")


def main():
    import sys
    sys.path.insert(0, HERE)
    from refroot import reference_root
    REF = reference_root(sys.argv[1] if len(sys.argv) > 1 else None)
    out = {}
    for name in ("zn06_300K", "l12_cuzn3_5K"):
        d = json.load(open(os.path.join(REF, "benchmarks", "expected", name + ".json")))
        b = {"rule": d["rule"], "stages": {}}
        for stage, st in d["stages"].items():
            b["stages"][stage] = {
                "n_steps": st["n_steps"], "n_thermalization": st["n_thermalization"],
                "quantities": {q: {k: v for k, v in spec.items() if k in KEEP}
                               for q, spec in st["quantities"].items()}}
        if "zero_kelvin_reference" in d:
            zk = d["zero_kelvin_reference"]
            b["zero_kelvin_reference"] = {"values_GPa": zk["values_GPa"],
                                          "max_rel_deviation": zk["max_rel_deviation"]}
        out[name] = b
    path = os.path.join(HERE, "benchmarks_expected.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
