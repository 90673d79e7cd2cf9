"""Runs the reference's statistical benchmarks Z1 (zn06_300K) and L1 (l12_cuzn3_5K) on the
GPU through mdelast_b200.benchmarks and checks every quantity against the reference's
published expectations (tests/golden/benchmarks_expected.json, from
make_benchmark_expected.py): |value - expected| <= tol, or the one-sided bounds of the
conserved-energy checks, and for L1 the NVT constants against the 0 K values within
0.2 %. Not collected by pytest (several minutes of GPU time per benchmark):

    python tests/benchmark_verify.py zn06_300K l12_cuzn3_5K --precision fp64 --out res.json

Exit status 0 only if no check fails."""

import argparse
import json
import math
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "mdelast_b200", "lib")):
    if p not in sys.path:
        sys.path.insert(0, p)
EXPECTED = os.path.join(ROOT, "tests", "golden", "benchmarks_expected.json")


def check(name, value, spec):
    """(status, message) of one quantity against its spec."""
    if value is None or not math.isfinite(value):
        return "FAIL", f"{name}: missing or non-finite"
    unit = spec.get("unit", "")
    if "info" in spec:
        ref = spec.get("expected")
        return "INFO", f"{name} = {value:.6g} {unit} (reference {ref:.6g}; not checked)" \
            if ref is not None else f"{name} = {value:.6g} {unit} (not checked)"
    if spec.get("expected") is not None and spec.get("tol") is not None:
        d = value - spec["expected"]
        ok = abs(d) <= spec["tol"]
        return ("PASS" if ok else "FAIL"), (
            f"{name} = {value:.6g} {unit}, expected {spec['expected']:.6g} +/- {spec['tol']:.3g}"
            f" ({abs(d) / spec['tol']:.2f} of tol)")
    lo, hi = spec.get("min", -math.inf), spec.get("max", math.inf)
    if lo == -math.inf and hi == math.inf:
        return "INFO", f"{name} = {value:.6g} {unit} (no bound)"
    ok = lo <= value <= hi
    return ("PASS" if ok else "FAIL"), f"{name} = {value:.6g} {unit}, bound [{lo:.3g}, {hi:.3g}]"


def verify(result, expected):
    rows = []
    for stage, st in expected["stages"].items():
        s = result[stage]
        for q, spec in st["quantities"].items():
            rows.append(check(f"{stage}.{q}", s.get(q), spec))
    zk = expected.get("zero_kelvin_reference")
    if zk:
        for q, ref in zk["values_GPa"].items():
            dev = (result["nvt"][q] - ref) / ref
            rows.append(check(f"nvt.{q} vs 0 K {ref} GPa (relative)", dev,
                              {"min": -zk["max_rel_deviation"], "max": zk["max_rel_deviation"]}))
    return rows


def main():
    import md_driver_module as m

    from mdelast_b200.benchmarks import run_benchmark
    from mdelast_b200.potentials import find_potential, read_setfl
    ap = argparse.ArgumentParser()
    ap.add_argument("benchmarks", nargs="+", choices=("zn06_300K", "l12_cuzn3_5K"))
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    exp = json.load(open(EXPECTED))
    t = read_setfl(find_potential("ZnCu.eam.alloy"))
    results, n_fail = {}, 0
    for name in a.benchmarks:
        r = run_benchmark(m, t, name, a.precision)
        rows = verify(r, exp[name])
        r["checks"] = rows
        results[name] = r
        print(f"== {name} ({a.precision}, {r['atoms']} atoms)", flush=True)
        for status, msg in rows:
            print(f"  {status:4}  {msg}", flush=True)
        n_fail += sum(1 for s, _ in rows if s == "FAIL")
    if a.out:
        with open(a.out, "w") as f:
            json.dump(results, f, indent=1)
    print("failed checks:", n_fail)
    sys.exit(1 if n_fail else 0)


if __name__ == "__main__":
    main()
