"""The reference's two statistical benchmarks run on the device, with the quantities its
verification reads.

Z1 (sample_case/run.py:218-300) is the 5x5x5 Cu-Zn cell (500 atoms, 30 Zn placed by
RandomState(42)) at 300 K, L1 (benchmarks/l12_cuzn3_5K/run.py) the 20x20x20 ordered L1_2
CuZn3 cell (32,000 atoms) at 5 K. Both run
an NPT stage at zero pressure and an NVT stage in the NPT production-mean box, each of
50,000 thermalisation and 100,000 production steps at dt = 2 fs, tau_T = 50 fs,
tau_P = 500 fs, neighbour list r_skin 1.2 rebuilt every 20 steps, observables every step,
with the scripts' seeds (NPT velocities 0; NVT 0 for Z1, 500 for L1) and the scripts'
handoff (the final NPT positions scaled by the production-mean (V/V0)^(1/3), wrapped into
the mean box).

`summarize_stage` returns, for one stage, what benchmarks/bench_lib.py:46-106 reads from a
run's series file: the cubic averages of the total constants C, the Born term CB, the
stress-fluctuation term fluc and the ideal-gas term kin (C = CB - fluc + kin [+ K in NPT],
molecular_dynamics.py:826-958), the NPT bulk-modulus term K_npt, the production means of
T_kin, pressure and L/L0, the configurational temperature both as 1/<1/T_conf> and as
<T_conf>, and the conserved-energy checks (largest |E_cons(t)/E_cons(0) - 1| over the
stage, slope of E_cons(t)/E_cons(0) - 1 over the production window per ns). The samples
stay on the device (the sample ring and the fluctuation sums); the host drains the ring
once per 1,024 steps.

    python -m mdelast_b200.benchmarks zn06_300K --precision fp64 --out z1.json
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .protocol import RING, _nvt_cells
from .systems import Cell, cuzn_cell, l12_cell, make_batch
from .units import Units as U

CUBIC = {"11": ((0, 0), (1, 1), (2, 2)), "12": ((0, 1), (0, 2), (1, 2)),
         "44": ((3, 3), (4, 4), (5, 5))}

BENCHMARKS = {
    # name: (cell builder, NVT velocity seed)
    "zn06_300K": (lambda t: cuzn_cell(t, 5, n_zn=30, T=300.0, ensemble=2, placement_seed=42,
                                      velocity_seed=0), 0),
    "l12_cuzn3_5K": (lambda t: l12_cell(t, 20, T=5.0, ensemble=2, velocity_seed=0), 500),
}


def _cubic(M, key):
    return float(np.mean([M[i, j] for i, j in CUBIC[key]]))


def summarize_stage(b, cell: Cell, n_therm: int, n_prod: int, rebuild_every: int = 20,
                    log=None) -> dict:
    """Runs one stage of n_therm + n_prod steps of replica 0 of batch `b` (sampled every
    step) and returns its benchmark quantities; the fluctuation sums start with the
    production window."""
    V0 = float(np.prod(cell.box))
    econs, t_s, done, total = [], [], 0, n_therm + n_prod
    sums = {"T_kin": 0., "inv_tconf": 0., "tconf": 0., "pressure": 0., "L_L0": 0., "V_V0": 0.}
    n_prod_samples = 0
    t0 = time.perf_counter()
    while done < total:
        if done == n_therm:
            b.fluctuation_start()
        k = min(RING, (n_therm - done) if done < n_therm else total - done)
        b.run(k, rebuild_every, 1, False)
        rec = b.drain_samples(0)
        econs.append(np.asarray(rec["etot_cons"], float))
        t_s.append(np.asarray(rec["time"], float))
        if done >= n_therm:
            inv = np.asarray(rec["temperature_conf_inverse"], float)
            vv = np.asarray(rec["volume"], float) / V0
            sums["T_kin"] += float(np.sum(rec["temperature_kin"]))
            sums["inv_tconf"] += float(np.sum(inv))
            sums["tconf"] += float(np.sum(1.0 / inv))
            sums["pressure"] += float(np.sum(rec["pressure"]))
            sums["L_L0"] += float(np.sum(vv ** (1.0 / 3.0)))
            sums["V_V0"] += float(np.sum(vv))
            n_prod_samples += len(inv)
        done += k
        if log and done % (50 * RING) < RING:
            log(f"  {done}/{total} steps, {time.perf_counter() - t0:.1f} s")
    econs = np.concatenate(econs)
    t_s = np.concatenate(t_s)
    rel = econs / econs[0] - 1.0
    n0 = len(econs) - n_prod_samples
    n = max(n_prod_samples, 1)
    out = {"n_steps": total, "n_thermalization": n_therm,
           "T_kin": sums["T_kin"] / n,
           "T_conf_recip": n / sums["inv_tconf"],
           "T_conf_sample": sums["tconf"] / n,
           "pressure": sums["pressure"] / n / U.GPa,
           "L_L0": sums["L_L0"] / n, "V_V0": sums["V_V0"] / n,
           "econs_err_max": float(np.max(np.abs(rel))),
           "econs_drift_per_ns": float(np.polyfit(t_s[n0:] * 1e9, rel[n0:], 1)[0])}
    out["econs_drift_abs_per_ns"] = abs(out["econs_drift_per_ns"])
    ec = b.elastic_constants(0)
    fl = b.fluctuations(0)
    C = np.asarray(ec["C"]) / U.GPa
    CB = np.asarray(fl["born_el_mean"]) / U.GPa
    kT = U.k_boltz * cell.T
    rho = float(fl["mean"][6])
    kin = np.zeros((6, 6))
    for i in range(6):
        kin[i, i] = (2.0 if i < 3 else 1.0) * rho * kT / U.GPa
    K = float(ec["bulk_modulus"]) / U.GPa
    bulk = np.zeros((6, 6))
    bulk[:3, :3] = K
    CBs = CB + np.triu(CB, 1).T  # the Born mean is stored as its upper triangle
    fluc = CBs + kin + bulk - C
    for key in CUBIC:
        out["C" + key] = _cubic(C, key)
        out["CB" + key] = _cubic(CBs, key)
        out["fluc" + key] = _cubic(fluc, key)
    out["kin11"] = _cubic(kin, "11")
    out["kin44"] = _cubic(kin, "44")
    out["K_npt"] = K
    out["cubic_spread_C11"] = float(np.ptp(np.diag(C)[:3]))
    out["wall_s"] = time.perf_counter() - t0
    return out


def run_benchmark(m, tables, name: str, precision: str = "fp64", n_therm: int = 50_000,
                  n_prod: int = 100_000, handoff: str = "reference", log=None) -> dict:
    """Both stages of benchmark `name` ("zn06_300K" or "l12_cuzn3_5K")."""
    build, nvt_seed = BENCHMARKS[name]
    cell = build(tables)
    b = make_batch(m, tables, [cell], r_skin=1.2, precision=precision)
    b.autotune(2)
    npt = summarize_stage(b, cell, n_therm, n_prod, log=log)
    snap = [(np.asarray(b.atoms(0, m.ATOM_POSITIONS)), np.asarray(b.atoms(0, m.ATOM_VELOCITIES)),
             b.chain(0, 0)[1])]
    crd = [np.asarray(b.atoms(0, m.ATOM_COORDINATES))]
    del b
    (nvt_cell,) = _nvt_cells(tables, [cell], snap, crd, [npt["V_V0"]], [nvt_seed], handoff)
    b = make_batch(m, tables, [nvt_cell], r_skin=1.2, precision=precision)
    b.autotune(2)
    nvt = summarize_stage(b, nvt_cell, n_therm, n_prod, log=log)
    del b
    return {"benchmark": name, "precision": precision, "handoff": handoff,
            "atoms": cell.n_atoms, "npt": npt, "nvt": nvt}


def _main():
    import md_driver_module as m

    from .potentials import find_potential, read_setfl
    ap = argparse.ArgumentParser()
    ap.add_argument("benchmark", choices=sorted(BENCHMARKS))
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--therm", type=int, default=50_000)
    ap.add_argument("--prod", type=int, default=100_000)
    ap.add_argument("--handoff", choices=("reference", "box"), default="reference")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    t = read_setfl(find_potential("ZnCu.eam.alloy"))
    r = run_benchmark(m, t, a.benchmark, a.precision, a.therm, a.prod, a.handoff, log=print)
    s = json.dumps(r, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s)
    print(s)


if __name__ == "__main__":
    _main()
