"""Benchmark S's consistency checks (``benchmarks/smoke/run_smoke.py``, bounds in
``benchmarks/expected/smoke.json``) restated on the GPU path, in FP64 and in mixed
precision.

Part A, on the fixed distorted 256-atom Cu-Zn cell (all-pairs force calls):
  A1 net force; A2 forces against central differences of the energy (16 atoms, 3
  directions, step 1e-4 A); A3 Born stress against dU/deta (strain step 1e-4); A4 Born
  constants against differences of the Born stress (strain step 1e-5); A5 the Laplacian
  against differences of the forces (every atom and direction, step 1e-4 A).
Part B, on the 500-atom 6 at.% Zn cell at 300 K from MolecularDynamics' initial state:
  NVE at dt 2 fs (1,000 steps) and 1 fs (2,000 steps), the conserved-energy error and the
  ratio of their second-half rms (dt^2 scaling); NVT and NPT at 2 fs (2,000 steps, the last
  1,000 averaged), conserved-energy error and the kinetic and configurational temperatures.

Every perturbed cell is one replica of a BatchedMDDriver, so each part is one construction.

FP64 must meet every smoke.json bound (and reproduces the reference's own observed values
to 3-4 digits). In mixed precision positions and pair terms are FP32: a pair distance is
rounded to ~2.4e-7 A at 2.5 A, so a finite-difference step of 1e-4 A spans only a few
hundred of its rounding steps, and the rounding of the two evaluated configurations does not
cancel. At the smoke's steps the differences then measure that rounding, not the
derivative (A2 would need the total energy to 1e-9 eV), and no step size brings FP32
energies under A2's bound. The mixed path meets the smoke bounds of A1 and Part B, and for
A2-A5 it is held to ten times what it measured on a B200 when this test was written (A2
3.7e-3 eV/A, A3 3.8e-4 GPa, A4 0.13 GPa, A5 2.7e-5): a guard against regressions of the
mixed path, with the measured values reported beside the FP64 ones.
"""

import json
import os

import numpy as np
import pytest

from helpers import dynamics_case, gpu, tables
from mdelast_b200.lattice import smoke_static_cell
from mdelast_b200.systems import Cell, make_batch
from mdelast_b200.units import Units as U

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "smoke_static.json")))
BOUNDS = GOLD["bounds"]
DYN = GOLD["dynamics_bounds"]
H_POS, H_STRAIN, H_STRAIN_BORN, N_FORCE_ATOMS = 1e-4, 1e-4, 1e-5, 16
MIXED_A = {"static.force_fd_max_abs_err_eV_A": 3.7e-2,
           "static.born_stress_fd_max_abs_err_GPa": 3.8e-3,
           "static.born_C_fd_max_abs_err_GPa": 1.3, "static.laplacian_fd_rel_err": 2.7e-4}
REPORT = {}


def _cell(pos_cm, types, lengths_cm):
    n = len(pos_cm)
    L = np.asarray(lengths_cm, dtype=float)
    pos = np.mod(pos_cm + L / 2, L) - L / 2
    return Cell(positions=pos, velocities=np.zeros_like(pos), types=np.asarray(types, np.uint32),
                box=L, T=300.0, ensemble=0, thermo_q=np.array([1e-30]),
                thermo_p_eta=np.array([0.0]), baro_q=np.array([1e-30]),
                baro_p_eta=np.array([0.0]), baro_w=1e-30, baro_p_eps=0.0, Nf=3.0 * n,
                pressure=0.0)


def _batch(t, cells, precision):
    import md_driver_module as m
    return make_batch(m, t, cells, dt=1e-15, neighbors=False, r_skin=1.0, precision=precision)


def part_a(precision):
    import md_driver_module as m
    t = tables()
    names = [e[0] for e in t.elements]
    pos0, types, Lc = smoke_static_cell(names)
    N = len(pos0)
    L = np.full(3, Lc)
    V = float(np.prod(L))
    ev_a = U.ev / U.angstrom
    hc = H_POS * U.angstrom
    res = {}
    # base cell, A2 and A3/A4 perturbations in one batch
    cells = [_cell(pos0, types, L)]
    atoms = np.random.RandomState(1).choice(N, size=N_FORCE_ATOMS, replace=False)
    for i in atoms:
        for a in range(3):
            for s in (1, -1):
                p = pos0.copy()
                p[i, a] += s * hc
                cells.append(_cell(p, types, L))
    strains = []
    for h in (H_STRAIN, H_STRAIN_BORN):
        for a in range(3):
            for s in (1, -1):
                eta = np.zeros(3)
                eta[a] = s * h
                lam = np.sqrt(1.0 + 2.0 * eta)
                strains.append(lam)
                cells.append(_cell(pos0 * lam, types, L * lam))
    b = _batch(t, cells, precision)
    obs = [b.observables(r) for r in range(b.n_replicas)]
    E = np.array([o["epot_atom"] * N for o in obs])
    F0 = np.asarray(b.atoms(0, m.ATOM_FORCES))
    res["net_force_rel"] = float(np.abs(F0.sum(0)).max() / np.abs(F0).max())
    fd, an = [], []
    k = 1
    for i in atoms:
        for a in range(3):
            fd.append(-(E[k] - E[k + 1]) / (2 * hc))
            an.append(F0[i, a])
            k += 2
    fd, an = np.array(fd), np.array(an)
    res["force_fd_max_abs_err_eV_A"] = float(np.abs(fd - an).max() / ev_a)
    # A3: (1/V) dU/deta_a
    born0 = np.array(obs[0]["born_stress_tensor"])[:3]
    ds = np.array([(E[k + 2 * a] - E[k + 2 * a + 1]) / (2 * H_STRAIN) / V for a in range(3)])
    res["born_stress_fd_max_abs_err_GPa"] = float(np.abs(ds - born0).max() / 1e10)
    k += 6
    # A4: C^B_ab = (1/V0) d T_a / d eta_b with T_a = V(eta) sigma^B_a(eta) / lambda_a^2
    CB = np.array(obs[0]["born_elasticity_tensor"])
    CB = np.where(CB == 0.0, CB.T, CB)
    M = np.zeros((3, 3))
    for bb in range(3):
        tp = []
        for s in range(2):
            r = k + 2 * bb + s
            lam = strains[6 + 2 * bb + s]
            tp.append(V * np.prod(lam) * np.array(obs[r]["born_stress_tensor"])[:3] / lam**2)
        M[:, bb] = (tp[0] - tp[1]) / (2 * H_STRAIN_BORN) / V
    M = 0.5 * (M + M.T)
    pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
    res["born_C_fd_max_abs_err_GPa"] = float(max(abs(CB[a, c] - M[a, c]) for a, c in pairs) / 1e10)
    lap_an = float(obs[0]["total_laplacian"])
    del b
    # A5: the Laplacian from differences of the forces, every atom and direction
    cells = []
    for i in range(N):
        for a in range(3):
            for s in (1, -1):
                p = pos0.copy()
                p[i, a] += s * hc
                cells.append(_cell(p, types, L))
    b = _batch(t, cells, precision)
    lap = 0.0
    r = 0
    for i in range(N):
        for a in range(3):
            fp = np.asarray(b.atoms(r, m.ATOM_FORCES))[i, a]
            fm = np.asarray(b.atoms(r + 1, m.ATOM_FORCES))[i, a]
            lap += -(fp - fm) / (2 * hc)
            r += 2
    del b
    res["laplacian_fd_rel_err"] = float(abs(lap - lap_an) / abs(lap_an))
    return res


def _run_records(g, n):
    """n steps with the list every 20 steps and observables every step; the per-step
    records of the run (the sample ring drained every 1,000 steps)."""
    out = {"etot_cons": [], "temperature_kin": [], "temperature_conf_inverse": []}
    done = 0
    while done < n:
        k = min(1000, n - done)
        g.run(k, 20, 1, False)
        rec = g.drain_samples()
        assert rec["lost"] == 0
        for key in out:
            out[key].extend(rec[key])
        done += k
    return {k: np.asarray(v) for k, v in out.items()}


def dynamics(precision, ensemble, dt_fs, n_th, n_prod):
    c = dynamics_case(nside=5, n_zn=30, ensemble=ensemble, dt=dt_fs * 1e-15)
    g = gpu(c, precision=precision)
    # n_th + n_prod + 1 steps, each recorded, as run_smoke.py's loops and run() record them
    rec = _run_records(g, n_th + n_prod + 1)
    econs = rec["etot_cons"]
    rel = econs / econs[0] - 1.0
    half = rel[len(rel) // 2:]
    return {"econs_err_max": float(np.abs(rel).max()),
            "econs_err_rms_second_half": float(np.sqrt(np.mean((half - half.mean()) ** 2))),
            "T_kin": float(np.mean(rec["temperature_kin"][n_th:])),
            "T_conf_recip": float(1.0 / np.mean(rec["temperature_conf_inverse"][n_th:]))}


def part_b(precision):
    out = {"nve_dt2": dynamics(precision, 0, 2.0, 500, 500),
           "nve_dt1": dynamics(precision, 0, 1.0, 1000, 1000),
           "nvt": dynamics(precision, 1, 2.0, 1000, 1000),
           "npt": dynamics(precision, 2, 2.0, 1000, 1000)}
    out["nve_dt_ratio"] = (out["nve_dt2"]["econs_err_rms_second_half"]
                           / out["nve_dt1"]["econs_err_rms_second_half"])
    return out


def _check_b(res):
    for key, b in DYN.items():
        path = key.split(".")[1:]
        v = res
        for p in path:
            v = v[p]
        if "max" in b:
            assert v <= b["max"], (key, v, b)
        if "min" in b:
            assert v >= b["min"], (key, v, b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_part_a(precision):
    res = part_a(precision)
    REPORT.setdefault(precision, {})["static"] = res
    print(precision, json.dumps(res))
    for key, bound in BOUNDS.items():
        if not key.startswith("static."):
            continue
        name = key[len("static."):]
        if precision == "mixed" and key in MIXED_A:
            bound = MIXED_A[key]
        assert res[name] <= bound, (precision, name, res[name], bound)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_part_b(precision):
    res = part_b(precision)
    REPORT.setdefault(precision, {})["dynamics"] = res
    print(precision, json.dumps(res))
    _check_b(res)
    out = os.environ.get("MDELAST_SMOKE_REPORT")
    if out:
        with open(out, "w") as fh:
            json.dump(REPORT, fh, indent=1)
