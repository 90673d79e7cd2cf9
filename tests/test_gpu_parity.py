"""GPU parity: the CUDA path against the oracle (the C restatement of the reference) on the
same inputs. FP64 mode; tolerance 1e-10 relative for forces and every observable, as the
target states; neighbour lists must be identical. These tests call the kernels through the
C-ABI (via the pybind11 module that wraps it)."""

import numpy as np
import pytest

from helpers import (dynamics_case, gpu, gpu_atoms, gpu_scalars, l12_case, nialco_case,
                     nialco_golden, oracle, rel_err, static_case, tables)

pytestmark = pytest.mark.gpu

TOL = 1e-10


def compare_state(g, o, tol, check_atoms=True):
    s_o = o.scalar_dict()
    s_g = gpu_scalars(g)
    for k in ["epot_eam_atom", "epot_atom", "ekin_atom", "etot_atom", "etot_cons",
              "total_laplacian", "total_force2", "temperature_kin", "temperature_conf_inverse",
              "pressure", "time", "cycle"]:
        assert rel_err(s_g[k], s_o[k]) <= tol, (k, s_g[k], s_o[k])
    for k in ["born_stress_tensor", "stress_tensor", "born_elasticity_tensor", "box"]:
        assert rel_err(s_g[k], s_o[k]) <= tol, (k, s_g[k], s_o[k])
    assert abs(s_g["baro_p_epsilon"] - s_o["baro_p_epsilon"]) <= tol * max(abs(s_o["baro_p_epsilon"]), 1e-300) + 1e-300
    if check_atoms:
        for f in ["forces", "velocities", "positions", "coordinates"]:
            assert rel_err(gpu_atoms(g, f), o.atoms(f)) <= tol, f
        for f in ["rho_eam", "energies_pot", "energies_kin"]:
            assert rel_err(gpu_atoms(g, f), o.atoms(f)) <= tol, f


def test_static_cell_matches_oracle():
    c = static_case()
    o = oracle(c)
    g = gpu(c)
    compare_state(g, o, TOL)
    # the upper triangle is stored, zeros below (run_smoke.py:217 relies on it)
    cb = np.array(g.born_elasticity_tensor)
    assert np.all(np.tril(cb, -1) == 0.0)


def test_static_cell_golden_values():
    """Benchmark S Part A6 golden values (smoke.json, quintic) at their rel 1e-7."""
    import json, os
    from mdelast_b200.units import Units as U
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "smoke_static.json")))
    g = gpu(static_case())
    CB = np.array(g.born_elasticity_tensor) / 1e10
    CB = np.where(CB == 0.0, CB.T, CB)
    vals = {
        "static_epot_eV_per_atom": g.epot_atom / U.ev,
        "static_pressure_GPa": g.pressure / 1e10,
        "static_CB11_GPa": np.mean([CB[0, 0], CB[1, 1], CB[2, 2]]),
        "static_CB12_GPa": np.mean([CB[0, 1], CB[0, 2], CB[1, 2]]),
        "static_CB44_GPa": np.mean([CB[3, 3], CB[4, 4], CB[5, 5]]),
        "laplacian_eV_A2": g.total_laplacian / (U.ev / U.angstrom**2),
        "static_T_conf_K": 1.0 / g.temperature_conf_inverse,
    }
    for k, v in vals.items():
        e = gold["quintic"][k]
        assert abs(v / e - 1.0) < 1e-7, (k, v, e)


@pytest.mark.parametrize("nside", [5, 8])
def test_neighbor_list_identical(nside):
    """The list of md_driver.cpp:279-298, entry for entry (5^3: all-pairs search;
    8^3: cell list)."""
    c = dynamics_case(nside=nside, n_zn=int(0.06 * 4 * nside**3))
    o = oracle(c)
    g = gpu(c)
    po, no = o.neighbors()
    pg, ng = g.neighbor_list()
    assert np.array_equal(np.asarray(pg), po)
    assert np.array_equal(np.asarray(ng), no)


@pytest.mark.parametrize("ensemble", [0, 1, 2])
def test_short_trajectory(ensemble):
    """20 steps of NVE / NVT / NPT with list rebuilds and alternating sampling."""
    c = dynamics_case(nside=5, ensemble=ensemble)
    o = oracle(c)
    g = gpu(c)
    for step in range(20):
        if step % 10 == 0:
            o.calculate_neighbors()
            g.calculate_neighbors()
        flag = step % 3 != 1
        o.set_sample_observables(flag)
        g.sample_observables = flag
        o.integrate()
        g.integrate()
    compare_state(g, o, 1e-9)
    for which in (0, 1):
        po, eo = o.chain(which)
        th = g.thermostat if which == 0 else g.barostat.thermostat
        assert rel_err(th.p_eta, po) < 1e-9
        assert rel_err(th.eta, eo) < 1e-9 or np.max(np.abs(eo)) == 0


@pytest.mark.parametrize("ensemble", [1, 2])
def test_chain_beyond_series_range(ensemble):
    """Chain momenta whose exponential arguments leave the branch-free series' range: the
    top link of both chains at 4e15 1/s (x = dt p/Q up to 2.6, so every half step is redone
    with the exact exponentials), the middle links at 2e14 1/s (x up to 0.13, inside the
    range). 10 steps against the oracle, which takes the library exp throughout."""
    import dataclasses
    c = dynamics_case(nside=5, ensemble=ensemble)
    T, q, p_eta, nf = c.thermo
    q = np.asarray(q)
    sign = np.where(np.arange(len(q)) % 2, 1.0, -1.0)
    v = np.full(len(q), 2e14)
    v[-1] = 4e15
    p = np.asarray(p_eta, float).copy()
    p[1:] = (sign * v * q)[1:]
    Tb, qb, _, nfb = c.baro_thermo
    qb = np.asarray(qb)
    vb = np.full(len(qb), 2e14)
    vb[-1] = 4e15
    c = dataclasses.replace(c, thermo=(T, list(q), list(p), nf),
                            baro_thermo=(Tb, list(qb), list(vb * qb), nfb))
    o = oracle(c)
    g = gpu(c)
    for _ in range(10):
        o.integrate()
        g.integrate()
    compare_state(g, o, 1e-9)
    for which in (0, 1):
        po, eo = o.chain(which)
        th = g.thermostat if which == 0 else g.barostat.thermostat
        assert rel_err(th.p_eta, po) < 1e-9
        assert rel_err(th.eta, eo) < 1e-9


def test_all_pairs_dynamics():
    """neighbors=False: every force call searches all pairs within the cutoff."""
    c = dynamics_case(nside=5, ensemble=1, neighbors=False, r_skin=1000.0)
    o = oracle(c)
    g = gpu(c)
    for _ in range(10):
        o.integrate()
        g.integrate()
    compare_state(g, o, 1e-9)


def test_l12_cell():
    """L1_2 CuZn3 at 5 K. The initial lattice is nearly perfect, so its forces are at the
    round-off level (|F|^2 ~ 1e-35 in cgs) and no relative comparison means anything; the
    comparison is made after 10 steps, when every atom has a thermal force."""
    c = l12_case(n=4)
    o = oracle(c)
    g = gpu(c)
    o.integrate(10)
    g.integrate_n(10)
    compare_state(g, o, 1e-9)


def test_ternary_cell():
    """Ni-Al-Co 500-atom cell of benchmark S Part C against the oracle and, at the
    benchmark's own bounds (smoke.json:90-113), against the stored LAMMPS values."""
    from mdelast_b200.units import Units as U
    c = nialco_case()
    o = oracle(c)
    g = gpu(c)
    compare_state(g, o, TOL)
    ref = nialco_golden()
    F = gpu_atoms(g, "forces") / (U.ev / U.angstrom)
    assert abs(g.epot_atom / U.ev - float(ref["epot"])) < 1e-10
    assert np.max(np.abs(F - ref["forces"])) < 2e-6
    vir = -np.array(g.born_stress_tensor) / 1e10
    assert np.max(np.abs(vir - ref["virial"])) < 1e-5
    CB = np.array(g.born_elasticity_tensor) / 1e10
    order = [(0, 0), (1, 1), (2, 2), (3, 3), (4, 4), (5, 5), (0, 1), (0, 2), (0, 3), (0, 4),
             (0, 5), (1, 2), (1, 3), (1, 4), (1, 5), (2, 3), (2, 4), (2, 5), (3, 4), (3, 5),
             (4, 5)]
    born = np.array([CB[i, j] for i, j in order])
    assert np.max(np.abs(born - ref["born"])) < 4e-3
