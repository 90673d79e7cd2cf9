"""The oracle (C restatement, oracle/mdelast_oracle.c) pinned two ways, on the CPU:
bit for bit against the reference's own C++ core compiled in place (oracle/_ref), and
against the golden values the reference's benchmark S stores (smoke.json)."""

import json
import os

import numpy as np
import pytest

from helpers import dynamics_case, l12_case, nialco_case, nialco_golden, oracle, static_case
from mdelast_b200.units import Units as U
from oracle import ref

needs_ref = pytest.mark.skipif(not ref.available("ref"), reason="oracle/_ref not built")
needs_oracle = pytest.mark.skipif(not ref.available("oracle"), reason="oracle not built")

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "smoke_static.json")))


def a6_values(d):
    s = d.scalar_dict()
    CB = s["born_elasticity_tensor"] / 1e10
    CB = np.where(CB == 0.0, CB.T, CB)
    return {
        "static_epot_eV_per_atom": s["epot_atom"] / U.ev,
        "static_pressure_GPa": s["pressure"] / 1e10,
        "static_CB11_GPa": np.mean([CB[0, 0], CB[1, 1], CB[2, 2]]),
        "static_CB12_GPa": np.mean([CB[0, 1], CB[0, 2], CB[1, 2]]),
        "static_CB44_GPa": np.mean([CB[3, 3], CB[4, 4], CB[5, 5]]),
        "laplacian_eV_A2": s["total_laplacian"] / (U.ev / U.angstrom**2),
        "static_T_conf_K": 1.0 / s["temperature_conf_inverse"],
    }


@needs_oracle
def test_oracle_static_golden():
    """Benchmark S Part A6 (smoke.json:34-88, quintic) within its rel 1e-7."""
    vals = a6_values(oracle(static_case()))
    for k, v in vals.items():
        assert abs(v / GOLD["quintic"][k] - 1.0) < GOLD["rel_tol"], k


@needs_oracle
def test_oracle_net_force():
    """Part A1: the net force vanishes (smoke.json bound 1e-12 relative)."""
    F = oracle(static_case()).atoms("forces")
    assert np.abs(F.sum(0)).max() / np.abs(F).max() < 1e-12


@needs_oracle
def test_oracle_ternary_vs_lammps():
    """Part C: Ni-Al-Co cell against the stored LAMMPS values at smoke.json:90-113."""
    d = oracle(nialco_case())
    g = nialco_golden()
    s = d.scalar_dict()
    assert abs(s["epot_atom"] / U.ev - float(g["epot"])) < 1e-10
    F = d.atoms("forces") / (U.ev / U.angstrom)
    assert np.max(np.abs(F - g["forces"])) < 2e-6
    assert np.max(np.abs(-s["born_stress_tensor"] / 1e10 - g["virial"])) < 1e-5


@needs_ref
@needs_oracle
@pytest.mark.parametrize("maker", [static_case, nialco_case])
def test_oracle_bitwise_static(maker):
    c = maker()
    a, b = oracle(c, "ref"), oracle(c, "oracle")
    assert np.array_equal(a.scalars(), b.scalars())
    for f in ("forces", "energies_pot", "rho_eam"):
        assert np.array_equal(a.atoms(f), b.atoms(f))


@needs_ref
@needs_oracle
@pytest.mark.parametrize("ensemble", [0, 1, 2])
def test_oracle_bitwise_dynamics(ensemble):
    """30 steps NVE/NVT/NPT with list rebuilds and sampling toggled: bit-identical."""
    c = dynamics_case(nside=5, ensemble=ensemble)
    a, b = oracle(c, "ref"), oracle(c, "oracle")
    for step in range(30):
        if step % 20 == 0:
            a.calculate_neighbors()
            b.calculate_neighbors()
        a.set_sample_observables(step % 3 != 0)
        b.set_sample_observables(step % 3 != 0)
        a.integrate()
        b.integrate()
    assert np.array_equal(a.scalars(), b.scalars())
    for f in ("positions", "coordinates", "velocities", "forces"):
        assert np.array_equal(a.atoms(f), b.atoms(f))
    for w in (0, 1):
        for x, y in zip(a.chain(w), b.chain(w)):
            assert np.array_equal(x, y)
    pa, na = a.neighbors()
    pb, nb = b.neighbors()
    assert np.array_equal(pa, pb) and np.array_equal(na, nb)


@needs_ref
@needs_oracle
def test_oracle_bitwise_configurational_coupling():
    c = dynamics_case(nside=4, n_zn=15, ensemble=1, coupling=2)
    a, b = oracle(c, "ref"), oracle(c, "oracle")
    a.integrate(15)
    b.integrate(15)
    assert np.array_equal(a.scalars(), b.scalars())


@needs_ref
@needs_oracle
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_oracle_bitwise_pair_correlation(mode):
    c = dynamics_case(nside=4, n_zn=15)
    a, b = oracle(c, "ref"), oracle(c, "oracle")
    ga, gpa = a.pair_correlation(mode)
    gb, gpb = b.pair_correlation(mode)
    assert np.array_equal(ga, gb) and np.array_equal(gpa, gpb)


@needs_ref
@needs_oracle
def test_oracle_bitwise_l12():
    c = l12_case(n=3)
    a, b = oracle(c, "ref"), oracle(c, "oracle")
    a.integrate(5)
    b.integrate(5)
    assert np.array_equal(a.scalars(), b.scalars())


@needs_ref
@pytest.mark.parametrize("which", ["ref", "oracle"])
def test_bspline_static_golden(which):
    """Benchmark S Part A6 with the "bspline" tables of versions <= 1.1 (smoke.json:34-88,
    bspline column) within its rel 1e-7: the compiled reference through the project's
    cubic B-spline shim, and the C restatement."""
    from dataclasses import replace
    vals = a6_values(oracle(replace(static_case(), interpolation="bspline"), which))
    for k, v in vals.items():
        assert abs(v / GOLD["bspline"][k] - 1.0) < GOLD["rel_tol"], k


@needs_ref
@needs_oracle
@pytest.mark.parametrize("maker", ["static", "npt"])
def test_oracle_bitwise_bspline(maker):
    from dataclasses import replace
    c = static_case() if maker == "static" else dynamics_case(nside=4, n_zn=15, ensemble=2)
    c = replace(c, interpolation="bspline")
    a, b = oracle(c, "ref"), oracle(c, "oracle")
    a.integrate(10)
    b.integrate(10)
    assert np.array_equal(a.scalars(), b.scalars())
    assert np.array_equal(a.atoms("forces"), b.atoms("forces"))


@needs_ref
@needs_oracle
def test_oracle_bitwise_cu01():
    """Pure Cu with the single-element 10,000-node Cu01 tables (the pure-Cu example):
    a displaced static cell and 20 NVT steps with a list rebuild, bit-identical."""
    from helpers import cu01_case
    c = cu01_case(sigma_ang=0.08)
    a, b = oracle(c, "ref"), oracle(c, "oracle")
    assert np.array_equal(a.scalars(), b.scalars())
    assert np.array_equal(a.atoms("forces"), b.atoms("forces"))
    c = cu01_case()
    a, b = oracle(c, "ref"), oracle(c, "oracle")
    for step in range(20):
        if step % 10 == 0:
            a.calculate_neighbors()
            b.calculate_neighbors()
        a.integrate()
        b.integrate()
    assert np.array_equal(a.scalars(), b.scalars())
    for f in ("positions", "velocities", "forces"):
        assert np.array_equal(a.atoms(f), b.atoms(f))
