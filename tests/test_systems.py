"""Cell builders of mdelast_b200.systems on the CPU: the random FCC alloy's site counts and
placement, and the chain masses set for a temperature other than the target."""

import numpy as np

from helpers import tables
from mdelast_b200.systems import fcc_alloy_cell
from mdelast_b200.units import Units as U


def test_fcc_alloy_counts_and_placement():
    t = tables("Mishin_updated-Ni-Al-Co-2013.eam.alloy")
    x = (0.5, 0.3, 0.2)
    c = fcc_alloy_cell(t, 4, x, T=300.0, a_ang=3.6, placement_seed=5)
    n = 4 * 4**3
    assert c.n_atoms == n and sum(c.meta["counts"]) == n
    assert c.meta["counts"][:2] == [round(0.5 * n), round(0.3 * n)]
    assert np.bincount(c.types, minlength=3).tolist() == c.meta["counts"]
    c2 = fcc_alloy_cell(t, 4, x, T=300.0, a_ang=3.6, placement_seed=5)
    assert np.array_equal(c.types, c2.types)
    c3 = fcc_alloy_cell(t, 4, x, T=300.0, a_ang=3.6, placement_seed=6)
    assert not np.array_equal(c.types, c3.types)
    assert np.allclose(c.box, 4 * 3.6 * U.angstrom)


def test_chain_masses_for_another_temperature():
    t = tables("Mishin_updated-Ni-Al-Co-2013.eam.alloy")
    x = (0.4, 0.2, 0.4)
    cold = fcc_alloy_cell(t, 4, x, T=6.0, a_ang=3.6, velocity_seed=3)
    floor = fcc_alloy_cell(t, 4, x, T=6.0, a_ang=3.6, velocity_seed=3, mass_T=50.0)
    # masses proportional to kT: set for 50 K they are 50/6 times heavier
    assert np.allclose(floor.thermo_q / cold.thermo_q, 50.0 / 6.0)
    assert np.isclose(floor.baro_w / cold.baro_w, 50.0 / 6.0)
    # the velocities and the thermostat target stay those of 6 K
    assert np.array_equal(floor.velocities, cold.velocities)
    assert floor.T == cold.T == 6.0
