"""Host side of the elastic-constant protocol: the NVT cells built at the NPT -> NVT
handoff (sample_case/run.py:251-285), and the time-to-accuracy reading of checkpoints."""

import numpy as np

from mdelast_b200.dump import handoff_positions
from mdelast_b200.protocol import ProtocolResult, Stages, _nvt_cells, time_to_within
from mdelast_b200.systems import Cell


class _Tables:
    masses = [1.0e-22, 1.1e-22]


def _cell(n=8, L=10e-8):
    rng = np.random.default_rng(1)
    return Cell(positions=(rng.random((n, 3)) - 0.5) * L, velocities=np.zeros((n, 3)),
                types=np.array([0, 1] * (n // 2), np.uint32), box=np.array([L, L, L]),
                T=300.0, ensemble=2, thermo_q=np.ones(10), thermo_p_eta=np.zeros(10),
                baro_q=np.ones(10), baro_p_eta=np.zeros(10), baro_w=1.0, baro_p_eps=0.0,
                Nf=21.0)


def test_box_handoff_places_snapshot_coordinates_in_mean_box():
    c = _cell()
    u = np.random.default_rng(2).random((8, 3)) * 3 - 1.5  # unwrapped scaled coordinates
    snap = [(np.zeros((8, 3)), np.ones((8, 3)), [0.5] * 10)]
    V_V0 = 1.03
    (nv,) = _nvt_cells(_Tables, [c], snap, [u], [V_V0], [7], "box")
    L = c.box * V_V0 ** (1 / 3)
    assert np.allclose(nv.box, L, rtol=1e-15)
    w = nv.positions / L
    assert np.all(np.abs(w) < 0.5)
    assert np.allclose(w - u, np.round(w - u), atol=1e-12)  # same point modulo the box
    assert nv.ensemble == 1 and not np.array_equal(nv.velocities, snap[0][1])


def test_continue_handoff_carries_velocities_and_chain():
    c = _cell()
    snap = [(np.zeros((8, 3)), np.full((8, 3), 3.0), [0.25] * 10)]
    (nv,) = _nvt_cells(_Tables, [c], snap, [np.zeros((8, 3))], [1.0], [7], "continue")
    assert np.array_equal(nv.velocities, snap[0][1])
    assert np.array_equal(nv.thermo_p_eta, snap[0][2])


def test_reference_handoff_is_the_scripts_arithmetic():
    c = _cell()
    p = c.positions * 1.01
    (nv,) = _nvt_cells(_Tables, [c], [(p, None, None)], [None], [1.0303], [7], "reference")
    assert np.array_equal(nv.positions, handoff_positions(p, 1.0303)[0])


def test_time_to_within_needs_to_stay_inside():
    target = {"C11": 100.0, "C12": 50.0, "C44": 40.0}
    r = ProtocolResult("fp64", 1, 8, Stages(), [1.0], [0.0], target, [target],
                       checkpoints=[(1, 1.0, 101, 50, 40), (2, 2.0, 110, 50, 40),
                                    (3, 3.0, 101.5, 50.5, 40.2), (4, 4.0, 100, 50, 40)])
    assert time_to_within(r, target) == 3.0
    assert time_to_within(r, target, tol=0.001) == 4.0
    r.checkpoints.append((5, 5.0, 90, 50, 40))
    assert time_to_within(r, target) is None
