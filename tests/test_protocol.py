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
    c = _cell(n=64)
    p = c.positions * 1.05  # a snapshot in a box 5 % larger than the mean box
    (nv,) = _nvt_cells(_Tables, [c], [(p, None, None)], [None], [1.0303], [7], "reference")
    q = handoff_positions(p, 1.0303)[0]
    L = nv.box
    inside = np.all(np.abs(q) < 0.5 * L, axis=1)
    assert inside.any() and not inside.all()
    # scaled positions kept where inside the mean box, wrapped by one edge where not
    assert np.array_equal(nv.positions[inside], q[inside])
    out = ~inside
    assert np.allclose(nv.positions[out], q[out] - L * np.round(q[out] / L), rtol=0, atol=1e-20)
    assert np.all(nv.positions >= -0.5 * L) and np.all(nv.positions < 0.5 * L)


def test_time_to_within_needs_to_stay_inside():
    target = {"C11": 100.0, "C12": 50.0, "C44": 40.0}
    r = ProtocolResult("fp64", 1, 8, Stages(), [1.0], [0.0], target, [target],
                       checkpoints=[(1, 1.0, 101, 50, 40), (2, 2.0, 110, 50, 40),
                                    (3, 3.0, 101.5, 50.5, 40.2), (4, 4.0, 100, 50, 40)])
    assert time_to_within(r, target) == 3.0
    assert time_to_within(r, target, tol=0.001) == 4.0
    r.checkpoints.append((5, 5.0, 90, 50, 40))
    assert time_to_within(r, target) is None


def test_continue_handoff_keeps_the_npt_thermostat_masses():
    c = _cell()
    c.thermo_q = np.full(10, 7.0)  # masses of the NPT stage (e.g. set for a floor temperature)
    snap = [(np.zeros((8, 3)), np.ones((8, 3)), [0.25] * 10)]
    (nv,) = _nvt_cells(_Tables, [c], snap, [np.zeros((8, 3))], [1.0], [7], "continue")
    assert np.array_equal(nv.thermo_q, c.thermo_q)


class _FakeBatch:
    """A batch whose window pressure follows p = -3 B (L / L_eq - 1) per replica; it
    records the boxes it was built with."""
    B_GPa = 200.0
    built = []

    def __init__(self, cells, L_eq):
        from mdelast_b200.units import Units as U
        self.cells, self.L_eq, self.U = cells, L_eq, U
        self.n_replicas = len(cells)
        _FakeBatch.built.append([float(c.box[0]) for c in cells])

    def autotune(self, n):
        return {}

    def run(self, *a):
        pass

    def fluctuation_start(self):
        pass

    def set_sample_ring(self, n):
        pass

    def drain_samples(self, r):
        p = -3.0 * self.B_GPa * (self.cells[r].box[0] / self.L_eq[r] - 1.0)
        return {"pressure": np.full(4, p * self.U.GPa)}

    def atoms(self, r, field):
        c = self.cells[r]
        return c.positions / c.box if field == "coords" else c.velocities

    def chain(self, r, which):
        return None, self.cells[r].thermo_p_eta, None

    def elastic_constants(self, r):
        return {"C11": 1.0, "C12": 1.0, "C44": 1.0}


def _warm(monkeypatch, bulk, offset):
    import mdelast_b200.protocol as P
    from mdelast_b200.warmstart import judge

    class _M:
        ATOM_COORDINATES, ATOM_VELOCITIES = "coords", "vel"

    cells = [_cell(), _cell(L=12e-8)]
    L_eq = [c.box[0] / (1.0 + offset) for c in cells]
    _FakeBatch.built = []
    monkeypatch.setattr(P, "make_batch", lambda m, t, cs, **k: _FakeBatch(cs, L_eq))
    fell_back = []

    def fake_protocol(*a, **k):
        fell_back.append(True)
        return ProtocolResult("mixed", 2, 8, Stages(), [1.0, 1.0], [0.0, 0.0], {}, [])

    monkeypatch.setattr(P, "run_protocol", fake_protocol)
    st = Stages(0, 0, 100, 400, 5, 20, 200)
    res = P.run_warm_start(_M, _Tables, cells, stages=st, judge=judge, check_steps=100,
                           bulk_GPa=bulk, autotune=False)
    return res, fell_back, L_eq


def test_warm_start_corrects_the_box_from_the_window_pressure(monkeypatch):
    # 0.1% too large an edge: the window reads -0.6 GPa, outside the 0.2 GPa tolerance;
    # one Newton step with the right bulk modulus lands on the equilibrium box
    res, fell_back, L_eq = _warm(monkeypatch, [200.0, 200.0], 1e-3)
    assert not fell_back and res.accepted_start and res.corrections == 1
    assert len(_FakeBatch.built) == 2
    assert np.allclose(_FakeBatch.built[1], L_eq, rtol=2e-6)
    assert all(abs(p) < 0.01 for p in res.npt_pressure_GPa)


def test_warm_start_without_bulk_moduli_falls_back(monkeypatch):
    res, fell_back, _ = _warm(monkeypatch, None, 1e-3)
    assert fell_back and not res.accepted_start and res.corrections == 0


def test_warm_start_accepts_a_good_box_untouched(monkeypatch):
    res, fell_back, _ = _warm(monkeypatch, [200.0, 200.0], 1e-5)
    assert not fell_back and res.corrections == 0 and len(_FakeBatch.built) == 1


def test_born_stability_and_linear_guess():
    from mdelast_b200.warmstart import _nialco_guess, born_stable, nialco_guess_a
    ok = born_stable([250, 100, 250, 250], [150, 120, 150, -200], [90, 50, -1, 90])
    assert ok.tolist() == [True, False, False, False]
    x = np.array([[1.0, 0.0, 0.0], [0.2, 0.1, 0.7]])
    g = _nialco_guess(x, [300.0, 600.0])
    assert g[0] == nialco_guess_a(x[0], 300.0) and g[1] == nialco_guess_a(x[1], 600.0)
    assert abs(g[0] - 3.52) < 1e-12
