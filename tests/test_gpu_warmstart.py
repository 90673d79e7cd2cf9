"""The learned warm start end to end on the GPU: training runs generated by the package's
own batched NPT/NVT protocol, the network trained by the device kernels, and what it gains
over the method without it: a run started in the proposed box is at equilibrium pressure,
one started at the Vegard's-law guess is not; a rejected proposal falls back to NPT."""

import numpy as np
import pytest

from helpers import tables

pytestmark = pytest.mark.gpu


def _cells(t, a_ang, R=4):
    from mdelast_b200.systems import cuzn_cell
    return [cuzn_cell(t, 4, n_zn=16, T=300.0, a_ang=a_ang, ensemble=1, velocity_seed=50 + k)
            for k in range(R)]


def test_warm_start_gain_over_vegard_start():
    import md_driver_module as m
    from mdelast_b200.protocol import Stages, run_warm_start
    from mdelast_b200.systems import vegard_a
    from mdelast_b200.warmstart import WarmStart, generate, judge
    t = tables()
    data = generate(m, t, n_runs=48, nside=4, batch=48, seed=7,
                    stages=Stages(1000, 1000, 200, 600, 5, 20, 600), T_range=(100.0, 600.0))
    assert np.all(np.abs(data["P_GPa"]) < 0.5)
    ws = WarmStart.fit(data, steps=3000)
    x, T = 16 / 256, 300.0
    a_ml = float(ws.propose(x, T)["a"][0])
    a_vg = vegard_a(x, T)
    st = Stages(0, 0, 500, 1000, 5, 20, 500)
    r_ml = run_warm_start(m, t, _cells(t, a_ml), stages=st, check_steps=1000)
    r_vg = run_warm_start(m, t, _cells(t, a_vg), stages=st, check_steps=1000)
    p_ml, p_vg = np.mean(r_ml.npt_pressure_GPa), np.mean(r_vg.npt_pressure_GPa)
    # the guess misses the equilibrium lattice constant by ~1 %: several GPa
    assert abs(p_vg) > 2.0
    assert abs(p_ml) < 0.25 * abs(p_vg) and abs(p_ml) < 0.5
    assert judge(p_ml, 0.5) and not judge(p_vg, 0.5)


def test_rejected_proposal_falls_back_to_npt():
    import md_driver_module as m
    from mdelast_b200.protocol import Stages, run_warm_start
    from mdelast_b200.systems import vegard_a
    from mdelast_b200.warmstart import judge
    t = tables()
    bad = vegard_a(0.06, 300.0) * 0.99
    r = run_warm_start(m, t, _cells(t, bad, R=2), stages=Stages(0, 0, 200, 600, 5, 20, 300),
                       judge=lambda p: judge(p, 0.2), check_steps=300,
                       fallback=Stages(800, 800, 200, 600, 5, 20, 300))
    assert not r.accepted_start
    assert all(abs(p) < 0.5 for p in r.npt_pressure_GPa)  # the NPT stage found the box
    assert all(v > 1.01 for v in r.V_V0)
