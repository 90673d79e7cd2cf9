"""The statistical-benchmark driver (mdelast_b200.benchmarks) end to end on the GPU, on a
short version of Z1 (the 500-atom sample case at 300 K, 1,000 + 3,000 steps per stage):
every quantity the reference's verification reads comes out, and the ones that converge
within such a run (box ratio, Born term, temperatures, conserved energy) are already near
the reference's published full-length values."""

import numpy as np
import pytest

from helpers import tables

pytestmark = pytest.mark.gpu


def test_short_z1_runs_and_is_near_the_published_values():
    import md_driver_module as m
    from mdelast_b200.benchmarks import run_benchmark
    r = run_benchmark(m, tables(), "zn06_300K", "mixed", n_therm=1000, n_prod=3000)
    assert r["atoms"] == 500
    for stage in ("npt", "nvt"):
        s = r[stage]
        for k in ("C11", "C12", "C44", "CB11", "CB12", "CB44", "fluc11", "kin11", "T_kin",
                  "T_conf_recip", "T_conf_sample", "pressure", "L_L0", "econs_err_max",
                  "econs_drift_per_ns"):
            assert np.isfinite(s[k]), (stage, k)
        assert s["n_steps"] == 4000 and s["n_thermalization"] == 1000
        assert abs(s["T_kin"] - 300.0) < 15.0
        assert abs(s["CB11"] - 163.4) < 1.0 and abs(s["CB44"] - 76.07) < 0.5
        assert s["econs_err_max"] < 1e-4
    assert abs(r["npt"]["L_L0"] - 1.0089) < 1e-3
    assert abs(r["nvt"]["L_L0"] - 1.0) < 1e-12  # NVT: the box is the NPT mean box
    assert abs(r["nvt"]["kin11"] - 0.672) < 0.01
