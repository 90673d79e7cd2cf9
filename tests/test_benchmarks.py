"""Host side of the statistical benchmarks (mdelast_b200.benchmarks): the stage summary
against direct numpy evaluation on a fake batch with known sample series, and the
expectation fixture read from the reference's published benchmark files."""

import json
import os

import numpy as np

from mdelast_b200.benchmarks import summarize_stage
from mdelast_b200.systems import Cell
from mdelast_b200.units import Units as U

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "benchmarks_expected.json")


class _FakeBatch:
    """One replica whose sample series are drawn from a seeded stream; the fluctuation
    readouts return fixed tensors."""

    def __init__(self, V0, seed=3):
        self.rs = np.random.RandomState(seed)
        self.V0 = V0
        self.t = 0.0
        self.pending = []
        self.all = []
        self.prod_from = None
        self.C = self.rs.uniform(50, 150, (6, 6)) * U.GPa
        self.CB = np.triu(self.rs.uniform(60, 170, (6, 6))) * U.GPa
        self.rho, self.K = 8.5e22, 120.0 * U.GPa

    def fluctuation_start(self):
        self.prod_from = len(self.all)

    def run(self, k, rebuild, stride, timed):
        for _ in range(k):
            self.t += 2e-15
            r = {"time": self.t, "etot_cons": -1e-8 * (1 + 1e-6 * self.rs.randn() + 3e-4 * self.t / 1e-9),
                 "temperature_conf_inverse": 1 / (300 + self.rs.randn()),
                 "temperature_kin": 300 + self.rs.randn(), "pressure": 1e7 * self.rs.randn(),
                 "volume": self.V0 * (1.01 + 1e-3 * self.rs.randn())}
            self.pending.append(r)
            self.all.append(r)

    def drain_samples(self, r):
        out = {k: np.array([x[k] for x in self.pending]) for k in self.pending[0]}
        self.pending = []
        return out

    def elastic_constants(self, r):
        return {"C": self.C, "bulk_modulus": self.K}

    def fluctuations(self, r):
        mean = np.zeros(9)
        mean[6] = self.rho
        return {"born_el_mean": self.CB, "mean": mean}


def _cell(L=3e-7):
    z = np.zeros(10)
    return Cell(positions=np.zeros((4, 3)), velocities=np.zeros((4, 3)),
                types=np.zeros(4, np.uint32), box=np.array([L, L, L]), T=300.0, ensemble=2,
                thermo_q=z + 1, thermo_p_eta=z, baro_q=z + 1, baro_p_eta=z, baro_w=1.0,
                baro_p_eps=0.0, Nf=9.0)


def test_stage_summary_matches_direct_evaluation():
    c = _cell()
    V0 = float(np.prod(c.box))
    b = _FakeBatch(V0)
    s = summarize_stage(b, c, n_therm=1500, n_prod=2600)
    prod = b.all[b.prod_from:]
    assert b.prod_from == 1500 and len(prod) == 2600 and s["n_steps"] == 4100
    inv = np.array([x["temperature_conf_inverse"] for x in prod])
    assert np.isclose(s["T_conf_recip"], 1 / inv.mean(), rtol=1e-12)
    assert np.isclose(s["T_conf_sample"], np.mean(1 / inv), rtol=1e-12)
    assert np.isclose(s["T_kin"], np.mean([x["temperature_kin"] for x in prod]), rtol=1e-12)
    assert np.isclose(s["pressure"], np.mean([x["pressure"] for x in prod]) / U.GPa, rtol=1e-12)
    vv = np.array([x["volume"] for x in prod]) / V0
    assert np.isclose(s["L_L0"], np.mean(vv ** (1 / 3)), rtol=1e-12)
    e = np.array([x["etot_cons"] for x in b.all])
    rel = e / e[0] - 1
    assert np.isclose(s["econs_err_max"], np.abs(rel).max(), rtol=1e-12)
    t = np.array([x["time"] for x in b.all])
    slope = np.polyfit(t[1500:] * 1e9, rel[1500:], 1)[0]
    assert np.isclose(s["econs_drift_per_ns"], slope, rtol=1e-9)
    # C = CB - fluc + kin + K (i, j < 3), in cubic averages
    kT = U.k_boltz * 300.0
    kin11, kin44 = 2 * b.rho * kT / U.GPa, b.rho * kT / U.GPa
    K = b.K / U.GPa
    assert np.isclose(s["kin11"], kin11) and np.isclose(s["kin44"], kin44)
    assert np.isclose(s["C11"], s["CB11"] - s["fluc11"] + kin11 + K)
    assert np.isclose(s["C12"], s["CB12"] - s["fluc12"] + K)
    assert np.isclose(s["C44"], s["CB44"] - s["fluc44"] + kin44)
    C = b.C / U.GPa
    assert np.isclose(s["C44"], (C[3, 3] + C[4, 4] + C[5, 5]) / 3)
    CB = b.CB / U.GPa
    assert np.isclose(s["CB12"], (CB[0, 1] + CB[0, 2] + CB[1, 2]) / 3)


def test_expectation_fixture():
    d = json.load(open(GOLDEN))
    z1, l1 = d["zn06_300K"], d["l12_cuzn3_5K"]
    nvt = z1["stages"]["nvt"]
    assert nvt["n_steps"] == 150000 and nvt["n_thermalization"] == 50000
    assert abs(nvt["quantities"]["C11"]["expected"] - 153.2387) < 1e-3
    assert nvt["quantities"]["C11"]["tol"] == 1.0
    assert nvt["quantities"]["econs_err_max"]["max"] == 3.2e-05
    assert abs(z1["stages"]["npt"]["quantities"]["L_L0"]["expected"] - 1.008903) < 1e-6
    assert abs(l1["stages"]["nvt"]["quantities"]["C44"]["expected"] - 42.8403) < 1e-3
    assert l1["zero_kelvin_reference"]["max_rel_deviation"] == 0.002
    assert "info" in z1["stages"]["npt"]["quantities"]["C11"]
