"""Device sample ring and fluctuation sums: the ring holds exactly what the reference's
append_sample reads after each sampled step (molecular_dynamics.py:1218-1238), the device
sums equal Welford sums of those samples, and the elastic constants from the sums equal
the reference's estimator (oracle/fluct.py, pinned to perform_thermal_average) applied to
the samples, and to the oracle's own trajectory."""

import numpy as np
import pytest

from helpers import dynamics_case, gpu, oracle, rel_err

pytestmark = pytest.mark.gpu

SCALARS = ["time", "temperature_kin", "temperature_conf_inverse", "total_laplacian",
           "total_force2", "pressure", "etot_atom", "epot_atom", "epot_eam_atom",
           "ekin_atom", "etot_cons", "etot_cons_err"]


def test_ring_records_equal_attributes_after_sampled_steps():
    d = gpu(dynamics_case(nside=4, n_zn=15, ensemble=2, T=600.0))
    d.drain_samples()
    want = []
    for k in range(12):
        d.sample_observables = k % 3 != 1
        d.integrate()
        if d.sample_observables:
            row = {n: getattr(d, n) for n in SCALARS}
            row["stress_tensor"] = np.array(d.stress_tensor)
            row["born_stress_tensor"] = np.array(d.born_stress_tensor)
            row["born_elasticity_tensor"] = np.array(d.born_elasticity_tensor)
            row["volume"] = d.box.volume()
            want.append(row)
    rec = d.drain_samples()
    assert rec["lost"] == 0 and len(rec["time"]) == len(want) == 8
    for k, row in enumerate(want):
        for n in SCALARS + ["stress_tensor", "born_stress_tensor", "born_elasticity_tensor"]:
            assert np.array_equal(rec[n][k], row[n]), (k, n)
        assert rec["volume"][k] == pytest.approx(row["volume"], rel=1e-15)
    assert len(d.drain_samples()["time"]) == 0


def test_ring_overflow_counts_lost_records():
    d = gpu(dynamics_case(nside=4, n_zn=15, ensemble=1))
    d.set_sample_ring(4)
    d.run(10, 0, 1)
    rec = d.drain_samples()
    assert rec["lost"] == 6 and list(rec["cycle"]) == [7.0, 8.0, 9.0, 10.0]
    d.run(3, 0, 1)
    rec = d.drain_samples()
    assert rec["lost"] == 0 and list(rec["cycle"]) == [11.0, 12.0, 13.0]
    d.run(4, 0, 2)  # sampled steps only: cycles 14 and 16
    assert list(d.drain_samples()["cycle"]) == [14.0, 16.0]


def _x(rec, N):
    return np.vstack([rec["born_stress_tensor"].T, N / rec["volume"], rec["volume"],
                      rec["etot_atom"]])


def _oracle_C(rec, ens, N, V0, T, P):
    from oracle.fluct import elastic_constants
    return elastic_constants(rec["born_stress_tensor"].T,
                             np.moveaxis(rec["born_elasticity_tensor"], 0, -1),
                             rec["volume"] / V0, rec["etot_atom"], ens, N, V0, T, P, 0)


@pytest.mark.parametrize("ens", [1, 2])
def test_device_sums_and_estimator(ens):
    from oracle.fluct import welford
    c = dynamics_case(nside=5, n_zn=30, ensemble=ens, T=300.0)
    d = gpu(c)
    d.run(10, 5, 1)
    d.drain_samples()
    d.fluctuation_start()
    d.run(80, 20, 1)
    rec = d.drain_samples()
    assert len(rec["time"]) == 80
    f = d.fluctuations()
    assert f["n"] == 80 and f["n_atoms"] == c.N
    mean, M = welford(_x(rec, c.N))
    assert rel_err(f["mean"], mean) < 1e-13
    Md = f["comoment"][np.triu_indices(9)]
    scale = np.sqrt(np.outer(np.diag(f["comoment"]), np.diag(f["comoment"])))[np.triu_indices(9)]
    ok = scale > 0
    assert np.max(np.abs(Md - M)[ok] / scale[ok]) < 1e-10
    assert rel_err(f["born_el_mean"], rec["born_elasticity_tensor"].mean(axis=0)) < 1e-13
    V0 = np.prod(np.diag(c.box))
    T, P = c.thermo[0], c.baro[0]
    e = d.elastic_constants()
    o = _oracle_C(rec, ens, c.N, V0, T, P)
    scaleC = np.max(np.abs(o["C"]))
    assert np.max(np.abs(e["C"] - o["C"])) / scaleC < 1e-9
    for k in ["C11", "C12", "C44"]:
        assert abs(e[k] - o[k]) / scaleC < 1e-9, k
    if ens == 2:
        for k in ["bulk_modulus", "compressibility", "volume_thermal_expansion"]:
            assert e[k] == pytest.approx(o[k], rel=1e-8), k
    else:
        assert e["bulk_modulus"] == 0.0


@pytest.mark.parametrize("ens", [1, 2])
def test_estimator_against_oracle_trajectory(ens):
    """The whole chain against the CPU oracle: its trajectory sampled every step, the
    reference's estimator on its samples, vs the GPU sums of the same steps."""
    from oracle.fluct import elastic_constants
    c = dynamics_case(nside=4, n_zn=15, ensemble=ens, T=300.0)
    d, o = gpu(c), oracle(c)
    d.fluctuation_start()
    bs, be, vol, et = [], [], [], []
    for _ in range(40):
        d.integrate()
        o.integrate(1)
        s = o.scalar_dict()
        bs.append(s["born_stress_tensor"])
        be.append(s["born_elasticity_tensor"])
        vol.append(np.prod(np.diag(s["box"])))
        et.append(s["etot_atom"])
    V0 = np.prod(np.diag(c.box))
    T, P = c.thermo[0], c.baro[0]
    ref = elastic_constants(np.array(bs).T, np.moveaxis(np.array(be), 0, -1),
                            np.array(vol) / V0, np.array(et), ens, c.N, V0, T, P, 0)
    e = d.elastic_constants()
    scale = np.max(np.abs(ref["C"]))
    assert np.max(np.abs(e["C"] - ref["C"])) / scale < 1e-6
    for k in ["C11", "C12", "C44"]:
        assert abs(e[k] - ref[k]) / scale < 1e-6, k


def test_batch_replicas_accumulate_separately():
    import md_driver_module as m
    from mdelast_b200.systems import cuzn_cell, make_batch
    from helpers import tables
    t = tables()
    cells = [cuzn_cell(t, 4, n_zn=15, T=300.0, ensemble=1, velocity_seed=1),
             cuzn_cell(t, 5, x_zn=0.2, T=600.0, ensemble=2, placement_seed=7, velocity_seed=2)]
    b = make_batch(m, t, cells, dt=2e-15)
    b.fluctuation_start()
    b.run(40, 20, 1)
    for r, cell in enumerate(cells):
        rec = b.drain_samples(r)
        assert len(rec["time"]) == 40 and rec["lost"] == 0
        V0 = float(np.prod(cell.box))
        o = _oracle_C(rec, cell.ensemble, cell.n_atoms, V0, cell.T, cell.pressure)
        e = b.elastic_constants(r)
        assert np.max(np.abs(e["C"] - o["C"])) / np.max(np.abs(o["C"])) < 1e-9, r
        assert b.fluctuations(r)["n_atoms"] == cell.n_atoms
