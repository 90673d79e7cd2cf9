"""Batched replicas: several independent cells of different sizes, compositions,
temperatures and ensembles advanced together must each follow their own oracle run."""

import numpy as np
import pytest

from helpers import quiet_fd1, rel_err, tables

pytestmark = pytest.mark.gpu


def oracle_for(t, cell, dt, neighbors=True, r_skin=1.2):
    from mdelast_b200.systems import rg_bins
    from oracle.ref import OracleDriver
    with quiet_fd1():
        return OracleDriver(t, cell.positions, cell.velocities, cell.types,
                            ensemble=cell.ensemble,
                            thermo=(cell.T, cell.thermo_q, cell.thermo_p_eta, cell.Nf),
                            baro=(cell.pressure, cell.baro_w, cell.baro_p_eps),
                            baro_thermo=(cell.T, cell.baro_q, cell.baro_p_eta, 1.0),
                            box=np.diag(cell.box), rg=rg_bins(cell), Nf=cell.Nf, dt=dt,
                            neighbors=neighbors, r_skin=r_skin)


def test_batch_replicas_follow_their_oracles():
    import md_driver_module as m
    from mdelast_b200.systems import cuzn_cell, l12_cell, make_batch
    t = tables()
    cells = [cuzn_cell(t, 4, n_zn=15, T=300.0, ensemble=1, velocity_seed=1),
             cuzn_cell(t, 5, x_zn=0.2, T=600.0, ensemble=2, placement_seed=7, velocity_seed=2),
             l12_cell(t, 4, T=5.0, ensemble=1)]
    dt = 2e-15
    b = make_batch(m, t, cells, dt=dt)
    assert b.n_replicas == 3 and b.n_atoms == sum(c.n_atoms for c in cells)
    orcs = [oracle_for(t, c, dt) for c in cells]
    n_steps, every = 12, 5
    b.run(n_steps, every, 1)
    for o in orcs:
        for s in range(n_steps):
            if s % every == 0:
                o.calculate_neighbors()
            o.integrate()
    for r, o in enumerate(orcs):
        obs, so = b.observables(r), o.scalar_dict()
        for k in ["epot_atom", "ekin_atom", "etot_cons", "pressure", "total_laplacian",
                  "temperature_kin", "time"]:
            assert rel_err(obs[k], so[k]) < 1e-9, (r, k, obs[k], so[k])
        for k in ["born_stress_tensor", "born_elasticity_tensor", "stress_tensor"]:
            assert rel_err(obs[k], so[k]) < 1e-9, (r, k)
        assert rel_err(b.atoms(r, m.ATOM_FORCES), o.atoms("forces")) < 1e-9
        assert rel_err(b.atoms(r, m.ATOM_POSITIONS), o.atoms("positions")) < 1e-9
        assert obs["cycle"] == n_steps


def test_batch_uneven_sizes_mixed_precision():
    """The 64-replica workload shape (n in [4, 20]) at a reduced count: every replica
    conserves its extended energy over 40 mixed-precision steps."""
    import md_driver_module as m
    from mdelast_b200.systems import make_batch, uneven_replicas
    t = tables()
    cells = uneven_replicas(t, count=6, n_range=(4, 9))
    b = make_batch(m, t, cells, dt=1e-15, precision="mixed")
    e0 = [b.observables(r)["etot_cons"] for r in range(b.n_replicas)]
    b.run(40, 20, 1)
    for r in range(b.n_replicas):
        o = b.observables(r)
        assert o["status"] & 0xff == 0
        assert abs(o["etot_cons"] / e0[r] - 1.0) < 5e-5, (r, cells[r].T)
    # the batch-wide readout holds the same values, replica along the first axis
    allo = b.observables_all()
    for r in range(b.n_replicas):
        o = b.observables(r)
        for k in ("etot_cons", "pressure", "temperature_kin", "time", "volume", "cycle",
                  "status"):
            assert allo[k][r] == o[k], k
        for k in ("stress_tensor", "born_stress_tensor", "born_elasticity_tensor"):
            assert np.array_equal(allo[k][r], np.asarray(o[k])), k
        assert tuple(allo["box"][r]) == tuple(o["box"])


def test_memory_reused_and_released():
    """A batch created in the memory its predecessor freed (kept by the device's pool)
    gives the same results as the first, and again after the pool was handed back."""
    import md_driver_module as m
    from mdelast_b200.systems import cuzn_cell, make_batch
    t = tables()
    cells = [cuzn_cell(t, 5, n_zn=30, velocity_seed=s) for s in (0, 1)]

    def run():
        b = make_batch(m, t, cells, precision="mixed")
        b.run(30, 20, 1)
        out = [(b.observables(r)["etot_cons"], b.observables(r)["pressure"])
               for r in range(b.n_replicas)]
        del b
        return out

    first = run()
    assert run() == first
    m.release_cached_memory(0)
    assert run() == first
