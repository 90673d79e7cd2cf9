"""The pair list of the pair passes (the neighbour list's pairs within factor * r_cut,
refreshed when atoms have moved far enough): the same results as walking the whole
neighbour list, in FP64 against the oracle over runs with list rebuilds and refreshes, and
in mixed precision against the full-list run."""

import numpy as np
import pytest

from helpers import dynamics_case, gpu, gpu_atoms, oracle, rel_err, tables

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("factor", [0.0, 1.02, 1.06])
def test_fp64_run_follows_oracle(factor):
    """A small margin (1.02) forces frequent refreshes at 900 K."""
    c = dynamics_case(nside=5, n_zn=30, ensemble=1, T=900.0)
    g, o = gpu(c), oracle(c)
    g.set_pair_list(factor)
    g.run(60, 20, 1)
    for s in range(60):
        if s % 20 == 0:
            o.calculate_neighbors()
        o.integrate()
    so = o.scalar_dict()
    for k in ["etot_cons", "pressure", "epot_atom", "temperature_kin", "total_laplacian"]:
        assert rel_err(getattr(g, k), so[k]) < 1e-9, (factor, k)
    assert rel_err(gpu_atoms(g, "forces"), o.atoms("forces")) < 1e-9
    assert rel_err(gpu_atoms(g, "positions"), o.atoms("positions")) < 1e-9


def test_mixed_batch_same_as_full_list():
    import md_driver_module as m
    from mdelast_b200.systems import cuzn_cell, make_batch
    t = tables()
    cells = [cuzn_cell(t, 5, x_zn=0.1, T=900.0, velocity_seed=k) for k in range(3)]
    a = make_batch(m, t, cells, precision="mixed")
    b = make_batch(m, t, cells, precision="mixed")
    a.set_pair_list(0.0)
    b.set_pair_list(1.03)
    a.run(40, 20, 1)
    b.run(40, 20, 1)
    for r in range(3):
        oa, ob = a.observables(r), b.observables(r)
        for k in ["etot_cons", "pressure", "epot_atom"]:
            assert rel_err(ob[k], oa[k]) < 1e-6, (r, k)
