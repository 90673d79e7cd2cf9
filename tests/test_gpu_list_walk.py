"""The neighbour list of a cell-list replica from k_nbr_build's per-atom walk over the half
cells (MDELAST_CELL_STAGING=0; the path the build takes for cells too crowded for
k_nbr_cells' staging, and for boxes an NPT run has shrunk) against the default staged build
and the oracle: the list of md_driver.cpp:279-298 entry for entry, forces within 1e-12 of
the staged build's (the rows hold the same pairs in another order), and a 40-step NPT
trajectory with list rebuilds within 1e-9 of the oracle."""

import os

import numpy as np
import pytest

from helpers import dynamics_case, gpu, gpu_atoms, oracle, rel_err

pytestmark = pytest.mark.gpu


def _make(case, staging):
    old = os.environ.get("MDELAST_CELL_STAGING")
    try:
        if staging:
            os.environ.pop("MDELAST_CELL_STAGING", None)
        else:
            os.environ["MDELAST_CELL_STAGING"] = "0"
        return gpu(case)
    finally:
        if old is None:
            os.environ.pop("MDELAST_CELL_STAGING", None)
        else:
            os.environ["MDELAST_CELL_STAGING"] = old


def test_cell_walk_equals_staged_and_oracle():
    # 10^3 cell: 4 cells of at least 1.05 list radii per edge, 8 half cells
    c = dynamics_case(nside=10, n_zn=240, ensemble=2, T=600.0)
    walk, staged, o = _make(c, False), _make(c, True), oracle(c)
    pw, nw = walk.neighbor_list()
    ps, ns = staged.neighbor_list()
    po, no = o.neighbors()
    assert np.array_equal(np.asarray(pw), po) and np.array_equal(np.asarray(nw), no)
    assert np.array_equal(np.asarray(ps), po) and np.array_equal(np.asarray(ns), no)
    assert rel_err(gpu_atoms(walk, "forces"), gpu_atoms(staged, "forces")) < 1e-12
    walk.run(40, 20, 1)
    for s in range(40):
        if s % 20 == 0:
            o.calculate_neighbors()
        o.integrate()
    pw, nw = walk.neighbor_list()
    po, no = o.neighbors()
    assert np.array_equal(np.asarray(pw), po) and np.array_equal(np.asarray(nw), no)
    so = o.scalar_dict()
    for k in ["etot_cons", "pressure", "epot_atom", "temperature_kin"]:
        assert rel_err(getattr(walk, k), so[k]) < 1e-9, k
    assert rel_err(gpu_atoms(walk, "forces"), o.atoms("forces")) < 1e-9
    assert rel_err(gpu_atoms(walk, "positions"), o.atoms("positions")) < 1e-9
