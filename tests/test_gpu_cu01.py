"""Configuration C1, pure Cu with the single-element Mishin Cu01 tables (10,000 nodes per
function, the largest tables of the shipped potentials; ``examples/cu_300k/run.py:58-78``
loads them through ``get_EAM_file``), on the GPU against the oracle: FP64 within 1e-10 on a
displaced static cell, 20-step NVT trajectories within 1e-9 with the neighbour list and
with the all-pairs search the example uses (``neighbors`` left at False), and the mixed
path within the tolerances of ``test_gpu_mixed.py``."""

import numpy as np
import pytest

from helpers import cu01_case, gpu, gpu_atoms, oracle, rel_err
from test_gpu_parity import compare_state

pytestmark = pytest.mark.gpu


def test_cu01_static_fp64():
    c = cu01_case(sigma_ang=0.08)
    o, g = oracle(c), gpu(c)
    compare_state(g, o, 1e-10)
    F = gpu_atoms(g, "forces")
    assert np.abs(F.sum(0)).max() / np.abs(F).max() < 1e-12


@pytest.mark.parametrize("neighbors", [True, False])
def test_cu01_nvt_trajectory(neighbors):
    c = cu01_case(neighbors=neighbors, r_skin=1.2 if neighbors else 1000.0)
    o, g = oracle(c), gpu(c)
    for step in range(20):
        if neighbors and step % 10 == 0:
            o.calculate_neighbors()
            g.calculate_neighbors()
        o.integrate()
        g.integrate()
    compare_state(g, o, 1e-9)


def test_cu01_list_identical():
    c = cu01_case(nside=8)
    o, g = oracle(c), gpu(c)
    po, no = o.neighbors()
    pg, ng = g.neighbor_list()
    assert np.array_equal(np.asarray(pg), po)
    assert np.array_equal(np.asarray(ng), no)


def test_cu01_mixed_static():
    from test_gpu_mixed import check
    c = cu01_case(sigma_ang=0.08)
    g = gpu(c, precision="mixed")
    check(g, oracle(c))
    F = gpu_atoms(g, "forces")
    assert np.abs(F.sum(0)).max() / np.abs(F).max() < 1e-12
