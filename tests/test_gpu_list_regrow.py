"""run() outgrowing its neighbour-list capacity in mid-run: the reference grows its list
whenever a rebuild needs more room (md_driver.cpp:288-292). Here the capacity starts at
exactly the largest count (MDELAST_LIST_HEADROOM=0), the cell starts 3 % wider than its
equilibrium lattice constant, and the barostat compresses it over 300 NPT steps, so the
in-step rebuilds overflow repeatedly. The run must finish, report the resumed launches,
and follow the oracle (which grows its list as the reference does) within 1e-9, on the
all-pairs search (500 atoms) and the cell-list search (2,048 atoms)."""

import os

import pytest

from helpers import dynamics_case, gpu, oracle
from test_gpu_parity import compare_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nside", [5, 8])
def test_run_regrows_list(nside):
    c = dynamics_case(nside=nside, n_zn=int(0.06 * 4 * nside**3), ensemble=2, a_ang=3.75)
    old = os.environ.get("MDELAST_LIST_HEADROOM")
    os.environ["MDELAST_LIST_HEADROOM"] = "0"
    try:
        g = gpu(c)
        maxn0, _ = g.list_capacity
        for _ in range(3):
            g.run(100, 20, 1, False)
        maxn1, regrowths = g.list_capacity
    finally:
        if old is None:
            os.environ.pop("MDELAST_LIST_HEADROOM", None)
        else:
            os.environ["MDELAST_LIST_HEADROOM"] = old
    o = oracle(c)
    for step in range(300):
        if step % 20 == 0:
            o.calculate_neighbors()
        o.integrate()
    assert regrowths > 0 and maxn1 > maxn0, (maxn0, maxn1, regrowths)
    compare_state(g, o, 1e-9)
