"""List builds inside one run() while a barostat shrinks the box below the cell grid the run
started with: the build widens its stencil, so the neighbour list stays the reference's
(md_driver.cpp:279-298) entry for entry, and the trajectory follows the oracle."""

import numpy as np
import pytest

from helpers import dynamics_case, gpu, gpu_atoms, oracle, rel_err

pytestmark = pytest.mark.gpu


def test_shrinking_box_list_and_trajectory():
    # 8^3 Cu-Zn cell started 8% above its lattice constant: the NPT run compresses it by
    # about 7% within 40 steps. With r_skin 1.09 the list radius is 7.41 A and the run
    # starts with 4 cells of 7.85 A per edge, which end up about 7.3 A wide, below the
    # radius, while the 2a shell of the compressed lattice lies near 7.3 A.
    c = dynamics_case(nside=8, n_zn=120, ensemble=2, T=300.0, a_ang=3.6345 * 1.08,
                      r_skin=1.09)
    g, o = gpu(c), oracle(c)
    L0 = c.box[0, 0]
    g.run(60, 20, 1)
    for s in range(60):
        if s % 20 == 0:
            o.calculate_neighbors()
        o.integrate()
    r_list = c.tables.rcut * 1.09
    nc = int(np.floor(L0 / (r_list * 1.05)))
    assert nc == 4
    h = np.array(g.box.h).reshape(3, 3)
    assert h[0, 0] / nc < r_list, "the box did not shrink below the cell grid"
    po, no = o.neighbors()
    pg, ng = g.neighbor_list()
    assert np.array_equal(np.asarray(pg), po)
    assert np.array_equal(np.asarray(ng), no)
    so = o.scalar_dict()
    for k in ["etot_cons", "pressure", "epot_atom", "temperature_kin"]:
        assert rel_err(getattr(g, k), so[k]) < 1e-9, k
    assert rel_err(gpu_atoms(g, "forces"), o.atoms("forces")) < 1e-9
    assert rel_err(gpu_atoms(g, "positions"), o.atoms("positions")) < 1e-9


def test_batch_status_reads_every_replica():
    import md_driver_module as m
    from mdelast_b200.systems import cuzn_cell, make_batch
    from helpers import tables
    t = tables()
    cells = [cuzn_cell(t, 5, x_zn=0.1, T=300.0, velocity_seed=k) for k in range(3)]
    b = make_batch(m, t, cells, precision="fp64")
    b.run(20, 20, 5)
    st = b.status()
    assert st.shape == (3,)
    assert all(int(s) & 0xFF == 0 for s in st)
