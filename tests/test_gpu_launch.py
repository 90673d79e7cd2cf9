"""Launch shapes of the pair passes (lanes per atom, block targets) and the autotuner:
every shape gives the oracle's forces (FP64 within 1e-10, the parity bound), and a run
after autotune follows the oracle's trajectory."""

import numpy as np
import pytest

from helpers import dynamics_case, gpu, gpu_atoms, oracle, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tpa", [1, 4, 8, 16])
@pytest.mark.parametrize("blocks", [148 * 8, 148 * 64])
def test_every_launch_shape_gives_oracle_forces(tpa, blocks):
    c = dynamics_case(nside=5, n_zn=30, ensemble=1)
    d, o = gpu(c), oracle(c)
    d.set_launch(tpa, tpa, blocks, blocks)
    assert rel_err(gpu_atoms(d, "forces"), o.atoms("forces")) < 1e-10
    assert rel_err(gpu_atoms(d, "rho_eam"), o.atoms("rho_eam")) < 1e-10


def test_autotuned_run_follows_oracle():
    c = dynamics_case(nside=5, n_zn=30, ensemble=2, T=600.0)
    d, o = gpu(c), oracle(c)
    choice = d.autotune(2)
    assert choice["tpa_density"] in (1, 4, 8, 16) and choice["tpa_force"] in (1, 4, 8, 16)
    assert choice["ms_density"] > 0 and choice["ms_force"] > 0
    for _ in range(10):
        d.integrate()
    o.integrate(10)
    s = o.scalar_dict()
    for k in ["etot_cons", "pressure", "temperature_kin", "epot_atom"]:
        assert rel_err(getattr(d, k), s[k]) < 1e-9, k
    assert rel_err(gpu_atoms(d, "positions"), o.atoms("positions")) < 1e-9


def test_set_launch_mixed_batch_keeps_observables():
    import md_driver_module as m
    from helpers import tables
    from mdelast_b200.systems import cuzn_cell, make_batch
    t = tables()
    cells = [cuzn_cell(t, 4, n_zn=15, velocity_seed=1), cuzn_cell(t, 6, x_zn=0.1, velocity_seed=2)]
    ref = make_batch(m, t, cells, precision="mixed")
    ref.run(5, 20, 1)
    for shape in [(1, 16, 148 * 8, 148 * 64), (16, 1, 148 * 64, 148 * 8)]:
        b = make_batch(m, t, cells, precision="mixed")
        b.set_launch(*shape)
        b.run(5, 20, 1)
        for r in range(2):
            o, p = b.observables(r), ref.observables(r)
            for k in ["etot_cons", "pressure", "epot_atom"]:
                assert rel_err(o[k], p[k]) < 1e-5, (shape, r, k)
