"""The staged force pass (mixed precision, quintic tables copied into each block's shared
memory) against the unstaged one on the same state: per-atom forces and energies bit for
bit, the global sums (virial, Born stress and tensor, Laplacian) within 1e-12 of each other
(their FP64 block partial sums are grouped differently), and a 20-step NVT trajectory
within 1e-12. The Cu-Zn cell has every pair in the staged range; the Ni-Al-Co and Cu01
cells, whose tables are larger than the shared memory, have only their outer intervals
staged, so their pairs exercise both the shared-memory and the global reads."""

import numpy as np
import pytest

from helpers import cu01_case, dynamics_case, gpu, gpu_atoms, gpu_scalars, nialco_case, rel_err

pytestmark = pytest.mark.gpu


def _pair(maker):
    c = maker()
    a, b = gpu(c, precision="mixed"), gpu(c, precision="mixed")
    if a.force_staging is None:
        pytest.fail("no staged table copy for a quintic EAM potential")
    a.set_launch(4, 8, 148 * 32, 148 * 32)
    a.force_staging = False
    b.set_launch(4, 8, 148 * 32, 148)
    b.force_staging = True
    assert b.force_staging is True and a.force_staging is False
    return a, b


def _same(a, b, tol_sums):
    for f in ("forces", "energies_pot", "rho_eam"):
        assert np.array_equal(gpu_atoms(a, f), gpu_atoms(b, f)), f
    sa, sb = gpu_scalars(a), gpu_scalars(b)
    for k in ("epot_atom", "born_stress_tensor", "born_elasticity_tensor", "total_laplacian",
              "pressure", "total_force2"):
        assert rel_err(sb[k], sa[k]) <= tol_sums, (k, rel_err(sb[k], sa[k]))


@pytest.mark.parametrize("maker", [lambda: dynamics_case(nside=8, n_zn=123),
                                   nialco_case, lambda: cu01_case(sigma_ang=0.08)],
                         ids=["cuzn2048", "nialco500", "cu01_500"])
def test_staged_equals_unstaged_static(maker):
    a, b = _pair(maker)
    _same(a, b, 1e-12)


def test_staged_trajectory():
    a, b = _pair(lambda: dynamics_case(nside=8, n_zn=123, ensemble=1))
    for _ in range(2):
        a.run(10, 20, 1, False)
        b.run(10, 20, 1, False)
    for f in ("positions", "velocities", "forces"):
        assert rel_err(gpu_atoms(b, f), gpu_atoms(a, f)) <= 1e-12, f
    assert rel_err(b.etot_cons, a.etot_cons) <= 1e-12
