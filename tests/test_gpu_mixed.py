"""Mixed precision (FP32 pair and table math, FP64 sums and integrator) against the FP64
oracle on the same inputs. Tolerances (relative to the largest magnitude of each quantity)
are those of single-precision pair terms summed in double: 2e-5 for forces, 1e-6 for
energies, 1e-4 for the Born tensor, Laplacian and pressure."""

import numpy as np
import pytest

from helpers import dynamics_case, gpu, gpu_atoms, gpu_scalars, nialco_case, oracle, rel_err, static_case

pytestmark = pytest.mark.gpu

TOLS = {"forces": 2e-5, "epot_atom": 1e-6, "epot_eam_atom": 1e-6, "etot_atom": 1e-6,
        "etot_cons": 1e-6, "pressure": 1e-4, "born_stress_tensor": 1e-4,
        "born_elasticity_tensor": 1e-4, "total_laplacian": 1e-4, "total_force2": 1e-4,
        "rho_eam": 1e-6, "energies_pot": 1e-6}


def check(g, o):
    s_g, s_o = gpu_scalars(g), o.scalar_dict()
    for k in ["epot_atom", "epot_eam_atom", "etot_atom", "etot_cons", "pressure",
              "born_stress_tensor", "born_elasticity_tensor", "total_laplacian", "total_force2"]:
        assert rel_err(s_g[k], s_o[k]) <= TOLS[k], (k, rel_err(s_g[k], s_o[k]))
    for f in ["forces", "rho_eam", "energies_pot"]:
        assert rel_err(gpu_atoms(g, f), o.atoms(f)) <= TOLS[f], (f, rel_err(gpu_atoms(g, f), o.atoms(f)))


@pytest.mark.parametrize("maker", [static_case, nialco_case])
def test_mixed_static(maker):
    c = maker()
    check(gpu(c, precision="mixed"), oracle(c))


def test_mixed_net_force_vanishes():
    """Pair forces are antisymmetric in FP32 and summed in FP64: the net force stays at the
    FP64 round-off level (smoke.json bound 1e-12 relative)."""
    g = gpu(static_case(), precision="mixed")
    F = gpu_atoms(g, "forces")
    assert np.abs(F.sum(0)).max() / np.abs(F).max() < 1e-12


def test_mixed_dynamics_conserves():
    """500 NVE steps at dt = 1 fs (benchmark S Part B1 setting): the conserved energy drifts
    no more than the smoke bound 1.5e-5, and the momentum check never fires."""
    c = dynamics_case(nside=5, ensemble=0, dt=1e-15)
    g = gpu(c, precision="mixed")
    e0 = g.etot_cons
    worst = 0.0
    for blk in range(25):
        g.run(20, 20, 1, False)
        worst = max(worst, abs(g.etot_cons / e0 - 1.0))
    assert worst < 1.5e-5, worst


def test_mixed_short_trajectory_close_to_fp64():
    """10 NVT steps: mixed and FP64 trajectories stay within single-precision distance."""
    c = dynamics_case(nside=5, ensemble=1)
    o = oracle(c)
    g = gpu(c, precision="mixed")
    for _ in range(10):
        o.integrate()
        g.integrate()
    assert rel_err(gpu_atoms(g, "positions"), o.atoms("positions")) < 1e-6
    assert rel_err(g.etot_cons, o.scalar_dict()["etot_cons"]) < 1e-6
