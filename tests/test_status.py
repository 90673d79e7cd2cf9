"""The reference's run-ending checks and its print-only warnings on the GPU path.

The reference prints and calls exit(1) when rho leaves the embedding table
(eam.hpp:48-70), when the volume jumps by more than 5 % in one step (md_driver.cpp:493-497),
when the total momentum is not zero (:623-627) and when the conserved energy drifts beyond
fatal_conservation (:700-726); it prints and goes on when a pair comes closer than
rmin_fatal (potential.hpp:93-95). Here each is a status bit: the fatal ones end the driver
with a RuntimeError carrying the reference's message and the status word, the warnings stay
readable in `status`. Each case is checked twice: on the CPU, that the oracle (the C
restatement) raises exactly the expected bit for it, and on the GPU, that the driver's
status word equals the oracle's for the same inputs, in FP64 and in mixed precision."""

import dataclasses
import re

import numpy as np
import pytest

from helpers import dynamics_case, gpu, oracle, static_case
from mdelast_b200.units import Units as U
from oracle import ref

needs_oracle = pytest.mark.skipif(not ref.available("oracle"), reason="oracle not built")

RHO_MAX, VOLUME, MOMENTUM, CONSERVATION = 0x1, 0x2, 0x4, 0x10
WARN_RMIN = 0x200
MESSAGE = {RHO_MAX: "rho >rhomax_fatal", VOLUME: "volume change too large",
           MOMENTUM: "total momentum", CONSERVATION: "bad energy conservation"}


def rho_case():
    """rhomax_fatal just below the largest rho of the static cell: fatal in the first force
    call, the constructor's."""
    c = static_case()
    rho = oracle(c).atoms("rho_eam")
    t = dataclasses.replace(c.tables, rhomax=0.99 * float(np.max(rho)))
    return dataclasses.replace(c, tables=t), 0


def momentum_case():
    """A 300 K cell whose velocities all carry a drift of 2 m/s along x: the
    constructor's thermodynamics sees the net momentum."""
    c = dynamics_case()
    return dataclasses.replace(c, velocities=c.velocities + np.array([2e2, 0., 0.])), 0


def conservation_case():
    """fatal_conservation far below one step's energy error: fatal in the second step (the
    check skips the step that starts at cycle 0)."""
    return dataclasses.replace(dynamics_case(), fatal_conservation=1e-13), 2


def volume_case():
    """NPT with a barostat momentum that moves epsilon by 0.025 in one step (volume
    ×1.078)."""
    c = dynamics_case(ensemble=2)
    P, w, _ = c.baro
    return dataclasses.replace(c, baro=(P, w, 0.025 * w / c.dt)), 1


FATAL_CASES = {RHO_MAX: rho_case, MOMENTUM: momentum_case, CONSERVATION: conservation_case,
               VOLUME: volume_case}


def rmin_case(rmin_ang):
    c = static_case()
    t = dataclasses.replace(c.tables, rmin_fatal=rmin_ang * U.angstrom)
    return dataclasses.replace(c, tables=t)


def oracle_status(case, n_steps):
    o = oracle(case)
    if n_steps:
        o.integrate(n_steps)
    return o.status()


@needs_oracle
@pytest.mark.parametrize("bit", sorted(FATAL_CASES))
def test_oracle_raises_the_bit(bit):
    case, n_steps = FATAL_CASES[bit]()
    st = oracle_status(case, n_steps)
    assert st & 0xff == bit, hex(st)
    if n_steps:
        assert oracle_status(case, n_steps - 1) & 0xff == 0


@needs_oracle
def test_oracle_rmin_warning():
    assert oracle_status(rmin_case(3.0), 0) & WARN_RMIN
    assert not oracle_status(rmin_case(2.0), 0) & WARN_RMIN


def _status_word(err: RuntimeError) -> int:
    m = re.search(r"status 0x([0-9a-f]+)", str(err))
    assert m, str(err)
    return int(m.group(1), 16)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("bit", sorted(FATAL_CASES))
def test_gpu_fatal_matches_oracle(bit, precision):
    case, n_steps = FATAL_CASES[bit]()
    want = oracle_status(case, n_steps)
    with pytest.raises(RuntimeError, match=MESSAGE[bit]) as e:
        g = gpu(case, precision)
        assert n_steps, "the constructor should have raised"
        g.integrate_n(n_steps)
        g.epot_atom
    assert _status_word(e.value) & 0xff == want & 0xff
    if n_steps:
        # the driver stays ended, as the reference's process would be
        with pytest.raises(RuntimeError, match=MESSAGE[bit]):
            g.integrate()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_rmin_warning_matches_oracle(precision):
    for rmin in (3.0, 2.0):
        case = rmin_case(rmin)
        g = gpu(case, precision)
        assert g.status & WARN_RMIN == oracle_status(case, 0) & WARN_RMIN
        g.integrate()  # a warning does not end the run
        assert np.isfinite(g.epot_atom)


@pytest.mark.gpu
def test_gpu_batch_status_per_replica():
    """In a batch each replica keeps its own status word: one atom of replica 1 pushed
    0.6 A towards its nearest neighbour raises the rmin warning there only."""
    import md_driver_module as m

    from mdelast_b200.systems import cuzn_cell, make_batch

    t = dataclasses.replace(static_case().tables, rmin_fatal=2.2 * U.angstrom)
    cells = [cuzn_cell(t, 4, n_zn=16, velocity_seed=s) for s in (0, 1)]
    pos = cells[1].positions.copy()
    L = cells[1].box
    d = pos - pos[0]
    d -= L * np.round(d / L)
    r = np.linalg.norm(d, axis=1)
    r[0] = np.inf
    j = int(np.argmin(r))
    pos[0] += 0.6 * U.angstrom * d[j] / r[j]
    pos[0] -= L * np.floor((pos[0] + 0.5 * L) / L)
    cells[1] = dataclasses.replace(cells[1], positions=pos)
    b = make_batch(m, t, cells)
    st = np.asarray(b.status())
    assert st[0] & WARN_RMIN == 0 and st[1] & WARN_RMIN, [hex(x) for x in st]
    assert not np.any(st & 0xff)
