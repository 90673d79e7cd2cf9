"""The pair list of the pair passes with 16-bit entries (offsets within the replica, the
default when every replica has at most 65,536 atoms) against 32-bit entries
(MDELAST_PAIR_LIST_16=0): the same pairs in the same order, so forces and trajectories are
identical bit for bit, in FP64 and in mixed precision, in a batch of uneven replicas."""

import os

import numpy as np
import pytest

from helpers import dynamics_case, gpu, gpu_atoms

pytestmark = pytest.mark.gpu


def _make(case, precision, wide):
    old = os.environ.get("MDELAST_PAIR_LIST_16")
    try:
        if wide:
            os.environ["MDELAST_PAIR_LIST_16"] = "0"
        else:
            os.environ.pop("MDELAST_PAIR_LIST_16", None)
        return gpu(case, precision=precision)
    finally:
        if old is None:
            os.environ.pop("MDELAST_PAIR_LIST_16", None)
        else:
            os.environ["MDELAST_PAIR_LIST_16"] = old


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pair16_equals_pair32(precision):
    c = dynamics_case(nside=8, n_zn=123, ensemble=2, T=600.0)
    a, b = _make(c, precision, True), _make(c, precision, False)
    for f in ("forces", "energies_pot"):
        assert np.array_equal(gpu_atoms(a, f), gpu_atoms(b, f)), f
    for _ in range(3):
        a.run(20, 20, 1, False)
        b.run(20, 20, 1, False)
    for f in ("positions", "velocities", "forces"):
        assert np.array_equal(gpu_atoms(a, f), gpu_atoms(b, f)), f
    assert a.etot_cons == b.etot_cons


def test_pair16_batch_uneven():
    import md_driver_module as m
    from mdelast_b200.systems import make_batch, uneven_replicas
    from helpers import tables
    t = tables()
    cells = uneven_replicas(t, 6, master_seed=7)
    old = os.environ.get("MDELAST_PAIR_LIST_16")
    out = []
    try:
        for wide in (True, False):
            if wide:
                os.environ["MDELAST_PAIR_LIST_16"] = "0"
            else:
                os.environ.pop("MDELAST_PAIR_LIST_16", None)
            b = make_batch(m, t, cells, precision="mixed")
            b.run(30, 20, 1, False)
            out.append([np.asarray(b.atoms(r, m.ATOM_POSITIONS)) for r in range(b.n_replicas)])
    finally:
        if old is None:
            os.environ.pop("MDELAST_PAIR_LIST_16", None)
        else:
            os.environ["MDELAST_PAIR_LIST_16"] = old
    for x, y in zip(*out):
        assert np.array_equal(x, y)
