"""The reference's own callers driving a ``md_driver_module``, replayed call for call.

``golden/dropin_traces.npz`` holds every call that ``run_smoke.py``'s Part B dynamics
(``MolecularDynamics.run()`` in NPT and NVT, and NVE through ``integrate()``), its Part C
ternary cell and the pure-Cu example (``examples/cu_300k/run.py``) made on
``md_driver_module``, with the values the reference's C++ core returned
(``golden/make_dropin_trace.py``). Here those calls are replayed:

* on the CPU against the same reference core and against the oracle's C restatement: every
  value read must come back bit for bit (the replay is faithful and the restatement exact);
* on the GPU (``-m gpu``) against this package's ``md_driver_module``, FP64 and mixed
  precision: every attribute the run loop reads after every step, every g(r) histogram,
  every XYZ dump's positions and velocities, and the ternary cell's forces, against the
  reference's values. The tolerances are relative to the largest magnitude the reference
  gave for the same attribute in the session (``etot_cons_err``, itself a relative energy
  error, is compared as it is): FP64 1e-9; mixed precision 1e-4 for observables, 2e-5 for
  positions, velocities and forces, 1e-6 for ``etot_cons_err`` (the conserved energy
  agrees to ~2e-8), and the summed g(r) deviation within 1e-2 of the histogram's sum (a
  count moves to the next bin when a pair distance crosses a bin edge, and the mixed and
  FP64 trajectories drift apart over a run of several hundred steps).
"""

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import dropin  # noqa: E402
from mdelast_b200.potentials import find_potential, read_setfl  # noqa: E402

TRACE = os.path.join(HERE, "golden", "dropin_traces.npz")
SESSIONS = dropin.load(TRACE)
POTENTIALS = ["ZnCu.eam.alloy", "Mishin_updated-Ni-Al-Co-2013.eam.alloy", "Cu01.eam.alloy.txt"]
ABSOLUTE = ("etot_cons_err",)


@pytest.fixture(scope="module")
def tables():
    paths = [find_potential(n) for n in POTENTIALS]
    if any(p is None for p in paths):
        pytest.skip("potential files not staged")
    return dropin.table_arrays([read_setfl(p) for p in paths])


def _flat(v):
    if isinstance(v, dict):
        return np.concatenate([_flat(x).ravel() for x in v.values()])
    return np.atleast_1d(np.asarray(v, dtype=float))


class Checker:
    """Compares each replayed read with the reference's and keeps the worst deviation per
    attribute, relative to that attribute's largest recorded magnitude."""

    def __init__(self, events, arrays):
        self.arrays = arrays
        self.scale = {}
        for ev in events:
            if ev[0] in ("get", "call"):
                want = _flat(dropin.uncanon(ev[3] if ev[0] == "get" else ev[4], arrays))
                m = float(np.max(np.abs(want))) if want.size else 0.0
                self.scale[ev[2]] = max(self.scale.get(ev[2], 0.0), m)
        self.worst = {}
        self.exact = True

    def __call__(self, i, ev, got):
        want = dropin.uncanon(ev[3] if ev[0] == "get" else ev[4], self.arrays)
        g, w = _flat(got), _flat(want)
        assert g.shape == w.shape, (i, ev[2], g.shape, w.shape)
        # the reference's own NaNs (e.g. an empty partial g(r) of a one-element cell) must
        # come back as NaNs; the rest is compared by value
        nan = np.isnan(w)
        assert np.array_equal(nan, np.isnan(g)), (i, ev[2], "NaN pattern differs")
        g, w = g[~nan], w[~nan]
        if not np.array_equal(g, w):
            self.exact = False
        name = ev[2]
        if name in ABSOLUTE:
            err = float(np.max(np.abs(g - w))) if g.size else 0.0
        elif name in ("gr", "gr_partial"):
            err = float(np.sum(np.abs(g - w)) / max(np.sum(np.abs(w)), 1e-300))
        else:
            err = float(np.max(np.abs(g - w)) / max(self.scale[name], 1e-300)) if g.size else 0.0
        self.worst[name] = max(self.worst.get(name, 0.0), err)


def _replay(name, module, tables):
    events, arrays = SESSIONS[name]
    chk = Checker(events, arrays)
    dropin.replay(events, arrays, module, tables, chk)
    return chk


@pytest.mark.parametrize("which", ["ref", "oracle"])
@pytest.mark.parametrize("name", sorted(SESSIONS))
def test_replay_cpu_bitwise(name, which, tables):
    from oracle import ref
    from oracle import ref_module
    if not ref.available(which):
        pytest.skip(f"{which} library not built")
    chk = _replay(name, ref_module.module(which), tables)
    assert chk.exact, {k: v for k, v in chk.worst.items() if v}


def _gpu_module(precision):
    import md_driver_module as m
    if not m.device_available():
        pytest.fail("no CUDA device for the GPU replay")
    m.set_default_precision(precision)
    return m


TOL_FP64 = 1e-9
TOL_MIXED = {"default": 1e-4, "positions": 2e-5, "velocities": 2e-5, "forces": 2e-5,
             "etot_cons_err": 1e-6, "gr": 1e-2, "gr_partial": 1e-2}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SESSIONS))
def test_replay_gpu_fp64(name, tables):
    m = _gpu_module("fp64")
    try:
        chk = _replay(name, m, tables)
    finally:
        m.set_default_precision("fp64")
    print(name, "fp64 worst:", {k: f"{v:.1e}" for k, v in sorted(chk.worst.items()) if v})
    bad = {k: v for k, v in chk.worst.items() if v > TOL_FP64}
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SESSIONS))
def test_replay_gpu_mixed(name, tables):
    m = _gpu_module("mixed")
    try:
        chk = _replay(name, m, tables)
    finally:
        m.set_default_precision("fp64")
    print(name, "mixed worst:", {k: f"{v:.1e}" for k, v in sorted(chk.worst.items()) if v})
    bad = {k: v for k, v in chk.worst.items() if v > TOL_MIXED.get(k, TOL_MIXED["default"])}
    assert not bad, bad
