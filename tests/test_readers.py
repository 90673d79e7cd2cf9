"""The SETFL readers of ``mdelast_b200.potentials`` against the reference's own loaders
(``get_potential.py:58-257``): every node array handed to ``TablePotential`` and ``EAM``
must be bit-identical (sha256 of the float64 bytes) and every scalar exact, for the three
potentials mdelast ships (when their files are present) and for seeded synthetic files in
the three layouts the loaders accept. The fixture ``golden/reader_pins.json`` was made by
``golden/make_reader_golden.py`` running the reference's loader."""

import json
import os
import sys

import pytest

from mdelast_b200 import potentials as P

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from reader_record import element_record, recording_module  # noqa: E402
import synthetic_setfl  # noqa: E402

PINS = json.load(open(os.path.join(HERE, "golden", "reader_pins.json")))["pins"]


@pytest.fixture(scope="module")
def synth_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("setfl")
    return synthetic_setfl.write_all(str(d))


def _split(records):
    return ([r for r in records if r["kind"] == "TablePotential"],
            [r for r in records if r["kind"] == "EAM"])


@pytest.mark.parametrize("key", sorted(PINS))
def test_reader_matches_reference_loader(key, synth_dir):
    name, interp = key.split("|")
    path = synth_dir.get(name) or P.find_potential(name)
    if path is None:
        pytest.skip(f"{name} not staged (mdelast_b200/data/potentials or $MDELAST_POTENTIALS)")
    t = P.read_setfl(path)
    log = []
    elements, _, _ = P.make_objects(recording_module(log), t, interp)
    pin = PINS[key]
    pots, eams = _split(log)
    ref_pots, ref_eams = _split(pin["objects"])
    assert len(pots) == len(ref_pots) and len(eams) == len(ref_eams)
    for mine, ref in zip(pots + eams, ref_pots + ref_eams):
        assert mine == ref, f"{key}: {mine['kind']} differs from the reference loader"
    if "elements" in pin:
        assert element_record(elements) == pin["elements"]
    else:
        assert float.hex(float(elements[0][2])) == pin["atomic_weight"]
        assert float.hex(float(t.meta["a_lattice"])) == pin["a_lattice"]


def test_fs_core_fill_replaced(synth_dir):
    t = P.read_setfl(synth_dir["synth1.eam.fs.txt"])
    n = synthetic_setfl.FS_FILL_NODES
    assert (t.rho[0, :n] == t.rho[0, n]).all()
    assert not (t.phi[0] > 1e10).any()


def test_block_boundary_inside_line(tmp_path):
    # values may run on across lines; a block that ends inside a line still parses
    p = synthetic_setfl.write_all(str(tmp_path))["synth3.eam.alloy"]
    lines = open(p).read().split("\n")
    head, body = lines[:6], lines[6:]
    packed = head[:5] + [head[5]] + [" ".join(body[k:min(k + 3, 1000)]) for k in range(0, 1000, 3)]
    # element 1's F and rho blocks (1000 values) are now three to a line, the last line
    # holding one value; the rest of the file follows unchanged
    packed += body[1000:]
    q = tmp_path / "packed.eam.alloy"
    q.write_text("\n".join(packed))
    a, b = P.read_setfl(p), P.read_setfl(str(q))
    assert (a.rho == b.rho).all() and (a.F == b.F).all() and (a.phi == b.phi).all()
