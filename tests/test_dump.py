"""XYZ snapshots: the writer reproduces the reference's MolecularDynamics.dump byte for
byte (golden written by the reference itself), the reader inverts it, and the device-state
handoff equals the reference's text round trip (sample_case/run.py:251-285)."""

import os

import numpy as np

from mdelast_b200.dump import handoff_positions, read_xyz, xyz_text

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "dump_inputs.npz"))
REF = open(os.path.join(HERE, "golden", "dump_ref.xyz")).read()
SPECIES = [str(s) for s in G["species"]]


def _text():
    return xyz_text(G["positions"], G["velocities"], SPECIES, G["types"], float(G["time"]),
                    float(G["a"]), int(G["nside"]))


def test_writer_matches_reference_dump_bytes():
    assert _text() == REF


def test_reader_inverts_writer():
    pos, vel, typ = read_xyz(REF, SPECIES)
    assert np.array_equal(typ, G["types"])
    # angstrom text round trip: exact in angstrom, within one ulp back in cm
    assert np.array_equal(pos / 1e-8, G["positions"] / 1e-8)
    assert np.allclose(pos, G["positions"], rtol=2e-16, atol=0)
    assert np.allclose(vel, G["velocities"], rtol=4e-16, atol=0)


def test_handoff_equals_text_round_trip():
    V_V0 = 1.0123456789
    pos_text, _, _ = read_xyz(REF, SPECIES)
    scale = V_V0 ** (1.0 / 3.0)
    want = pos_text * scale  # what sample_case/run.py:273-279 computes from the file
    got, s = handoff_positions(G["positions"], V_V0)
    assert s == scale and np.array_equal(got, want)
