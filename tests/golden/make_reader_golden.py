"""Generate tests/golden/reader_pins.json: what the reference's own potential loaders
(``src/python/get_potential.py``: ``get_EAM_alloy_file`` and ``get_EAM_file``) hand to the
``TablePotential`` and ``EAM`` constructors, as sha256 digests of every node array and the
exact scalars, for the three potentials mdelast ships and for the seeded synthetic files of
``synthetic_setfl.py`` (a three-element alloy, a single-element setfl and a single-element
Finnis-Sinclair file). ``tests/test_readers.py`` compares this package's reader with them.

    python tests/golden/make_reader_golden.py [path/to/mdelast]
"""

import json
import logging
import os
import sys
import tempfile
import types

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [HERE, ROOT]

from refroot import reference_root  # noqa: E402
from reader_record import element_record, recording_module  # noqa: E402
import synthetic_setfl  # noqa: E402

SHIPPED_ALLOY = ["ZnCu.eam.alloy", "Mishin_updated-Ni-Al-Co-2013.eam.alloy"]
SHIPPED_SINGLE = ["Cu01.eam.alloy.txt"]


def main():
    ref = reference_root(sys.argv[1] if len(sys.argv) > 1 else None)
    log = []
    sys.modules["md_driver_module"] = recording_module(log)
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    sys.path.insert(0, os.path.join(ref, "src", "python"))
    import get_potential
    logging.disable(logging.CRITICAL)
    out = {}
    tmp = tempfile.mkdtemp()
    synth = synthetic_setfl.write_all(tmp)
    jobs = [(n, n, "alloy") for n in SHIPPED_ALLOY] + [(n, n, "single") for n in SHIPPED_SINGLE]
    jobs += [("synth3.eam.alloy", synth["synth3.eam.alloy"], "alloy"),
             ("synth1.eam.alloy.txt", synth["synth1.eam.alloy.txt"], "single"),
             ("synth1.eam.fs.txt", synth["synth1.eam.fs.txt"], "single")]
    for name, arg, kind in jobs:
        for interp in ("quintic", "bspline"):
            del log[:]
            if kind == "alloy":
                elements, _, _ = get_potential.get_EAM_alloy_file(arg, interpolation=interp)
                rec = {"elements": element_record(elements)}
            else:
                mat = get_potential.get_EAM_file(file_name=arg, a_factor=1.0,
                                                 interpolation=interp)
                rec = {"atomic_weight": float.hex(float(mat.atomic_weight[0])),
                       "a_lattice": float.hex(float(mat.a_lattice))}
            rec["objects"] = list(log)
            out[f"{name}|{interp}"] = rec
    path = os.path.join(HERE, "reader_pins.json")
    with open(path, "w") as fh:
        json.dump({"source": "mdelast src/python/get_potential.py (MIT)", "pins": out}, fh,
                  indent=1, sort_keys=True)
    print("wrote", path, len(out), "entries")


if __name__ == "__main__":
    main()
