"""Generate tests/golden/dump_ref.xyz and dump_inputs.npz: the reference's own
MolecularDynamics.dump (molecular_dynamics.py:644-662) writing a seeded 32-atom Cu-Zn
state, and that state, for the XYZ writer's byte-for-byte check.

    python tests/golden/make_dump_golden.py /path/to/mdelast
"""

import logging
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    sys.path.insert(0, HERE)
    from refroot import reference_root
    ref = reference_root(sys.argv[1] if len(sys.argv) > 1 else None)
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    sys.path[:0] = [os.path.join(ref, "src", "python"), os.path.join(ROOT, "mdelast_b200", "lib")]
    import md_driver_module as m
    import molecular_dynamics as md
    logging.disable(logging.CRITICAL)
    rng = np.random.RandomState(7)
    n, a, nside = 32, 3.6345e-8, 2
    pos = (rng.random_sample((n, 3)) - 0.5) * nside * a
    vel = rng.normal(0.0, 3e4, (n, 3))
    typ = rng.randint(0, 2, n)
    t = 123 * 2e-15
    o = object.__new__(md.MolecularDynamics)
    tmp = tempfile.mkdtemp()
    o.dump_dir = tmp
    o.dump_counter = 0
    o.Nparticles = n
    o.xyz_lattice_str = f"a= {a / m.Units.angstrom} n= {nside} {nside} {nside}"
    o.driver = types.SimpleNamespace(time=t, positions=[m.Vector3d(*p) for p in pos],
                                     velocities=[m.Vector3d(*v) for v in vel])
    o.material = types.SimpleNamespace(atom_name="Cu-Zn")
    o.Ntypes = [int(x) for x in typ]
    o.dump()
    with open(os.path.join(tmp, "0.xyz")) as f:
        text = f.read()
    with open(os.path.join(HERE, "dump_ref.xyz"), "w") as f:
        f.write(text)
    np.savez(os.path.join(HERE, "dump_inputs.npz"), positions=pos, velocities=vel, types=typ,
             time=t, a=a, nside=nside, species=np.array(["Cu", "Zn"]))
    print("wrote dump_ref.xyz,", len(text), "bytes")


if __name__ == "__main__":
    main()
