"""XYZ snapshots in the reference's format and the NPT -> NVT handoff from device state.

``xyz_text`` writes what MolecularDynamics.dump writes (molecular_dynamics.py:644-662):
the atom count, a comment line with the lattice, the extended-XYZ properties and the time
in ps, then one line per atom with its species, position in angstrom and velocity in
angstrom/fs, every number in Python's shortest round-trip form. ``read_xyz`` reads such a
file back. ``handoff_positions`` applies the reference's NPT -> NVT handoff
(sample_case/run.py:251-285: positions of the final NPT snapshot scaled by the production
mean (V/V0)^(1/3)) to positions taken straight from the device, with the same arithmetic
as the text round trip, so no file is needed.
"""

from __future__ import annotations

import numpy as np

ANGSTROM = 1e-8  # units.hpp
PS = 1e-12
FS = 1e-15


def xyz_text(positions, velocities, species, type_of, time_s, a_lattice_cm, nside) -> str:
    """positions, velocities: (N, 3) in cm and cm/s; species: element names by type;
    type_of: the type of every atom; time_s: the driver's time; a_lattice_cm, nside: the
    lattice the cell was built from (its comment line)."""
    head = (f"{len(positions)}\n"
            f"a= {a_lattice_cm / ANGSTROM} n= {nside} {nside} {nside} "
            f"Properties=species:S:1:pos:R:3:vel:R:3 Time={time_s / PS}\n")
    vu = ANGSTROM / FS
    lines = [f"{species[int(t)]} "
             f"{float(p[0]) / ANGSTROM} {float(p[1]) / ANGSTROM} {float(p[2]) / ANGSTROM} "
             f"{float(v[0]) / vu} {float(v[1]) / vu} {float(v[2]) / vu}"
             for p, v, t in zip(positions, velocities, type_of)]
    # print(str_file, file=...) ends the file with one newline
    return head + "\n".join(lines) + "\n"


def write_xyz(path, driver, species, type_of, a_lattice_cm, nside, replica=None):
    """Write the current state of an MDDriver (or of one replica of a BatchedMDDriver)."""
    import md_driver_module as m
    if replica is None:
        pos = np.asarray(driver.atoms_array(m.ATOM_POSITIONS))
        vel = np.asarray(driver.atoms_array(m.ATOM_VELOCITIES))
        t = driver.time
    else:
        pos = np.asarray(driver.atoms(replica, m.ATOM_POSITIONS))
        vel = np.asarray(driver.atoms(replica, m.ATOM_VELOCITIES))
        t = driver.observables(replica)["time"]
    with open(path, "w") as f:
        f.write(xyz_text(pos, vel, species, type_of, t, a_lattice_cm, nside))


def read_xyz(path_or_text, species):
    """(positions cm (N, 3), velocities cm/s (N, 3), types (N,)) from an XYZ snapshot, as
    sample_case/run.py:258-272 reads it."""
    text = path_or_text
    if "\n" not in path_or_text:
        with open(path_or_text) as f:
            text = f.read()
    index = {s: k for k, s in enumerate(species)}
    pos, vel, typ = [], [], []
    for line in text.splitlines()[2:]:
        fields = line.split()
        if len(fields) < 7:
            continue
        pos.append([float(x) * ANGSTROM for x in fields[1:4]])
        vel.append([float(x) * (ANGSTROM / FS) for x in fields[4:7]])
        typ.append(index[fields[0]])
    return np.array(pos), np.array(vel), np.array(typ, dtype=np.int64)


def handoff_positions(positions_cm, V_V0_mean):
    """Positions for the NVT stage: the snapshot's positions through the angstrom text
    round trip ((p / A) * A, exact for Python's round-trip float repr) scaled by
    (V/V0)^(1/3), as sample_case/run.py:273-279 does. Returns (positions, scale)."""
    scale = V_V0_mean ** (1.0 / 3.0)
    p = (np.asarray(positions_cm, dtype=float) / ANGSTROM) * ANGSTROM
    return p * scale, scale
