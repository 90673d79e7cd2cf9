"""A stand-in for ``md_driver_module`` that records what a potential loader hands to the
``TablePotential`` and ``EAM`` constructors, as sha256 digests of the float64 node arrays
and the exact scalars. Used by ``make_reader_golden.py`` (with the reference's loader) and
by ``tests/test_readers.py`` (with this package's reader), so both sides are digested the
same way."""

import hashlib
import types

import numpy as np

from mdelast_b200.units import Units


def digest(a) -> str:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return hashlib.sha256(a.astype("<f8").tobytes()).hexdigest()


def _scalar(x):
    return float.hex(float(x))


def recording_module(log):
    """A module whose constructors append one record each to ``log``."""

    class TablePotential:
        def __init__(self, rcut, rmin_fatal, dr, V, dV, d2V, interpolation="quintic"):
            log.append({"kind": "TablePotential", "rcut": _scalar(rcut),
                        "rmin_fatal": _scalar(rmin_fatal), "dr": _scalar(dr), "n": len(V),
                        "V": digest(V), "dV": digest(dV), "d2V": digest(d2V),
                        "interpolation": interpolation})

    class EAM:
        def __init__(self, rcut, rhomax_fatal, dr, drho, rho, drhodr, d2rhodr2, F, dFdrho,
                     d2Fdrho2, interpolation="quintic"):
            log.append({"kind": "EAM", "rcut": _scalar(rcut), "rhomax": _scalar(rhomax_fatal),
                        "dr": _scalar(dr), "drho": _scalar(drho), "n_r": len(rho),
                        "n_rho": len(F), "rho": digest(rho), "drhodr": digest(drhodr),
                        "d2rhodr2": digest(d2rhodr2), "F": digest(F), "dF": digest(dFdrho),
                        "d2F": digest(d2Fdrho2), "interpolation": interpolation})

    class LennardJones:
        def __init__(self, *a):
            log.append({"kind": "LennardJones"})

    m = types.ModuleType("md_driver_module")
    m.TablePotential, m.EAM, m.LennardJones, m.Units = TablePotential, EAM, LennardJones, Units
    return m


def element_record(elements):
    return [[e[0]] + [_scalar(x) for x in e[1:4]] for e in elements]
