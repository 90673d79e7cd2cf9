"""A ``md_driver_module`` in Python over the reference's own C++ core (the compiled
``oracle/_ref/libmdelast_ref.so``, through ``oracle/ref.py``). TEST INFRASTRUCTURE ONLY.

The reference's binding (``src/md_driver_module.cpp:16-224``) needs Eigen's pybind11
caster, which this image lacks, so the reference's Python layer cannot import its own
module here. This file gives that layer the same names over the same compiled core, so
that the reference's scripts (``molecular_dynamics.py``, ``get_potential.py``,
``benchmarks/smoke/run_smoke.py``) can run unchanged against the reference physics:
``tests/golden/make_dropin_trace.py`` runs them and records every call they make on the
module, and ``tests/test_dropin_replay.py`` replays those calls.

Only what those scripts use is here: the table and EAM constructors (their node arrays
are collected and handed to the core as one table set), Vector3d, Box, Thermostat,
Barostat, the MDDriver constructor, its state attributes, ``sample_observables`` and
methods, and Units.
"""

from __future__ import annotations

import enum
import os
import sys
from types import ModuleType, SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from mdelast_b200.units import Units  # noqa: E402,F401  (the CGS table of units.hpp:6-24)
from oracle import ref as _ref  # noqa: E402


class Vector3d:
    __slots__ = ("x", "y", "z")

    def __init__(self, x=0.0, y=0.0, z=0.0):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def length2(self):
        return self.x * self.x + self.y * self.y + self.z * self.z

    def length(self):
        return self.length2() ** 0.5

    def __repr__(self):
        return f"({self.x}, {self.y}, {self.z})"


class PotentialValue:
    def __init__(self, V, dVdr, d2Vdr2):
        self.V, self.dVdr, self.d2Vdr2 = V, dVdr, d2Vdr2


class Potential:
    pass


class TablePotential(Potential):
    def __init__(self, rcut, rmin_fatal, dr, V, dV, d2V, interpolation="quintic"):
        self.rcut, self.rmin_fatal, self.dr = float(rcut), float(rmin_fatal), float(dr)
        self.V, self.dV, self.d2V = (np.array(a, dtype=float) for a in (V, dV, d2V))
        self.interpolation = interpolation


class EAM:
    def __init__(self, rcut, rhomax_fatal, dr, drho, rho, drhodr, d2rhodr2, F, dFdrho,
                 d2Fdrho2, interpolation="quintic"):
        self.rcut, self.rhomax_fatal = float(rcut), float(rhomax_fatal)
        self.dr, self.drho = float(dr), float(drho)
        self.rho_t, self.drho_t, self.d2rho_t = (np.array(a, dtype=float)
                                                 for a in (rho, drhodr, d2rhodr2))
        self.F_t, self.dF_t, self.d2F_t = (np.array(a, dtype=float) for a in (F, dFdrho, d2Fdrho2))
        self.interpolation = interpolation


class PotentialVector(list):
    pass


class EAMVector(list):
    pass


class Box:
    def __init__(self, h):
        self.h = np.array(h, dtype=float).reshape(3, 3)

    def volume(self):
        return float(np.linalg.det(self.h))

    def length(self):
        return np.diag(self.h).copy()


class Thermostat:
    def __init__(self, temperature, q, p_eta, Nf):
        self.temperature = float(temperature)
        self.q = np.array(q, dtype=float)
        self.p_eta = np.array(p_eta, dtype=float)
        self.eta = np.zeros(len(self.q))
        self.nchain = len(self.q)
        self.Nf = float(Nf)


class Barostat:
    def __init__(self, pressure, w, p_epsilon, thermostat):
        self.pressure, self.w = float(pressure), float(w)
        self.epsilon, self.p_epsilon = 0.0, float(p_epsilon)
        self.thermostat = thermostat


class BarostatFlex:
    pass


class _Ensamble(enum.IntEnum):
    NVE = 0
    NVT = 1
    NPT = 2
    NPT_FLEX = 3


class _Coupling(enum.IntEnum):
    THERMOSTAT_KINETIC = 0
    THERMOSTAT_CONFIGURATIONAL = 1
    THERMOSTAT_AVERAGE = 2


def _v3(a):
    return [Vector3d(*r) for r in np.asarray(a).reshape(-1, 3)]


class MDDriver:
    _driver_cls = _ref.RefDriver
    Ensamble = _Ensamble
    ThermostatCoupling = _Coupling
    NVE, NVT, NPT, NPT_FLEX = _Ensamble.NVE, _Ensamble.NVT, _Ensamble.NPT, _Ensamble.NPT_FLEX
    THERMOSTAT_KINETIC = _Coupling.THERMOSTAT_KINETIC
    THERMOSTAT_CONFIGURATIONAL = _Coupling.THERMOSTAT_CONFIGURATIONAL
    THERMOSTAT_AVERAGE = _Coupling.THERMOSTAT_AVERAGE

    def __init__(self, positions, velocities, potentials, eams, ensamble, thermostat_coupling,
                 thermostat, barostat, box, rg, Nf, mass, types, dt, neighbors, r_skin,
                 fatal_conservation):
        pots, eams = list(potentials), list(eams)
        p0, n_types = pots[0], len(eams)
        e0 = eams[0]
        tab = SimpleNamespace(
            n_types=n_types, rcut=p0.rcut, rmin_fatal=p0.rmin_fatal, dr=p0.dr, n_r=len(p0.V),
            phi=np.stack([p.V for p in pots]), dphi=np.stack([p.dV for p in pots]),
            d2phi=np.stack([p.d2V for p in pots]), rhomax=e0.rhomax_fatal, drho=e0.drho,
            n_rho=len(e0.F_t), rho=np.stack([e.rho_t for e in eams]),
            drho_dr=np.stack([e.drho_t for e in eams]),
            d2rho_dr2=np.stack([e.d2rho_t for e in eams]), F=np.stack([e.F_t for e in eams]),
            dF=np.stack([e.dF_t for e in eams]), d2F=np.stack([e.d2F_t for e in eams]),
            masses=[float(m) for m in mass])
        if e0.rcut != p0.rcut or e0.dr != p0.dr:
            raise NotImplementedError("pair and EAM tables on different r grids")
        pos = np.array([[v.x, v.y, v.z] for v in positions])
        vel = np.array([[v.x, v.y, v.z] for v in velocities])
        th, ba = thermostat, barostat
        bt = ba.thermostat
        self._d = self._driver_cls(
            tab, pos, vel, np.asarray(types, dtype=np.uint32), ensemble=int(ensamble),
            coupling=int(thermostat_coupling),
            thermo=(th.temperature, list(th.q), list(th.p_eta), th.Nf),
            baro=(ba.pressure, ba.w, ba.p_epsilon),
            baro_thermo=(bt.temperature, list(bt.q), list(bt.p_eta), bt.Nf),
            box=np.asarray(box.h), rg=list(rg), Nf=float(Nf), dt=float(dt),
            neighbors=bool(neighbors), r_skin=float(r_skin),
            fatal_conservation=float(fatal_conservation),
            interpolation=p0.interpolation)
        self.ensamble = _Ensamble(int(ensamble))
        self.thermostat_coupling = _Coupling(int(thermostat_coupling))
        self._th = (th.temperature, th.q.copy(), th.Nf)
        self._bt = (ba.pressure, ba.w, bt.temperature, bt.q.copy(), bt.Nf)
        self.box_initial = Box(box.h)
        self.rg = [float(x) for x in rg]
        self.dt_global = float(dt)
        self.fatal_conservation = float(fatal_conservation)
        self.mass = [float(m) for m in mass]
        self.types = [int(t) for t in types]
        self.Nparticles_per_type = [self.types.count(k) for k in range(n_types)]
        self._sample = True
        self._npart = n_types * (n_types + 1) // 2
        self._gr = np.zeros(len(self.rg))
        self._grp = np.zeros((self._npart, len(self.rg)))

    # state
    def _s(self):
        return self._d.scalar_dict()

    def __getattr__(self, name):
        if name in _SCALARS:
            return float(self._s()[name])
        raise AttributeError(name)

    @property
    def cycle(self):
        return int(self._s()["cycle"])

    @property
    def born_stress_tensor(self):
        return self._s()["born_stress_tensor"]

    @property
    def stress_tensor(self):
        return self._s()["stress_tensor"]

    @property
    def born_elasticity_tensor(self):
        return self._s()["born_elasticity_tensor"]

    @property
    def box(self):
        return Box(self._s()["box"])

    @property
    def thermostat(self):
        T, q, Nf = self._th
        p, e = self._d.chain(0)
        t = Thermostat(T, q, p, Nf)
        t.eta = e
        return t

    @property
    def barostat(self):
        P, w, Tb, qb, Nfb = self._bt
        p, e = self._d.chain(1)
        t = Thermostat(Tb, qb, p, Nfb)
        t.eta = e
        s = self._s()
        b = Barostat(P, w, s["baro_p_epsilon"], t)
        b.epsilon = s["baro_epsilon"]
        return b

    @property
    def positions(self):
        return _v3(self._d.atoms("positions"))

    @property
    def coordinates(self):
        return _v3(self._d.atoms("coordinates"))

    @property
    def velocities(self):
        return _v3(self._d.atoms("velocities"))

    @property
    def forces(self):
        return _v3(self._d.atoms("forces"))

    @property
    def rho_eam(self):
        return list(self._d.atoms("rho_eam"))

    @property
    def energies_pot(self):
        return list(self._d.atoms("energies_pot"))

    @property
    def energies_kin(self):
        return list(self._d.atoms("energies_kin"))

    @property
    def gr(self):
        return list(self._gr)

    @property
    def gr_partial(self):
        return [list(r) for r in self._grp]

    @property
    def sample_observables(self):
        return self._sample

    @sample_observables.setter
    def sample_observables(self, flag):
        self._sample = bool(flag)
        self._d.set_sample_observables(self._sample)

    # methods
    def integrate(self):
        self._d.integrate(1)

    def calculate_neighbors(self):
        self._d.calculate_neighbors()

    def _pc(self, mode):
        gr, grp = self._d.pair_correlation(mode)
        if mode in (0, 1):
            self._gr = gr
        if mode in (1, 2):
            self._grp = grp

    def calculate_pair_correlation(self):
        self._pc(0)

    def calculate_pair_correlations(self):
        self._pc(1)

    def calculate_partial_pair_correlation(self):
        self._pc(2)


_SCALARS = {"epot_eam_atom", "epot_atom", "ekin_atom", "etot_atom", "etot_cons",
            "etot_cons_err", "total_laplacian", "total_force2", "temperature_kin",
            "temperature_conf_inverse", "pressure", "time"}


def module(which="ref"):
    """This file as the module object a script imports as ``md_driver_module``: over the
    reference's compiled core (``which="ref"``) or over the C restatement
    (``which="oracle"``, a copy of the module whose MDDriver drives ``OracleDriver``)."""
    this = sys.modules[__name__]
    if which == "ref":
        return this
    clone = ModuleType(__name__ + "_oracle")
    for k in dir(this):
        if not k.startswith("__"):
            setattr(clone, k, getattr(this, k))

    class OracleMDDriver(MDDriver):
        _driver_cls = _ref.OracleDriver

    OracleMDDriver.__name__ = "MDDriver"
    clone.MDDriver = OracleMDDriver
    return clone
