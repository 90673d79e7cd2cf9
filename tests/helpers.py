"""Test helpers: one description of a cell and its run settings, turned into the oracle
(C restatement), the compiled reference and the GPU driver with identical inputs."""

from __future__ import annotations

import contextlib
import os
from dataclasses import dataclass, field

import numpy as np
import pytest

from mdelast_b200.lattice import fcc_lattice, initial_state, l12_lattice, smoke_static_cell, substitute
from mdelast_b200.potentials import find_potential, make_objects, read_setfl
from mdelast_b200.units import Units as U

_TABLES = {}


def tables(name="ZnCu.eam.alloy"):
    """Node arrays of a potential staged by the build (or under $MDELAST_POTENTIALS);
    skip if absent."""
    if name not in _TABLES:
        path = find_potential(name)
        if path is None:
            pytest.skip(f"potential {name} not staged (python -m mdelast_b200.build)")
        _TABLES[name] = read_setfl(path)
    return _TABLES[name]


@dataclass
class Case:
    tables: object
    positions: np.ndarray
    velocities: np.ndarray
    types: np.ndarray
    box: np.ndarray
    ensemble: int = 0
    coupling: int = 0
    thermo: tuple = (300.0, [1e-30], [0.0], None)
    baro: tuple = (0.0, 1e-30, 0.0)
    baro_thermo: tuple = (300.0, [1e-30], [0.0], 1.0)
    rg: list = field(default_factory=lambda: [(k + 0.5) * 0.01e-8 for k in range(10)])
    Nf: float | None = None
    dt: float = 1e-15
    neighbors: bool = False
    r_skin: float = 1.0
    fatal_conservation: float = 1e3
    interpolation: str = "quintic"

    @property
    def N(self):
        return len(self.positions)

    def kw(self):
        return dict(ensemble=self.ensemble, coupling=self.coupling, thermo=self.thermo,
                    baro=self.baro, baro_thermo=self.baro_thermo, box=self.box, rg=self.rg,
                    Nf=self.Nf if self.Nf is not None else 3.0 * self.N, dt=self.dt,
                    neighbors=self.neighbors, r_skin=self.r_skin,
                    fatal_conservation=self.fatal_conservation)


@contextlib.contextmanager
def quiet_fd1():
    """Silence C-level stdout (the compiled reference prints in its constructor)."""
    import sys
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        yield
    finally:
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)


def oracle(case: Case, which="oracle"):
    from oracle.ref import OracleDriver, RefDriver
    cls = OracleDriver if which == "oracle" else RefDriver
    with quiet_fd1():
        return cls(case.tables, case.positions, case.velocities, case.types,
                   interpolation=case.interpolation, **case.kw())


def gpu(case: Case, precision="fp64"):
    import md_driver_module as m
    t = case.tables
    _, pots, eams = make_objects(m, t, case.interpolation)
    P = [m.Vector3d(*p) for p in case.positions]
    V = [m.Vector3d(*v) for v in case.velocities]
    T, q, p_eta, nf = case.thermo
    kw = case.kw()
    th = m.Thermostat(T, list(q), list(p_eta), kw["Nf"] if nf is None else nf)
    Tb, qb, p_eta_b, nfb = case.baro_thermo
    baro = m.Barostat(case.baro[0], case.baro[1], case.baro[2],
                      m.Thermostat(Tb, list(qb), list(p_eta_b), nfb))
    return m.MDDriver(P, V, m.PotentialVector(pots), m.EAMVector(eams),
                      m.MDDriver.Ensamble(case.ensemble),
                      m.MDDriver.ThermostatCoupling(case.coupling), th, baro,
                      m.Box(case.box), list(case.rg), kw["Nf"], list(t.masses),
                      [int(x) for x in case.types], case.dt, case.neighbors, case.r_skin,
                      case.fatal_conservation, precision=precision)


def static_case(t=None) -> Case:
    """Benchmark S Part A cell (256 atoms, all-pairs force call)."""
    t = t or tables()
    names = [e[0] for e in t.elements]
    pos, typ, L = smoke_static_cell(names)
    drg = 3.6345 / 500 * U.angstrom
    return Case(t, pos, np.zeros_like(pos), typ, np.diag([L] * 3),
                rg=[(k + 0.5) * drg for k in range(10)])


def dynamics_case(t=None, nside=5, n_zn=30, ensemble=1, T=300.0, dt=2e-15, seed=0,
                  a_ang=3.6345, neighbors=True, r_skin=1.2, coupling=0) -> Case:
    """The sample-case protocol on an nside^3 Cu-Zn FCC cell (sample_case/run.py)."""
    t = t or tables()
    names = [e[0] for e in t.elements]
    pos, L = fcc_lattice(nside, a_ang * U.angstrom)
    typ = substitute(len(pos), n_zn, 42, names.index("Cu"), names.index("Zn"))
    mass = np.array(t.masses)[typ]
    st = initial_state(mass, T, T, 5e-14, 5e-13, random_seed=seed)
    drg = a_ang * U.angstrom / 500
    ng = int(L / 2.0 / drg)
    return Case(t, pos, st.velocities, typ, np.diag([L] * 3), ensemble=ensemble,
                coupling=coupling,
                thermo=(T, st.thermo_q, st.thermo_p_eta, st.Nf),
                baro=(1e-10 * U.GPa, st.baro_w, st.baro_p_eps),
                baro_thermo=(T, st.baro_q, st.baro_p_eta, 1.0),
                rg=[(k + 0.5) * drg for k in range(ng)], Nf=st.Nf, dt=dt,
                neighbors=neighbors, r_skin=r_skin)


def l12_case(t=None, n=4, T=5.0, ensemble=1, seed=500) -> Case:
    """L1_2 CuZn3 cell (benchmarks/l12_cuzn3_5K/run.py:78-92), a0 = 3.7816 A."""
    t = t or tables()
    names = [e[0] for e in t.elements]
    pos, typ, L = l12_lattice(3.7816 * U.angstrom, n, names.index("Zn"), names.index("Cu"))
    mass = np.array(t.masses)[typ]
    st = initial_state(mass, T, T, 5e-14, 5e-13, random_seed=seed)
    return Case(t, pos, st.velocities, typ, np.diag([L] * 3), ensemble=ensemble,
                thermo=(T, st.thermo_q, st.thermo_p_eta, st.Nf),
                baro=(1e-10 * U.GPa, st.baro_w, st.baro_p_eps),
                baro_thermo=(T, st.baro_q, st.baro_p_eta, 1.0), Nf=st.Nf, dt=2e-15,
                neighbors=True, r_skin=1.2)


def nialco_case() -> Case:
    """The fixed 500-atom Ni-Al-Co cell of benchmark S Part C (run_smoke.py:281-303)."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "nialco_lammps.npz"))
    t = tables(str(g["potential"]))
    L = float(g["L"]) * U.angstrom
    pos = g["positions"] * U.angstrom
    return Case(t, pos, np.zeros_like(pos), g["types"], np.diag([L] * 3))


def nialco_golden():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "nialco_lammps.npz"))


SCALARS = ["epot_eam_atom", "epot_atom", "ekin_atom", "etot_atom", "etot_cons",
           "virial_proxy", "total_laplacian", "total_force2", "temperature_kin",
           "temperature_conf_inverse", "pressure"]


def gpu_scalars(d) -> dict:
    out = {k: getattr(d, k) for k in ["epot_eam_atom", "epot_atom", "ekin_atom", "etot_atom",
                                      "etot_cons", "total_laplacian", "total_force2",
                                      "temperature_kin", "temperature_conf_inverse",
                                      "pressure", "time"]}
    out["cycle"] = float(d.cycle)
    out["born_stress_tensor"] = np.array(d.born_stress_tensor)
    out["stress_tensor"] = np.array(d.stress_tensor)
    out["born_elasticity_tensor"] = np.array(d.born_elasticity_tensor)
    out["box"] = np.array(d.box.h)
    b = d.barostat
    out["baro_epsilon"], out["baro_p_epsilon"] = b.epsilon, b.p_epsilon
    return out


def rel_err(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


def gpu_atoms(d, field):
    import md_driver_module as m
    code = {"positions": m.ATOM_POSITIONS, "coordinates": m.ATOM_COORDINATES,
            "velocities": m.ATOM_VELOCITIES, "forces": m.ATOM_FORCES, "rho_eam": m.ATOM_RHO,
            "energies_pot": m.ATOM_EPOT, "energies_kin": m.ATOM_EKIN}[field]
    return np.asarray(d.atoms_array(code))


CU01 = "Cu01.eam.alloy.txt"


def cu01_case(nside=5, ensemble=1, T=300.0, dt=1e-15, seed=0, neighbors=True, r_skin=1.2,
              sigma_ang=0.0, displace_seed=2026) -> Case:
    """Pure Cu with the single-element Mishin Cu01 tables (10,000 nodes): the pure-Cu
    example's FCC cell at the file's lattice constant (``examples/cu_300k/run.py:58-78``,
    ``get_EAM_file``), 300 K, dt 1 fs. ``sigma_ang`` > 0 displaces every atom by a seeded
    Gaussian (a static cell with non-zero forces)."""
    t = tables(CU01)
    a = t.meta["a_lattice"]
    pos, L = fcc_lattice(nside, a)
    if sigma_ang > 0:
        rs = np.random.RandomState(displace_seed)
        pos = pos + rs.normal(scale=sigma_ang * U.angstrom, size=pos.shape)
        pos = np.mod(pos + L / 2, L) - L / 2
    typ = np.zeros(len(pos), dtype=int)
    mass = np.array(t.masses)[typ]
    st = initial_state(mass, T, T, 5e-14, 5e-13, random_seed=seed)
    drg = a / 500
    ng = int(L / 2.0 / drg)
    return Case(t, pos, st.velocities, typ, np.diag([L] * 3), ensemble=ensemble,
                thermo=(T, st.thermo_q, st.thermo_p_eta, st.Nf),
                baro=(1e-10 * U.GPa, st.baro_w, st.baro_p_eps),
                baro_thermo=(T, st.baro_q, st.baro_p_eta, 1.0),
                rg=[(k + 0.5) * drg for k in range(ng)], Nf=st.Nf, dt=dt,
                neighbors=neighbors, r_skin=r_skin)
