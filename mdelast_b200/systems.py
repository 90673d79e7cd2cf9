"""Cells, run settings and their drivers for the workloads this package is measured on.

A :class:`Cell` holds one periodic cell and its thermostat/barostat state in the
reference's cgs units. The builders restate the reference's scripts:

* :func:`cuzn_cell` - random substitutional Cu-Zn FCC (``sample_case/run.py:50-70,
  224-227``): the 500-atom sample case, the 13,500-atom 15x15x15 cell, or any size and
  composition;
* :func:`l12_cell` - ordered L1_2 CuZn3 (``benchmarks/l12_cuzn3_5K/run.py:78-92``);
* :func:`pure_cell` - one element on an FCC lattice, the pure-Cu example
  (``examples/cu_300k/run.py:58-78``) with the single-element Cu01 tables;
* :func:`uneven_replicas` - independent cells of 4 n^3 atoms with n uniform in [4, 20], Zn
  fraction uniform in [0, 0.30], temperature uniform in [5, 900] K, separate seeds, drawn
  from one master ``RandomState``.

:func:`make_driver` builds ``md_driver_module.MDDriver`` for one cell and
:func:`make_batch` one ``BatchedMDDriver`` for many.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .lattice import fcc_lattice, initial_state, l12_lattice, substitute
from .potentials import SetflTables, make_objects
from .units import Units as U

A0_CUZN6 = 3.6345  # production lattice constant of 6 at.% Zn [A] (sample_case/run.py:215)
A0_CU = 3.615      # pure Cu (examples/cu_300k)
A0_L12 = 3.7816    # L1_2 CuZn3 at 5 K (benchmarks/l12_cuzn3_5K/run.py)


@dataclass
class Cell:
    positions: np.ndarray       # (N, 3) cm, inside [-L/2, L/2)
    velocities: np.ndarray      # (N, 3) cm/s
    types: np.ndarray           # (N,) uint32
    box: np.ndarray             # (3,) edges, cm
    T: float                    # thermostat temperature, K
    ensemble: int               # 0 NVE, 1 NVT, 2 NPT
    thermo_q: np.ndarray
    thermo_p_eta: np.ndarray
    baro_q: np.ndarray
    baro_p_eta: np.ndarray
    baro_w: float
    baro_p_eps: float
    Nf: float
    pressure: float = 1e-10 * U.GPa
    meta: dict = field(default_factory=dict)

    @property
    def n_atoms(self) -> int:
        return len(self.positions)


def _state(tables, positions, types, L, T, ensemble, seed, meta, mass_T=None):
    """Velocities at T and chain masses at mass_T (default T: the reference's choice,
    Q, W proportional to kT)."""
    mass = np.array(tables.masses)[types]
    st = initial_state(mass, T, T if mass_T is None else mass_T, 5e-14, 5e-13, random_seed=seed)
    return Cell(positions=positions, velocities=st.velocities, types=np.asarray(types, np.uint32),
                box=np.asarray(L, dtype=float), T=T, ensemble=ensemble,
                thermo_q=st.thermo_q, thermo_p_eta=st.thermo_p_eta, baro_q=st.baro_q,
                baro_p_eta=st.baro_p_eta, baro_w=st.baro_w, baro_p_eps=st.baro_p_eps, Nf=st.Nf,
                meta=meta)


def cuzn_cell(tables: SetflTables, nside: int, n_zn: int | None = None, x_zn: float = 0.06,
              T: float = 300.0, a_ang: float = A0_CUZN6, ensemble: int = 1,
              placement_seed: int = 42, velocity_seed: int = 0) -> Cell:
    names = [e[0] for e in tables.elements]
    pos, L = fcc_lattice(nside, a_ang * U.angstrom)
    n = len(pos)
    if n_zn is None:
        n_zn = int(round(x_zn * n))
    types = substitute(n, n_zn, placement_seed, names.index("Cu"), names.index("Zn"))
    return _state(tables, pos, types, [L] * 3, T, ensemble, velocity_seed,
                  {"kind": "cuzn_fcc", "nside": nside, "n_zn": n_zn, "a_ang": a_ang})


def fcc_alloy_cell(tables: SetflTables, nside: int, fractions, T: float = 300.0,
                   a_ang: float = 3.6, ensemble: int = 1, placement_seed: int = 42,
                   velocity_seed: int = 0, mass_T: float | None = None) -> Cell:
    """Random substitutional FCC solid solution of the potential's elements (in file order)
    with the given fractions: round(x_k N) sites of each type (the rest to the last type),
    placed by RandomState(placement_seed).permutation. mass_T, when given, is the
    temperature the thermostat and barostat masses are set for (the target stays T)."""
    pos, L = fcc_lattice(nside, a_ang * U.angstrom)
    n = len(pos)
    x = np.asarray(fractions, dtype=float)
    counts = np.floor(x / x.sum() * n + 0.5).astype(int)
    counts[-1] = n - counts[:-1].sum()
    types = np.repeat(np.arange(len(x), dtype=np.uint32), counts)
    types = types[np.random.RandomState(placement_seed).permutation(n)]
    return _state(tables, pos, types, [L] * 3, T, ensemble, velocity_seed,
                  {"kind": "fcc_alloy", "nside": nside, "counts": counts.tolist(),
                   "a_ang": a_ang}, mass_T=mass_T)


def l12_cell(tables: SetflTables, n: int, T: float = 5.0, ensemble: int = 1,
             velocity_seed: int = 500, a_ang: float = A0_L12) -> Cell:
    names = [e[0] for e in tables.elements]
    pos, types, L = l12_lattice(a_ang * U.angstrom, n, names.index("Zn"), names.index("Cu"))
    return _state(tables, pos, types, [L] * 3, T, ensemble, velocity_seed,
                  {"kind": "l12_cuzn3", "n": n, "a_ang": a_ang})


def pure_cell(tables: SetflTables, nside: int = 5, T: float = 300.0, ensemble: int = 1,
              velocity_seed: int = 0, a_ang: float | None = None) -> Cell:
    """FCC cell of the potential's first element at the file's lattice constant (the
    value ``get_EAM_file`` hands to ``Material``), or ``a_ang``."""
    a = tables.meta.get("a_lattice", A0_CU * U.angstrom) if a_ang is None else a_ang * U.angstrom
    pos, L = fcc_lattice(nside, a)
    types = np.zeros(len(pos), dtype=np.uint32)
    return _state(tables, pos, types, [L] * 3, T, ensemble, velocity_seed,
                  {"kind": "pure_fcc", "nside": nside, "a_ang": a / U.angstrom})


def vegard_a(x_zn: float, T: float) -> float:
    """Starting lattice constant [A]: linear between pure Cu (3.615) and L1_2 CuZn3 (3.7816
    at x = 0.75), with a thermal expansion of 1.7e-5 / K about 300 K."""
    return (A0_CU + (A0_L12 - A0_CU) * x_zn / 0.75) * (1.0 + 1.7e-5 * (T - 300.0))


def uneven_replicas(tables: SetflTables, count: int = 64, master_seed: int = 2026,
                    n_range=(4, 20), x_range=(0.0, 0.30), T_range=(5.0, 900.0),
                    ensemble: int = 1) -> list[Cell]:
    rs = np.random.RandomState(master_seed)
    cells = []
    for k in range(count):
        n = int(rs.randint(n_range[0], n_range[1] + 1))
        x = float(rs.uniform(*x_range))
        T = float(rs.uniform(*T_range))
        place, vel = int(rs.randint(0, 2**31 - 1)), int(rs.randint(0, 2**31 - 1))
        cells.append(cuzn_cell(tables, n, x_zn=x, T=T, a_ang=vegard_a(x, T), ensemble=ensemble,
                               placement_seed=place, velocity_seed=vel))
    return cells


def _thermostats(m, cell: Cell):
    th = m.Thermostat(cell.T, list(cell.thermo_q), list(cell.thermo_p_eta), cell.Nf)
    baro = m.Barostat(cell.pressure, cell.baro_w, cell.baro_p_eps,
                      m.Thermostat(cell.T, list(cell.baro_q), list(cell.baro_p_eta), 1.0))
    return th, baro


def rg_bins(cell: Cell, a_ang: float = A0_CUZN6):
    """g(r) bin centres as MolecularDynamics builds them (molecular_dynamics.py:507-511)."""
    drg = a_ang * U.angstrom / 500.0
    return [(k + 0.5) * drg for k in range(int(min(cell.box) / 2.0 / drg))]


def make_driver(m, tables: SetflTables, cell: Cell, dt=2e-15, neighbors=True, r_skin=1.2,
                precision="fp64", device=0, fatal_conservation=1e3, coupling=0):
    _, pots, eams = make_objects(m, tables)
    th, baro = _thermostats(m, cell)
    return m.MDDriver([m.Vector3d(*p) for p in cell.positions],
                      [m.Vector3d(*v) for v in cell.velocities], m.PotentialVector(pots),
                      m.EAMVector(eams), m.MDDriver.Ensamble(cell.ensemble),
                      m.MDDriver.ThermostatCoupling(coupling), th, baro, m.Box(np.diag(cell.box)),
                      rg_bins(cell), cell.Nf, list(tables.masses), [int(t) for t in cell.types],
                      dt, neighbors, r_skin, fatal_conservation, precision=precision,
                      device=device)


def make_batch(m, tables: SetflTables, cells: list[Cell], dt=2e-15, neighbors=True,
               r_skin=1.2, precision="fp64", device=0, fatal_conservation=1e3, rg=None):
    """One BatchedMDDriver over `cells`; g(r) bins `rg` shared by all replicas (default:
    those of the smallest cell)."""
    _, pots, eams = make_objects(m, tables)
    if rg is None:
        rg = rg_bins(min(cells, key=lambda c: min(c.box)))
    ths, baros = zip(*[_thermostats(m, c) for c in cells])
    return m.BatchedMDDriver([c.positions for c in cells], [c.velocities for c in cells],
                             [np.asarray(c.types, dtype=np.uint32) for c in cells],
                             m.PotentialVector(pots),
                             m.EAMVector(eams), [m.MDDriver.Ensamble(c.ensemble) for c in cells],
                             list(ths), list(baros), [m.Box(np.diag(c.box)) for c in cells],
                             [c.Nf for c in cells], list(tables.masses), dt,
                             neighbors=neighbors, r_skin=r_skin,
                             fatal_conservation=fatal_conservation, precision=precision,
                             device=device, rg=list(rg))
