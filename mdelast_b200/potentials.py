"""Readers for LAMMPS SETFL (and single-element Finnis-Sinclair) EAM potential files.

One tokenizer (:func:`_parse_setfl`) reads the layout, with values one or several to a
line. Two unit conversions then follow the two loaders of mdelast, because their
operation orders differ and the node arrays must be the reference's bit for bit:

* :func:`read_eam_alloy`: the alloy loader (``src/python/get_potential.py:58-147``),
  grids built in cgs, ``phi = (r phi) / r_cm * eV * angstrom``;
* :func:`read_eam_single`: the single-element loader (``get_potential.py:150-257``) of
  the pure-Cu example, grids built in angstrom, ``phi = (r phi) / r_A * eV``, then the
  grids and densities converted to cgs; ``*.eam.fs.txt`` files get the core-fill
  replacement of that loader.

Node derivatives come from ``scipy.interpolate.UnivariateSpline(k=5, s=0)``
(``get_potential.py:49-55``); pair blocks go to slot ``j(j+1)/2 + i``
(``get_potential.py:122-145``) and ``phi[0] = phi[1]``. ``tests/test_readers.py`` checks
every array against digests of the reference loader's output.

The readers return plain arrays (:class:`SetflTables`). :func:`make_objects` turns them
into the ``TablePotential``/``EAM`` objects of a ``md_driver_module``.
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np
from scipy.interpolate import UnivariateSpline

from .units import Units

INTERPOLATIONS = ("quintic", "bspline")
DEFAULT_INTERPOLATION = "quintic"


def get_derivatives(x, y):
    """First and second derivatives of the exact quintic spline through (x, y)
    (``get_potential.py:49-55``)."""
    spl = UnivariateSpline(x=x, y=y, k=5, s=0)
    return spl.derivative(n=1)(x), spl.derivative(n=2)(x)


@dataclass
class SetflTables:
    """Node arrays of one potential, CGS units, ready for the table constructors.

    ``phi*`` rows are pair slots ``j(j+1)/2 + i`` (i <= j); ``rho*``/``F*`` rows are
    element types in file order. ``elements`` rows are
    ``[symbol, atomic_number, atomic_weight, lattice_constant_angstrom]``.
    """

    elements: list
    n_r: int
    dr: float
    n_rho: int
    drho: float
    rcut: float            # r_grid[-1]: the cutoff the reference passes to both tables
    rhomax: float          # rho_grid[-1]: EAM rhomax_fatal
    rmin_fatal: float
    phi: np.ndarray
    dphi: np.ndarray
    d2phi: np.ndarray
    rho: np.ndarray
    drho_dr: np.ndarray
    d2rho_dr2: np.ndarray
    F: np.ndarray
    dF: np.ndarray
    d2F: np.ndarray
    source: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n_types(self) -> int:
        return self.rho.shape[0]

    @property
    def masses(self):
        """Atomic masses in grams (atomic weight / Avogadro)."""
        return [e[2] / Units.Navogadro for e in self.elements]


@dataclass
class _SetflText:
    """The numbers of one SETFL (or single-element Finnis-Sinclair) file, in file units:
    eV, angstrom, r*phi in eV angstrom. ``pair_rphi`` keeps the file's block order."""

    elements: list         # [symbol, Z, atomic weight, lattice constant (angstrom)]
    n_rho: int
    d_rho: float
    n_r: int
    d_r: float
    embed: list            # F(rho) per element
    density: list          # rho(r) per element
    pair_rphi: list        # r * phi(r), blocks 11, 21, 22, 31, ...


class _NumberStream:
    """Numbers of a text file read one after the other across line boundaries, with the
    line-level access that element header lines need."""

    def __init__(self, lines, first_line):
        self._lines = lines
        self._li = first_line
        self._pending = []

    def header_line(self):
        if self._pending:
            raise ValueError(f"element header expected at a line start (line {self._li})")
        line = self._lines[self._li].split()
        self._li += 1
        return line

    def take(self, count):
        out = np.empty(count)
        k = 0
        while k < count:
            if not self._pending:
                if self._li >= len(self._lines):
                    raise ValueError(f"file ends {count - k} numbers short of a block")
                self._pending = self._lines[self._li].split()[::-1]
                self._li += 1
                continue
            out[k] = float(self._pending.pop())
            k += 1
        return out


def _parse_setfl(path) -> _SetflText:
    """Parse the LAMMPS ``setfl`` layout: three comment lines, the element line, the grid
    line ``Nrho drho Nr dr rcut``, then per element a header ``Z mass a lattice`` followed by
    F(rho) and rho(r), then the pair blocks r*phi(r). Values may sit one or several to a
    line; blocks need not start on a new line."""
    with open(path) as fh:
        lines = fh.readlines()
    head = lines[3].split()
    n_el = int(head[0])
    symbols = head[1:1 + n_el]
    grid = lines[4].split()
    n_rho, n_r = int(grid[0]), int(grid[2])
    d_rho, d_r = float(grid[1]), float(grid[3])
    stream = _NumberStream(lines, 5)
    elements, embed, density = [], [], []
    for sym in symbols:
        z, weight, a0 = (float(x) for x in stream.header_line()[:3])
        elements.append([sym, z, weight, a0])
        embed.append(stream.take(n_rho))
        density.append(stream.take(n_r))
    pair = [stream.take(n_r) for _ in range(n_el * (n_el + 1) // 2)]
    return _SetflText(elements, n_rho, d_rho, n_r, d_r, embed, density, pair)


def _pair_slot_order(n_el):
    """Slot ``j(j+1)/2 + i`` of each file block (blocks run 11, 21, 22, 31, 32, 33, ...,
    i.e. (i, j) with i <= j and j the outer index; ``md_driver.cpp:341-343``)."""
    return [j * (j + 1) // 2 + i for j in range(n_el) for i in range(j + 1)]


FS_FILL = 1e12       # placeholder the Mendelev Cu2 FS file uses inside the core region


def _fill_core(values):
    """Finnis-Sinclair tables of the Mendelev Cu file fill the innermost nodes of rho(r)
    and r*phi(r) with 1e12; the reference replaces that run by the first real value
    (``get_potential.py:186-211``, where the run is the first 167 nodes)."""
    n = 0
    while n < len(values) and values[n] == FS_FILL:
        n += 1
    if 0 < n < len(values):
        values[:n] = values[n]
    return values


def read_eam_alloy(path) -> SetflTables:
    """Multi-element SETFL potential with the unit conversions of the reference's alloy
    loader (``get_potential.py:58-147``): the grids are built in cgs, r*phi is divided by
    the cgs radius and scaled by eV and angstrom afterwards."""
    f = _parse_setfl(path)
    A3 = Units.angstrom**3
    drho = f.d_rho / A3
    dr = f.d_r * Units.angstrom
    r_grid = np.linspace(0.0, dr * (f.n_r - 1.0), f.n_r)
    rho_grid = np.linspace(0.0, drho * (f.n_rho - 1.0), f.n_rho)
    embed = [F * Units.ev for F in f.embed]
    dens = [rho / A3 for rho in f.density]
    d_dens = [get_derivatives(x=r_grid, y=rho) for rho in dens]
    d_embed = [get_derivatives(x=rho_grid, y=F) for F in embed]
    n_pot = len(f.pair_rphi)
    phi_s, dphi_s, d2phi_s = [None] * n_pot, [None] * n_pot, [None] * n_pot
    with np.errstate(divide="ignore", invalid="ignore"):
        for slot, rphi in zip(_pair_slot_order(len(f.elements)), f.pair_rphi):
            phi = rphi / r_grid * Units.ev * Units.angstrom
            phi[0] = phi[1]
            phi_s[slot] = phi
            dphi_s[slot], d2phi_s[slot] = get_derivatives(x=r_grid, y=phi)
    return SetflTables(
        elements=f.elements, n_r=f.n_r, dr=dr, n_rho=f.n_rho, drho=drho,
        rcut=float(r_grid[-1]), rhomax=float(rho_grid[-1]),
        rmin_fatal=1e-2 * Units.angstrom,
        phi=np.array(phi_s), dphi=np.array(dphi_s), d2phi=np.array(d2phi_s),
        rho=np.array(dens), drho_dr=np.array([d[0] for d in d_dens]),
        d2rho_dr2=np.array([d[1] for d in d_dens]),
        F=np.array(embed), dF=np.array([d[0] for d in d_embed]),
        d2F=np.array([d[1] for d in d_embed]),
        source=str(path),
    )


def read_eam_single(path, a_factor=1.0) -> SetflTables:
    """Single-element potential (``*.eam.alloy.txt`` setfl or ``*.eam.fs.txt``
    Finnis-Sinclair) with the unit conversions of the reference's single-element loader
    (``get_potential.py:150-257``, the loader of the pure-Cu example): the grids are built in
    angstrom, r*phi is divided by the angstrom radius and scaled by eV, and the grids and
    densities are converted to cgs afterwards. ``meta["a_lattice"]`` is the file's lattice
    constant times ``a_factor`` in cm, as that loader hands it to ``Material``."""
    f = _parse_setfl(path)
    if len(f.elements) != 1:
        raise ValueError(f"{path}: single-element loader given {len(f.elements)} elements")
    rho_r, rphi = f.density[0], f.pair_rphi[0]
    if str(path).endswith("eam.fs.txt"):
        rho_r, rphi = _fill_core(rho_r.copy()), _fill_core(rphi.copy())
    r_ang = np.linspace(0.0, f.d_r * (f.n_r - 1.0), f.n_r)
    rho_grid_ang = np.linspace(0.0, f.d_rho * (f.n_rho - 1.0), f.n_rho)
    F = f.embed[0] * Units.ev
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = rphi / r_ang * Units.ev
    phi[0] = phi[1]
    A3 = Units.angstrom**3
    r_grid = r_ang * Units.angstrom
    rho = rho_r / A3
    rho_grid = rho_grid_ang / A3
    dphi, d2phi = get_derivatives(x=r_grid, y=phi)
    drho_dr, d2rho_dr2 = get_derivatives(x=r_grid, y=rho)
    dF, d2F = get_derivatives(x=rho_grid, y=F)
    el = f.elements[0]
    return SetflTables(
        elements=[list(el)], n_r=f.n_r, dr=f.d_r * Units.angstrom, n_rho=f.n_rho,
        drho=f.d_rho / A3, rcut=float(r_grid[-1]), rhomax=float(rho_grid[-1]),
        rmin_fatal=1e-2 * Units.angstrom,
        phi=phi[None, :], dphi=dphi[None, :], d2phi=d2phi[None, :],
        rho=rho[None, :], drho_dr=drho_dr[None, :], d2rho_dr2=d2rho_dr2[None, :],
        F=F[None, :], dF=dF[None, :], d2F=d2F[None, :],
        source=str(path), meta={"a_lattice": el[3] * Units.angstrom * a_factor},
    )


def read_setfl(path) -> SetflTables:
    """Pick the loader by file name as the reference's scripts do: the single-element
    loader for ``*.eam.alloy.txt`` and ``*.eam.fs.txt``, the alloy loader otherwise."""
    if str(path).endswith(("eam.alloy.txt", "eam.fs.txt")):
        return read_eam_single(path)
    return read_eam_alloy(path)


PACKAGE_POTENTIALS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                  "potentials")


def find_potential(name: str):
    """Locate a potential file by name: ``$MDELAST_POTENTIALS`` first, then the package's
    ``data/potentials`` directory (filled by ``mdelast_b200.build`` from an mdelast
    checkout; the files' licences keep them out of this repository's history). Returns
    None when absent."""
    cands = []
    env = os.environ.get("MDELAST_POTENTIALS")
    if env:
        cands.append(os.path.join(env, name))
    cands.append(os.path.join(PACKAGE_POTENTIALS, name))
    for c in cands:
        if os.path.isfile(c):
            return os.path.abspath(c)
    return None


def make_objects(mdm, tables: SetflTables, interpolation=None):
    """Build ``(elements, potentials, eams)`` for module ``mdm`` the way
    ``get_EAM_alloy_file`` returns them."""
    interp = DEFAULT_INTERPOLATION if interpolation is None else interpolation
    if interp not in INTERPOLATIONS:
        raise ValueError(f"interpolation must be one of {INTERPOLATIONS}, got {interp!r}")
    t = tables
    eams = [
        mdm.EAM(t.rcut, t.rhomax, t.dr, t.drho, t.rho[k], t.drho_dr[k], t.d2rho_dr2[k],
                t.F[k], t.dF[k], t.d2F[k], interp)
        for k in range(t.n_types)
    ]
    pots = [
        mdm.TablePotential(t.rcut, t.rmin_fatal, t.dr, t.phi[k], t.dphi[k], t.d2phi[k], interp)
        for k in range(t.phi.shape[0])
    ]
    return t.elements, pots, eams
