"""Readers for LAMMPS SETFL embedded-atom potential files.

They restate the node-array construction of mdelast's loader
(``src/python/get_potential.py:58-147`` for multi-element ``*.eam.alloy`` files and
``:150-257`` for the single-element ``*.eam.alloy.txt`` form). Each numpy/scipy
operation and its argument units are the same, so the node arrays handed to the
tables are bit-identical to the ones the reference builds its ``TablePotential`` and
``EAM`` objects from:

* values are converted to CGS exactly as the reference does (``Units.ev``,
  ``Units.angstrom``);
* node derivatives come from ``scipy.interpolate.UnivariateSpline(k=5, s=0)``
  (``get_potential.py:49-55``);
* pair blocks are read in SETFL order 11, 21, 22, 31, ... into slot
  ``j(j+1)/2 + i`` (``get_potential.py:122-145``), and ``phi = (r phi)/r`` with
  ``phi[0] = phi[1]``.

The reader returns plain arrays (:class:`SetflTables`). :func:`make_objects` turns
them into the ``TablePotential``/``EAM`` objects of a ``md_driver_module``.
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


def _tokens(lines, start):
    """Yield (line_index, token) for whitespace tokens from line ``start`` on."""
    for li in range(start, len(lines)):
        for tok in lines[li].split():
            yield li, tok


def read_eam_alloy(path) -> SetflTables:
    """Multi-element SETFL reader (``get_potential.py:58-147``)."""
    with open(path, "r") as f:
        lines = f.readlines()
    header_lines = 3
    element_info = lines[header_lines].split()
    num_elements = int(element_info[0])
    elements = [[element_info[i]] for i in range(1, num_elements + 1)]
    param_line = lines[header_lines + 1].split()
    Nrho = int(param_line[0])
    drho = float(param_line[1]) / Units.angstrom**3
    Nr = int(param_line[2])
    dr = float(param_line[3]) * Units.angstrom
    r_grid = np.linspace(0.0, dr * (Nr - 1.0), Nr)  # cm
    rho_grid = np.linspace(0.0, drho * (Nrho - 1.0), Nrho)

    # The file is a sequence of numbers after each element's header line. Collect the
    # numeric blocks line-wise so that one or several values per line both work.
    index = 5
    F_all, dF_all, d2F_all, rho_all, drho_all, d2rho_all = [], [], [], [], [], []
    for i in range(num_elements):
        atomic_number, atomic_weight, a_lattice = [
            float(s) for s in lines[index].split("\n")[0].split()[:-1]
        ]
        elements[i].extend([atomic_number, atomic_weight, a_lattice])
        index += 1
        vals, index = _read_numbers(lines, index, Nrho + Nr)
        F = np.array(vals[:Nrho]) * Units.ev
        rho = np.array(vals[Nrho:Nrho + Nr]) / Units.angstrom**3
        drhodr, d2rhodr2 = get_derivatives(x=r_grid, y=rho)
        dFdrho, d2Fdrho = get_derivatives(x=rho_grid, y=F)
        F_all.append(F); dF_all.append(dFdrho); d2F_all.append(d2Fdrho)
        rho_all.append(rho); drho_all.append(drhodr); d2rho_all.append(d2rhodr2)
    npot = num_elements * (num_elements + 1) // 2
    phi_all = [None] * npot
    dphi_all = [None] * npot
    d2phi_all = [None] * npot
    i, j = 0, 0
    with np.errstate(divide="ignore", invalid="ignore"):
        for _ in range(npot):
            pot_index = j * (j + 1) // 2 + i
            vals, index = _read_numbers(lines, index, Nr)
            phir = np.array(vals)
            phi = phir / r_grid * Units.ev * Units.angstrom
            phi[0] = phi[1]
            dphidr, d2phidr2 = get_derivatives(x=r_grid, y=phi)
            phi_all[pot_index], dphi_all[pot_index], d2phi_all[pot_index] = phi, dphidr, d2phidr2
            if i == j:
                j += 1
                i = 0
            else:
                i += 1
    return SetflTables(
        elements=elements, n_r=Nr, dr=dr, n_rho=Nrho, drho=drho,
        rcut=float(r_grid[-1]), rhomax=float(rho_grid[-1]),
        rmin_fatal=1e-2 * Units.angstrom,
        phi=np.array(phi_all), dphi=np.array(dphi_all), d2phi=np.array(d2phi_all),
        rho=np.array(rho_all), drho_dr=np.array(drho_all), d2rho_dr2=np.array(d2rho_all),
        F=np.array(F_all), dF=np.array(dF_all), d2F=np.array(d2F_all),
        source=str(path),
    )


def _read_numbers(lines, index, count):
    """Read ``count`` numbers starting at line ``index``; return (values, next line)."""
    vals = []
    li = index
    while len(vals) < count:
        toks = lines[li].split()
        vals.extend(float(t) for t in toks)
        li += 1
    if len(vals) != count:
        raise ValueError(f"SETFL block at line {index + 1}: expected {count} values, "
                         f"a line boundary falls inside the block")
    return vals, li


def read_eam_single(path, a_factor=1.0) -> SetflTables:
    """Single-element ``*.eam.alloy.txt`` reader (``get_potential.py:150-257``), the
    loader of the pure-Cu example. Units follow that function: the r grid is built in
    angstrom and scaled to cm afterwards."""
    with open(path, "r") as f:
        all_lines = f.readlines()
    line = all_lines[5].split("\n")[0].split()[:-1]
    atomic_number, atomic_weight, a_lattice = [float(s) for s in line]
    params = np.loadtxt(path, skiprows=4, max_rows=1)[:]
    Nrho, drho, Nr, dr, rcut = params
    Nrho = int(Nrho)
    Nr = int(Nr)
    r_grid = np.linspace(0.0, dr * (Nr - 1.0), Nr)  # angstrom
    rho_grid = np.linspace(0.0, drho * (Nrho - 1.0), Nrho)  # angstrom**-3
    data = np.loadtxt(path, skiprows=6)
    if not (len(data.shape) == 1 and data.shape[0] == Nrho + Nr + Nr):
        raise ValueError("unsupported single-element SETFL layout")
    F = data[:Nrho]
    rho = data[Nrho:Nrho + Nr]
    phir = data[Nrho + Nr:]
    F *= Units.ev
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = phir / r_grid * Units.ev
    phi[0] = phi[1]
    dr *= Units.angstrom
    rcut *= Units.angstrom
    r_grid *= Units.angstrom
    drho /= Units.angstrom**3
    rho /= Units.angstrom**3
    rho_grid /= Units.angstrom**3
    dphidr, d2phidr2 = get_derivatives(x=r_grid, y=phi)
    drhodr, d2rhodr2 = get_derivatives(x=r_grid, y=rho)
    dFdrho, d2Fdrho = get_derivatives(x=rho_grid, y=F)
    return SetflTables(
        elements=[["Cu", atomic_number, atomic_weight, a_lattice]],
        n_r=Nr, dr=float(dr), n_rho=Nrho, drho=float(drho),
        rcut=float(r_grid[-1]), rhomax=float(rho_grid[-1]),
        rmin_fatal=1e-2 * Units.angstrom,
        phi=phi[None, :], dphi=dphidr[None, :], d2phi=d2phidr2[None, :],
        rho=rho[None, :], drho_dr=drhodr[None, :], d2rho_dr2=d2rhodr2[None, :],
        F=F[None, :], dF=dFdrho[None, :], d2F=d2Fdrho[None, :],
        source=str(path), meta={"a_lattice": a_lattice * Units.angstrom * a_factor},
    )


def read_setfl(path) -> SetflTables:
    """Dispatch on the file name as the reference's two loaders are used:
    ``*.eam.alloy.txt`` single-element form, otherwise the multi-element reader."""
    if str(path).endswith("eam.alloy.txt"):
        return read_eam_single(path)
    return read_eam_alloy(path)


def find_potential(name: str):
    """Locate a potential file by name: ``$MDELAST_POTENTIALS``, then the copy the oracle
    build recipe places in ``oracle/_ref/potentials``. Returns None when absent."""
    here = os.path.dirname(os.path.abspath(__file__))
    cands = []
    env = os.environ.get("MDELAST_POTENTIALS")
    if env:
        cands.append(os.path.join(env, name))
    cands.append(os.path.join(here, "..", "oracle", "_ref", "potentials", name))
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
