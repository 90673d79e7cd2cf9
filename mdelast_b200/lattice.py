"""Synthetic cells and initial states with the shapes, seeds and random streams the
reference's scripts use, so that runs of this package start from the same inputs.

* ``fcc_lattice``: centred FCC basis with offset 0.25 (``molecular_dynamics.py:578-614``,
  ``sample_case/run.py:50-70``);
* ``smoke_static_cell``: the distorted 256-atom Cu-Zn cell of benchmark S, Part A
  (``benchmarks/smoke/run_smoke.py:91-129``);
* ``substitute``: random substitutional occupation by ``RandomState(seed).choice``
  (``sample_case/run.py:224-227``);
* ``l12_lattice``: L1_2 basis with the 1e-5 distortion
  (``benchmarks/l12_cuzn3_5K/run.py:78-92``);
* ``initial_state``: Maxwell-Boltzmann velocities and the NHC / barostat initial draws
  from the global numpy stream seeded with ``random_seed``
  (``molecular_dynamics.py:318,505,525-543,616-642``).

All returned positions are in cm, velocities in cm/s, masses in g.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .units import Units

FCC_BASIS = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])


def fcc_lattice(nside: int, a: float):
    """FCC positions in a cubic box of edge ``nside * a``, centred on the origin, in the
    loop order of ``MolecularDynamics.build_fcc_lattice``. Returns (positions (N,3), L)."""
    L = nside * a
    out = np.empty((4 * nside**3, 3))
    n = 0
    for i in range(nside):
        for j in range(nside):
            for k in range(nside):
                for m in range(4):
                    out[n, 0] = -L / 2.0 + (i + 0.25 + FCC_BASIS[m, 0]) * a
                    out[n, 1] = -L / 2.0 + (j + 0.25 + FCC_BASIS[m, 1]) * a
                    out[n, 2] = -L / 2.0 + (k + 0.25 + FCC_BASIS[m, 2]) * a
                    n += 1
    return out, L


def _smoke_fcc_angstrom(nside, a):
    pos = np.array([(np.array([i, j, k]) + 0.25 + b) * a
                    for i in range(nside) for j in range(nside)
                    for k in range(nside) for b in FCC_BASIS])
    return pos - nside * a / 2.0


def smoke_static_cell(element_names, a_ang=3.6345, nside=4, n_zn=15, sigma_ang=0.08,
                      seed=2026):
    """Benchmark S Part A cell: returns (positions cm (N,3), types (N,), L cm)."""
    rs = np.random.RandomState(seed)
    pos = _smoke_fcc_angstrom(nside, a_ang)
    pos = pos + rs.normal(scale=sigma_ang, size=pos.shape)
    L = nside * a_ang
    pos = np.mod(pos + L / 2, L) - L / 2
    types = np.full(len(pos), element_names.index("Cu"))
    types[rs.choice(len(pos), size=n_zn, replace=False)] = element_names.index("Zn")
    lengths = np.full(3, L)
    pos = np.mod(pos + lengths / 2, lengths) - lengths / 2
    return pos * Units.angstrom, types.astype(np.uint32), L * Units.angstrom


def substitute(n_atoms: int, n_solute: int, seed: int, host_type: int, solute_type: int):
    """Random substitutional occupation (``sample_case/run.py:224-227``)."""
    types = np.full(n_atoms, host_type, dtype=np.uint32)
    rng = np.random.RandomState(seed)
    for index in rng.choice(n_atoms, size=n_solute, replace=False):
        types[int(index)] = solute_type
    return types


def l12_lattice(a: float, n: int, majority_type: int, minority_type: int, distort=1e-5):
    """L1_2 cell (one minority site at the cube corner, three majority face sites), every
    site shifted by ``distort * a`` (``benchmarks/l12_cuzn3_5K/run.py:78-92``)."""
    L = n * a
    d = a * distort
    basis = [([0.0, 0.0, 0.0], minority_type), ([0.0, 0.5, 0.5], majority_type),
             ([0.5, 0.0, 0.5], majority_type), ([0.5, 0.5, 0.0], majority_type)]
    pos, types = [], []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                for frac, t in basis:
                    pos.append(((i + frac[0]) * a + d - L / 2,
                                (j + frac[1]) * a + d - L / 2,
                                (k + frac[2]) * a + d - L / 2))
                    types.append(t)
    return np.array(pos), np.array(types, dtype=np.uint32), L


@dataclass
class InitialState:
    velocities: np.ndarray  # (N, 3) cm/s
    Nf: float
    thermo_q: np.ndarray
    thermo_p_eta: np.ndarray
    baro_q: np.ndarray
    baro_p_eta: np.ndarray
    baro_w: float
    baro_p_eps: float


def initial_state(mass_per_atom, temperature_initial, temperature_thermostat,
                  tau_thermostat, tau_barostat, random_seed=0, nchains_thermostat=10,
                  nchains_barostat=10, velocities=None) -> InitialState:
    """The draws ``MolecularDynamics.__init__`` makes, in the same order from the same
    global stream (``np.random.seed(random_seed)``), so that a run started here matches
    one started by the reference's Python layer."""
    np.random.seed(random_seed)
    mass = np.asarray(mass_per_atom, dtype=float)
    N = len(mass)
    Nf = 3.0 * (N - 1.0)
    if velocities is None:
        sigmav = np.sqrt(Units.k_boltz * temperature_initial / mass)
        vx = np.random.normal(0.0, sigmav)
        vy = np.random.normal(0.0, sigmav)
        vz = np.random.normal(0.0, sigmav)
        vx -= np.sum(vx * mass) / np.sum(mass)
        vy -= np.sum(vy * mass) / np.sum(mass)
        vz -= np.sum(vz * mass) / np.sum(mass)
        ekin = (3.0 * N - 3.0) * Units.k_boltz * temperature_initial / 2.0
        scale = np.sqrt(ekin / (0.5 * np.sum(mass * (vx**2 + vy**2 + vz**2))))
        vx *= scale
        vy *= scale
        vz *= scale
        velocities = np.stack([vx, vy, vz], axis=1)
    kT = Units.k_boltz * temperature_thermostat
    q = np.ones(nchains_thermostat) * tau_thermostat**2.0 * kT
    q[0] *= Nf
    p_eta = np.random.normal(0.0, np.sqrt(q * kT))
    qb = np.ones(nchains_barostat) * tau_barostat**2.0 * kT
    p_eta_b = np.random.normal(0.0, np.sqrt(qb * kT))
    w = Nf * tau_barostat**2.0 * kT
    p_eps = np.random.normal(0.0, np.sqrt(w * kT))
    return InitialState(np.asarray(velocities, dtype=float), Nf, q, p_eta, qb, p_eta_b,
                        float(w), float(p_eps))
