"""Potentials whose functions do not share one cutoff: the density functions cut at 0.75 of
the pair cutoff (the module accepts any TablePotential / EAM cutoffs, md_driver.cpp:209-264
and potential.hpp:92-104 test each function's own). The mixed passes then keep their
per-function cutoff tests (the uniform-cutoff specialisation that every setfl potential
takes does not apply): mixed within its tolerances of the oracle with the same cutoffs,
FP64 within 1e-9 at the start and after 20 steps with a list rebuild."""

import copy

import numpy as np
import pytest

from helpers import dynamics_case, gpu_atoms, gpu_scalars, oracle, rel_err
from test_gpu_mixed import check as check_mixed

pytestmark = pytest.mark.gpu


def _gpu(case, precision, eam_rcut):
    import md_driver_module as m
    t = case.tables
    eams = [m.EAM(eam_rcut, t.rhomax, t.dr, t.drho, t.rho[k], t.drho_dr[k], t.d2rho_dr2[k],
                  t.F[k], t.dF[k], t.d2F[k], case.interpolation) for k in range(t.n_types)]
    pots = [m.TablePotential(t.rcut, t.rmin_fatal, t.dr, t.phi[k], t.dphi[k], t.d2phi[k],
                             case.interpolation) for k in range(t.phi.shape[0])]
    kw = case.kw()
    T, q, p_eta, nf = case.thermo
    th = m.Thermostat(T, list(q), list(p_eta), kw["Nf"] if nf is None else nf)
    Tb, qb, p_eta_b, nfb = case.baro_thermo
    baro = m.Barostat(case.baro[0], case.baro[1], case.baro[2],
                      m.Thermostat(Tb, list(qb), list(p_eta_b), nfb))
    return m.MDDriver([m.Vector3d(*p) for p in case.positions],
                      [m.Vector3d(*v) for v in case.velocities], m.PotentialVector(pots),
                      m.EAMVector(eams), m.MDDriver.Ensamble(case.ensemble),
                      m.MDDriver.ThermostatCoupling(case.coupling), th, baro, m.Box(case.box),
                      list(case.rg), kw["Nf"], list(t.masses), [int(x) for x in case.types],
                      case.dt, case.neighbors, case.r_skin, case.fatal_conservation,
                      precision=precision)


def _case():
    c = dynamics_case(nside=6, n_zn=52, ensemble=1)
    c.tables = copy.copy(c.tables)
    c.tables.eam_rcut = 0.75 * c.tables.rcut
    return c


def test_cut_changes_the_density():
    """The cut is felt: the oracle's densities differ from the uniform-cutoff potential's."""
    c = _case()
    rho_cut = oracle(c).atoms("rho_eam")
    rho_full = oracle(dynamics_case(nside=6, n_zn=52, ensemble=1)).atoms("rho_eam")
    assert rel_err(rho_cut, rho_full) > 1e-3


def test_mixed_density_cutoff_below_pair_cutoff():
    c = _case()
    check_mixed(_gpu(c, "mixed", c.tables.eam_rcut), oracle(c))


def test_fp64_density_cutoff_below_pair_cutoff():
    c = _case()
    o = oracle(c)
    g = _gpu(c, "fp64", c.tables.eam_rcut)
    for step in range(2):
        s_g, s_o = gpu_scalars(g), o.scalar_dict()
        for k in ["epot_atom", "epot_eam_atom", "pressure", "born_elasticity_tensor",
                  "total_laplacian"]:
            assert rel_err(s_g[k], s_o[k]) < 1e-9, (step, k)
        for f in ["forces", "rho_eam", "energies_pot"]:
            assert rel_err(gpu_atoms(g, f), o.atoms(f)) < 1e-9, (step, f)
        g.run(20, 20, 1)
        for s in range(20):
            if s % 20 == 0:
                o.calculate_neighbors()
            o.integrate()
