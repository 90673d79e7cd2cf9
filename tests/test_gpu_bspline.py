"""The "bspline" tables of versions <= 1.1 (poly_table.hpp:117-135: three cubic B-splines
through the node values of f, f', f'') on the GPU: FP64 results against the oracle within
the parity bound, the benchmark S Part A6 bspline golden values (smoke.json, rel 1e-7), a
short NPT trajectory, mixed precision within its tolerances with the net force at round-off,
and the device tables against the host evaluator."""

import ctypes as C
import json
import os
from dataclasses import replace

import numpy as np
import pytest

from helpers import dynamics_case, gpu, gpu_atoms, oracle, rel_err, static_case
from test_gpu_mixed import check as check_mixed
from test_gpu_parity import TOL, compare_state

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "smoke_static.json")))


def _bs(c):
    return replace(c, interpolation="bspline")


def test_bspline_static_matches_oracle_and_golden():
    from mdelast_b200.units import Units as U
    c = _bs(static_case())
    g, o = gpu(c), oracle(c)
    compare_state(g, o, TOL)
    CB = np.array(g.born_elasticity_tensor) / 1e10
    CB = np.where(CB == 0.0, CB.T, CB)
    vals = {
        "static_epot_eV_per_atom": g.epot_atom / U.ev,
        "static_pressure_GPa": g.pressure / 1e10,
        "static_CB11_GPa": np.mean([CB[0, 0], CB[1, 1], CB[2, 2]]),
        "static_CB12_GPa": np.mean([CB[0, 1], CB[0, 2], CB[1, 2]]),
        "static_CB44_GPa": np.mean([CB[3, 3], CB[4, 4], CB[5, 5]]),
        "laplacian_eV_A2": g.total_laplacian / (U.ev / U.angstrom**2),
        "static_T_conf_K": 1.0 / g.temperature_conf_inverse,
    }
    for k, v in vals.items():
        assert abs(v / GOLD["bspline"][k] - 1.0) < GOLD["rel_tol"], (k, v)


def test_bspline_npt_trajectory():
    c = _bs(dynamics_case(nside=4, n_zn=15, ensemble=2))
    g, o = gpu(c), oracle(c)
    for _ in range(10):
        g.integrate()
    o.integrate(10)
    compare_state(g, o, 1e-9)


def test_bspline_mixed_precision():
    c = _bs(static_case())
    g = gpu(c, precision="mixed")
    check_mixed(g, oracle(c))
    F = gpu_atoms(g, "forces")
    assert np.abs(F.sum(0)).max() / np.abs(F).max() < 1e-12


def test_bspline_device_tables_match_host():
    """mdelast_table_eval_device (the kernels' table code) against the host evaluator on
    a pair table, an electron-density table and an embedding table in "bspline" mode."""
    from helpers import tables
    t = tables()
    lib = C.CDLL(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                              "mdelast_b200", "lib", "libmdelast_cuda.so"))
    D, P = C.POINTER(C.c_double), C.c_void_p
    lib.mdelast_pair_table_create.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int64,
                                              D, D, D, C.c_int, C.POINTER(P)]
    lib.mdelast_eam_create.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_int64, D, D, D, C.c_int64, D, D, D, C.c_int,
                                       C.POINTER(P)]
    lib.mdelast_table_eval_device.argtypes = [P, P, C.c_int, D, C.c_int64, D]
    lib.mdelast_pair_eval.argtypes = [P, C.c_double, D]
    lib.mdelast_eam_eval.argtypes = [P, C.c_int, C.c_double, D]
    arr = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    phi, dphi, d2phi = arr(t.phi[0]), arr(t.dphi[0]), arr(t.d2phi[0])
    pair = P()
    assert lib.mdelast_pair_table_create(t.rcut, 0.0, t.dr, len(phi), phi.ctypes.data_as(D),
                                         dphi.ctypes.data_as(D), d2phi.ctypes.data_as(D), 1,
                                         C.byref(pair)) == 0
    rho, drho, d2rho = arr(t.rho[0]), arr(t.drho_dr[0]), arr(t.d2rho_dr2[0])
    F, dF, d2F = arr(t.F[0]), arr(t.dF[0]), arr(t.d2F[0])
    eam = P()
    assert lib.mdelast_eam_create(t.rcut, t.rhomax, t.dr, t.drho, len(rho),
                                  rho.ctypes.data_as(D), drho.ctypes.data_as(D),
                                  d2rho.ctypes.data_as(D), len(F), F.ctypes.data_as(D),
                                  dF.ctypes.data_as(D), d2F.ctypes.data_as(D), 1,
                                  C.byref(eam)) == 0
    xr = np.linspace(0.5 * t.rcut, t.rcut * 0.999, 300)
    xf = np.linspace(0.01 * t.rhomax, 0.9 * t.rhomax, 300)
    for which, x in [(0, xr), (1, xr), (2, xf)]:
        out = np.zeros((len(x), 3))
        rc = lib.mdelast_table_eval_device(pair if which == 0 else None,
                                           None if which == 0 else eam, which,
                                           x.ctypes.data_as(D), len(x), out.ctypes.data_as(D))
        assert rc == 0
        ref = np.zeros_like(out)
        for q, xv in enumerate(x):
            if which == 0:
                lib.mdelast_pair_eval(pair, xv, ref[q].ctypes.data_as(D))
            else:
                for d in range(3):
                    v = C.c_double()
                    lib.mdelast_eam_eval(eam, 3 * (which - 1) + d, xv, C.byref(v))
                    ref[q, d] = v.value
        assert rel_err(out, ref) < 1e-12, which
