"""The elastic-constant estimator (molecular_dynamics.py:663-1000) on the CPU: the oracle's
per-sample restatement equals the reference's own perform_thermal_average on the golden
series, and mdelast_elastic_constants (the C-ABI host estimator working from the sums the
device accumulates) reproduces it from Welford sums of the same samples."""

import ctypes as C
import os

import numpy as np
import pytest

from oracle.fluct import elastic_constants, welford

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, "mdelast_b200", "lib", "libmdelast_cuda.so")
GOLD = np.load(os.path.join(HERE, "golden", "fluct_estimator.npz"))
CASES = [(1, "nvt"), (2, "npt")]


class Fluct(C.Structure):
    _fields_ = [("n", C.c_double), ("n_atoms", C.c_double), ("mean", C.c_double * 9),
                ("comoment", C.c_double * 45), ("born_el_mean", C.c_double * 21)]


def _inputs(name):
    g = GOLD
    return dict(born_stress=g[f"{name}_in_born_stress"], born_el=g[f"{name}_in_born_el"],
                V_V0=g[f"{name}_in_V_V0"], etot_atom=g[f"{name}_in_etot_atom"],
                N=int(g["N"]), V0=float(g["V0"]), T=float(g["T"]), P=float(g["P"]),
                n_therm=int(g["n_therm"]))


@pytest.mark.parametrize("ens,name", CASES)
def test_oracle_estimator_equals_reference(ens, name):
    a = _inputs(name)
    r = elastic_constants(a["born_stress"], a["born_el"], a["V_V0"], a["etot_atom"], ens,
                          a["N"], a["V0"], a["T"], a["P"], a["n_therm"])
    assert np.array_equal(r["C"], GOLD[f"{name}_out_C"])
    for k in ["C11", "C12", "C44", "bulk_modulus"]:
        assert r[k] == GOLD[f"{name}_out_{k}"], k
    if ens == 2:
        assert r["compressibility"] == GOLD["npt_out_compressibility"]
        assert r["volume_thermal_expansion"] == GOLD["npt_out_volume_thermal_expansion"]


def fluct_from_samples(born_stress, born_el, V, etot_atom, N):
    """The device's sums, restated: Welford over x = (sigma^B[6], N/V, V, etot_atom)."""
    x = np.vstack([born_stress, N / V, V, etot_atom])
    mean, M = welford(x)
    n = x.shape[1]
    f = Fluct()
    f.n, f.n_atoms = n, N
    f.mean[:] = list(mean)
    f.comoment[:] = list(M)
    iu = np.triu_indices(6)
    f.born_el_mean[:] = list(np.asarray(born_el)[iu[0], iu[1], :].mean(axis=1))
    return f


def _lib():
    if not os.path.exists(LIB):
        pytest.skip("libmdelast_cuda.so not built")
    lib = C.CDLL(LIB)
    lib.mdelast_elastic_constants.argtypes = [C.POINTER(Fluct), C.c_int32, C.c_double,
                                              C.c_double, C.POINTER(C.c_double),
                                              C.POINTER(C.c_double)]
    lib.mdelast_last_error.restype = C.c_char_p
    return lib


@pytest.mark.parametrize("ens,name", CASES)
def test_host_estimator_from_sums_matches_reference(ens, name):
    lib = _lib()
    a = _inputs(name)
    prod = slice(a["n_therm"], None)
    V = a["V_V0"] * a["V0"]
    f = fluct_from_samples(a["born_stress"][:, prod], a["born_el"][:, :, prod], V[prod],
                           a["etot_atom"][prod], a["N"])
    Cm = (C.c_double * 36)()
    sm = (C.c_double * 6)()
    assert lib.mdelast_elastic_constants(C.byref(f), ens, a["T"], a["P"], Cm, sm) == 0
    Cref = GOLD[f"{name}_out_C"]
    scale = np.max(np.abs(Cref))
    assert np.max(np.abs(np.array(Cm[:]).reshape(6, 6) - Cref)) / scale < 1e-9
    for k, i in [("C11", 0), ("C12", 1), ("C44", 2)]:
        assert abs(sm[i] - GOLD[f"{name}_out_{k}"]) / scale < 1e-9, k
    if ens == 2:
        for k, i in [("bulk_modulus", 3), ("compressibility", 4),
                     ("volume_thermal_expansion", 5)]:
            ref = float(GOLD[f"npt_out_{k}"])
            assert abs(sm[i] / ref - 1.0) < 1e-9, (k, sm[i], ref)
    else:
        assert sm[3] == 0.0 and sm[4] == 0.0 and sm[5] == 0.0


def test_host_estimator_needs_two_samples():
    lib = _lib()
    f = Fluct()
    f.n = 1.0
    Cm = (C.c_double * 36)()
    rc = lib.mdelast_elastic_constants(C.byref(f), 1, 300.0, 0.0, Cm, None)
    assert rc == -1 and b"2 samples" in lib.mdelast_last_error()


def test_drain_into_series_mirrors_append_sample():
    """drain_into_series appends what append_sample (molecular_dynamics.py:1218-1238) would,
    into duck-typed series containers."""
    from mdelast_b200.samples import SCALARS, drain_into_series

    class Col(list):
        pass

    class Series:
        def __init__(self):
            self.time = []
            for k in SCALARS + ["stress_tensor", "born_stress_tensor",
                                "born_elasticity_tensor", "V_V0", "L_L0"]:
                setattr(self, k, Col())

    n = 5
    rng = np.random.default_rng(0)
    rec = {k: rng.random(n) for k in SCALARS + ["time", "cycle", "volume"]}
    rec.update(stress_tensor=rng.random((n, 6)), born_stress_tensor=rng.random((n, 6)),
               born_elasticity_tensor=np.triu(rng.random((6, 6)))[None].repeat(n, 0),
               status=np.zeros(n, np.uint32), lost=0)

    class Drv:
        def drain_samples(self):
            return rec

    s = Series()
    assert drain_into_series(Drv(), s, V0=2.0) == n
    assert s.time == list(rec["time"])
    assert s.etot_cons == list(rec["etot_cons"])
    assert np.array_equal(np.array(s.V_V0), rec["volume"] / 2.0)
    assert np.allclose(np.array(s.L_L0) ** 3, rec["volume"] / 2.0)
    assert np.array_equal(np.array(s.born_elasticity_tensor), rec["born_elasticity_tensor"])
    rec["lost"] = 3
    with pytest.raises(RuntimeError):
        drain_into_series(Drv(), Series(), V0=1.0)
