"""The C-ABI library without a GPU: it loads, exports every entry point include/mdelast.h
declares, builds the quintic tables exactly as the reference (bit for bit against the
oracle's restatement of poly_table.hpp:35-63), and refuses GPU work with
MDELAST_ERR_NO_DEVICE instead of falling back to the CPU."""

import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mdelast_b200", "lib", "libmdelast_cuda.so")
HEADER = os.path.join(ROOT, "include", "mdelast.h")
ORACLE = os.path.join(ROOT, "oracle", "_build", "libmdelast_oracle.so")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mdelast_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        pytest.fail(f"{LIB} is not built (python -m mdelast_b200.build)")
    return C.CDLL(LIB)


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_version(lib):
    assert lib.mdelast_abi_version() == 1


def _pair(lib, h, f, f1, f2, interp=0):
    D = C.POINTER(C.c_double)
    p = C.c_void_p()
    lib.mdelast_pair_table_create.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int64,
                                              D, D, D, C.c_int, C.POINTER(C.c_void_p)]
    rc = lib.mdelast_pair_table_create(10.0, 0.0, h, len(f), f.ctypes.data_as(D),
                                       f1.ctypes.data_as(D), f2.ctypes.data_as(D), interp,
                                       C.byref(p))
    return rc, p


def test_quintic_table_matches_oracle(lib):
    """Host table evaluation (Potential.calculate) against the oracle's restatement."""
    D = C.POINTER(C.c_double)
    rng = np.random.RandomState(3)
    n, h = 41, 0.0034
    f, f1, f2 = rng.normal(size=n), rng.normal(size=n), rng.normal(size=n)
    rc, p = _pair(lib, h, f, f1, f2)
    assert rc == 0
    orc = C.CDLL(ORACLE)
    coef = np.zeros(6 * (n - 1))
    orc.orc_quintic_coefficients(C.c_double(h), n, f.ctypes.data_as(D), f1.ctypes.data_as(D),
                                 f2.ctypes.data_as(D), coef.ctypes.data_as(D))
    lib.mdelast_pair_eval.argtypes = [C.c_void_p, C.c_double, D]
    orc.orc_quintic_eval.argtypes = [D, C.c_int, C.c_double, C.c_double, D]
    xs = np.concatenate([np.linspace(-0.01, n * h + 0.01, 997), [0.0, -0.0, (n - 1) * h,
                                                                 np.nextafter((n - 1) * h, 0)]])
    for x in xs:
        a, b = np.zeros(3), np.zeros(3)
        assert lib.mdelast_pair_eval(p, x, a.ctypes.data_as(D)) == 0
        orc.orc_quintic_eval(coef.ctypes.data_as(D), n - 1, h, x, b.ctypes.data_as(D))
        assert np.array_equal(a, b), x
    # NaN in, NaN out (poly_table.hpp:102-104; tests/test_tables.py:109-112)
    a = np.zeros(3)
    lib.mdelast_pair_eval(p, float("nan"), a.ctypes.data_as(D))
    assert np.isnan(a[0])
    lib.mdelast_pair_destroy(p)


def test_quintic_reproduces_quintic_polynomials(lib):
    """tools/test_poly_table.cpp test 1: a polynomial of degree <= 5 is reproduced."""
    D = C.POINTER(C.c_double)
    h, n = 0.1, 69
    x = np.arange(n) * h
    c = np.array([0.3, -1.1, 0.7, 0.25, -0.05, 0.01])
    f = sum(c[k] * (x - 3) ** k for k in range(6))
    f1 = sum(k * c[k] * (x - 3) ** (k - 1) for k in range(1, 6))
    f2 = sum(k * (k - 1) * c[k] * (x - 3) ** (k - 2) for k in range(2, 6))
    rc, p = _pair(lib, h, f, f1, f2)
    assert rc == 0
    for xv in np.linspace(0.0, (n - 1) * h, 501):
        o = np.zeros(3)
        lib.mdelast_pair_eval(p, C.c_double(xv), o.ctypes.data_as(D))
        ref = [sum(c[k] * (xv - 3) ** k for k in range(6)),
               sum(k * c[k] * (xv - 3) ** (k - 1) for k in range(1, 6)),
               sum(k * (k - 1) * c[k] * (xv - 3) ** (k - 2) for k in range(2, 6))]
        assert np.allclose(o, ref, rtol=1e-10, atol=1e-10)
    lib.mdelast_pair_destroy(p)


def test_bad_tables_are_rejected(lib):
    f = np.ones(1)
    rc, _ = _pair(lib, 0.1, f, f, f)
    assert rc == -1  # MDELAST_ERR_ARGUMENT: fewer than 2 nodes
    f = np.ones(4)
    rc, _ = _pair(lib, 0.1, f, f, f, interp=7)
    assert rc == -1


def test_no_device_no_fallback(lib):
    """Without a GPU the driver refuses to run (no CPU fallback)."""
    import md_driver_module as m
    if m.device_available():
        pytest.skip("a GPU is present")
    from helpers import gpu, static_case
    with pytest.raises(RuntimeError, match="no CUDA device"):
        gpu(static_case())
    # the memory-pool release has nothing to release and says why
    assert lib.mdelast_release_cached_memory(0) != 0
    with pytest.raises(RuntimeError):
        m.release_cached_memory(0)


def test_bspline_table_matches_oracle(lib):
    """"bspline" tables (poly_table.hpp:117-135): the host evaluator (Potential.calculate)
    gives the oracle's three spline values bit for bit."""
    D = C.POINTER(C.c_double)
    rng = np.random.RandomState(4)
    n, h = 57, 0.0021
    fs = [rng.normal(size=n) for _ in range(3)]
    rc, p = _pair(lib, h, *fs, interp=1)
    assert rc == 0
    orc = C.CDLL(ORACLE)
    orc.orc_bspline_value.argtypes = [C.c_double, C.c_int, D, C.c_double]
    orc.orc_bspline_value.restype = C.c_double
    lib.mdelast_pair_eval.argtypes = [C.c_void_p, C.c_double, D]
    for x in np.concatenate([np.linspace(0.0, (n - 1) * h, 613), [0.5 * h, 3 * h]]):
        a = np.zeros(3)
        assert lib.mdelast_pair_eval(p, x, a.ctypes.data_as(D)) == 0
        b = [orc.orc_bspline_value(h, n, f.ctypes.data_as(D), x) for f in fs]
        assert np.array_equal(a, b), x
    lib.mdelast_pair_destroy(p)
