"""mdelast_pair_correlation_static (g(r) with its scratch in a static device array, no
allocation) against the driver's g(r) entry point on the same coordinates: bit-identical,
as every g(r) comparison here, on two calls in a row and in all three modes; requests
beyond the static scratch are rejected before any device work."""

import ctypes as C
import os

import numpy as np
import pytest

from helpers import dynamics_case, gpu, gpu_atoms

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mdelast_b200", "lib", "libmdelast_cuda.so")
ERR_CAPACITY = -6
MAX_SLOTS = 65536  # MDELAST_GR_STATIC_MAX_SLOTS


def _lib():
    if not os.path.exists(LIB):
        pytest.skip("libmdelast_cuda.so not built")
    lib = C.CDLL(LIB)
    f = lib.mdelast_pair_correlation_static
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                  C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    lib.mdelast_last_error.restype = C.c_char_p
    return lib


def test_static_scratch_limits_rejected():
    lib = _lib()
    f = lib.mdelast_pair_correlation_static
    crd = np.zeros((4, 3))
    typ = np.zeros(4, dtype=np.uint32)
    box = (C.c_double * 3)(1.0, 1.0, 1.0)
    n_rg = MAX_SLOTS // 4 + 1  # two types: 4 histograms
    rg = np.arange(n_rg, dtype=float) + 0.5
    out = np.zeros(4 * n_rg)
    rc = f(crd.ctypes.data, typ.ctypes.data, 4, 2, box, rg.ctypes.data, n_rg, 1,
           out.ctypes.data, out.ctypes.data, None)
    assert rc == ERR_CAPACITY
    msg = lib.mdelast_last_error().decode()
    assert "MDELAST_GR_STATIC_MAX_SLOTS" in msg and str(MAX_SLOTS) in msg
    rc = f(crd.ctypes.data, typ.ctypes.data, 4, 9, box, rg.ctypes.data, 10, 0,
           out.ctypes.data, None, None)
    assert rc == ERR_CAPACITY


@pytest.mark.gpu
@pytest.mark.parametrize("nside,ensemble,steps", [(5, 1, 0), (8, 2, 6)])
def test_static_gr_equals_driver_gr(nside, ensemble, steps):
    import torch
    lib = _lib()
    f = lib.mdelast_pair_correlation_static
    case = dynamics_case(nside=nside, n_zn=nside ** 3 // 4, ensemble=ensemble)
    d = gpu(case)
    for _ in range(steps):
        d.integrate()
    crd = torch.tensor(gpu_atoms(d, "coordinates"), dtype=torch.float64, device="cuda")
    typ = torch.tensor(np.asarray(case.types, dtype=np.uint32).astype(np.int32),
                       device="cuda")
    rg = torch.tensor(np.asarray(d.rg), dtype=torch.float64, device="cuda")
    h = np.asarray(d.box.h)
    box = (C.c_double * 3)(h[0, 0], h[1, 1], h[2, 2])
    n, n_rg, nt = crd.shape[0], rg.shape[0], len(case.tables.masses)
    npair = nt * (nt + 1) // 2
    methods = ["calculate_pair_correlation", "calculate_pair_correlations",
               "calculate_partial_pair_correlation"]
    for mode in (1, 0, 2):
        getattr(d, methods[mode])()
        g_ref, gp_ref = np.array(d.gr), np.array(d.gr_partial)
        for call in range(2):
            g = torch.full((n_rg,), -1.0, dtype=torch.float64, device="cuda")
            gp = torch.full((npair, n_rg), -1.0, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            rc = f(crd.data_ptr(), typ.data_ptr(), n, nt, box, rg.data_ptr(), n_rg, mode,
                   g.data_ptr(), gp.data_ptr(), None)
            assert rc == 0, lib.mdelast_last_error().decode()
            torch.cuda.synchronize()
            g, gp = g.cpu().numpy(), gp.cpu().numpy()
            if mode != 2:
                assert g.sum() > 0 and np.array_equal(g, g_ref), (mode, call)
            else:
                assert np.all(g == -1.0)  # mode 2 leaves gr untouched
            if mode != 0:
                assert gp.sum() > 0 and np.array_equal(gp, gp_ref), (mode, call)
            else:
                assert np.all(gp == -1.0)
