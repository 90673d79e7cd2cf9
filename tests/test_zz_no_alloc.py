"""mdelast_pair_correlation_static (g(r) with its scratch in a static device array, no
allocation) against the driver's g(r) entry point on the same coordinates: bit-identical,
as every g(r) comparison here, on two calls in a row and in all three modes; on a side
stream, and with atoms whose type is out of range, against a NumPy restatement of the
reference's counting (md_driver.cpp:732-811) over the atoms in range; requests beyond the
static scratch or the launch grid are rejected before any device work."""

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


def test_grid_limit_rejected():
    """More than 2^31 - 1 tile-pair blocks: rejected with the sizes in the message."""
    lib = _lib()
    f = lib.mdelast_pair_correlation_static
    crd = np.zeros((4, 3))
    typ = np.zeros(4, dtype=np.uint32)
    box = (C.c_double * 3)(1.0, 1.0, 1.0)
    rg = np.arange(10, dtype=float) + 0.5
    out = np.zeros(10)
    n = 65536 * 128 + 1  # 65,537 tiles: 2,147,549,953 tile pairs
    rc = f(crd.ctypes.data, typ.ctypes.data, n, 1, box, rg.ctypes.data, 10, 0,
           out.ctypes.data, None, None)
    assert rc == ERR_CAPACITY
    assert "2^31" in lib.mdelast_last_error().decode()


def numpy_gr(crd, types, n_types, h, rg, mode):
    """md_driver.cpp:732-811 in NumPy over the atoms whose type is in [0, n_types): pairs
    i < j, the reference's min image, bin floor(r / drg) for r < rmaxg, and its
    normalisations in its operation order; N = the atoms in range."""
    keep = types < n_types
    c, t = crd[keep], types[keep].astype(np.int64)
    n = len(c)
    drg = rg[1] - rg[0]
    rmaxg = rg[-1] + 0.5 * drg
    i, j = np.triu_indices(n, 1)
    d = c[i] - c[j]
    d = d - np.where(d < 0, np.trunc(d - 0.5), np.trunc(d + 0.5))
    p = d * h
    r = np.sqrt((p[:, 0] * p[:, 0] + p[:, 1] * p[:, 1]) + p[:, 2] * p[:, 2])
    ok = r < rmaxg
    b = np.floor(r[ok] / drg).astype(np.int64)
    V = h[0] * (h[1] * h[2])
    gr = np.bincount(b, minlength=len(rg)).astype(float)
    gr = gr * (V / (2.0 * np.pi * n * n * rg * rg * drg))
    ti, tj = t[i][ok], t[j][ok]
    hi, lo = np.maximum(ti, tj), np.minimum(ti, tj)
    slot = hi * (hi + 1) // 2 + lo
    npair = n_types * (n_types + 1) // 2
    gp = np.zeros((npair, len(rg)))
    cnt = np.bincount(slot * len(rg) + b, minlength=npair * len(rg)).reshape(npair, -1)
    Nt = np.bincount(t, minlength=n_types).astype(float)
    s = 0
    for bb in range(n_types):
        for a in range(bb + 1):
            Na, Nb = Nt[a], Nt[bb]
            pc = (Na * (Na - 1.0) / 2.0 if Na > 1 else 0.0) if a == bb else Na * Nb
            if pc > 0.0:
                pref = V / (4.0 * np.pi * pc * drg)
                gp[s] = cnt[s] * (pref / (rg * rg))
            s += 1
    return gr, gp


@pytest.mark.gpu
def test_side_stream_and_types_out_of_range():
    """A torch side stream passed as the stream handle, and 10 % of the atoms given a type
    outside [0, n_types): those atoms take no part, the rest match the NumPy restatement."""
    import torch
    lib = _lib()
    f = lib.mdelast_pair_correlation_static
    case = dynamics_case(nside=5, n_zn=30, ensemble=1)
    d = gpu(case)
    for _ in range(4):
        d.integrate()
    crd_h = gpu_atoms(d, "coordinates")
    nt = len(case.tables.masses)
    types = np.asarray(case.types, dtype=np.uint32).copy()
    rs = np.random.RandomState(5)
    types[rs.choice(len(types), size=len(types) // 10, replace=False)] = nt + 3
    h = np.diag(np.asarray(d.box.h)).copy()
    rg_h = np.asarray(d.rg, dtype=float)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        crd = torch.tensor(crd_h, dtype=torch.float64, device="cuda")
        typ = torch.tensor(types.astype(np.int32), device="cuda")
        rg = torch.tensor(rg_h, dtype=torch.float64, device="cuda")
        npair = nt * (nt + 1) // 2
        box = (C.c_double * 3)(*h)
        for call in range(2):
            g = torch.full((len(rg_h),), -1.0, dtype=torch.float64, device="cuda")
            gp = torch.full((npair, len(rg_h)), -1.0, dtype=torch.float64, device="cuda")
            rc = f(crd.data_ptr(), typ.data_ptr(), len(types), nt, box, rg.data_ptr(),
                   len(rg_h), 1, g.data_ptr(), gp.data_ptr(), C.c_void_p(side.cuda_stream))
            assert rc == 0, lib.mdelast_last_error().decode()
            side.synchronize()
            g_np, gp_np = numpy_gr(crd_h, types, nt, h, rg_h, 1)
            assert np.abs(g.cpu().numpy() - g_np).max() <= 1e-12 * np.abs(g_np).max()
            assert np.abs(gp.cpu().numpy() - gp_np).max() <= 1e-12 * np.abs(gp_np).max()
            assert g_np.sum() > 0 and gp_np.sum() > 0


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
