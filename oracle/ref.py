"""ctypes access to the two CPU implementations of the path that ``oracle/Makefile``
builds. TEST INFRASTRUCTURE ONLY: used by tests as checkers and by
``bench.py --impl reference`` as the timed CPU baseline.

* ``RefDriver``: the reference's own C++ core (``oracle/_ref/libmdelast_ref.so``);
* ``OracleDriver``: the C restatement (``oracle/_build/libmdelast_oracle.so``).

Both take the same inputs as ``md_driver_module.MDDriver``
(``md_driver_module.cpp:95-102``) in array form and expose the same readouts.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libmdelast_ref.so")
ORACLE_PATH = os.path.join(HERE, "_build", "libmdelast_oracle.so")

_libs = {}

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int)
U = C.POINTER(C.c_uint)

N_SCALARS = 78
SCALAR_NAMES = (
    ["epot_eam_atom", "epot_atom", "ekin_atom", "etot_atom", "ekin_tot", "etot_cons_initial",
     "etot_cons", "etot_cons_err", "virial", "total_laplacian", "total_force2",
     "temperature_kin", "temperature_conf_inverse", "pressure", "time", "cycle"])
ATOM_FIELDS = {"positions": 0, "coordinates": 1, "velocities": 2, "forces": 3,
               "rho_eam": 4, "energies_pot": 5, "energies_kin": 6, "F_eam": 7,
               "dFdrho_eam": 8, "d2Fdrho2_eam": 9}


def available(which="ref") -> bool:
    return os.path.isfile(LIB_PATH if which == "ref" else ORACLE_PATH)


class _Api:
    """The functions of one library under their un-prefixed names."""

    def __init__(self, L, prefix):
        self._L, self._p = L, prefix

    def __getattr__(self, name):
        return getattr(self._L, self._p + name)


def lib(which="ref"):
    if which not in _libs:
        path, prefix = (LIB_PATH, "mref_") if which == "ref" else (ORACLE_PATH, "orc_")
        if not os.path.isfile(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle {'ref' if which == 'ref' else ''})")
        L = _Api(C.CDLL(path), prefix)
        L.create.restype = C.c_void_p
        L.create.argtypes = (
            [C.c_int, C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_int, D, D, D,
             C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, D, D, D, D, D, D,
             C.c_int, D, D, U, D, C.c_int, C.c_int,
             C.c_double, C.c_int, D, D, C.c_double,
             C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, D, D, C.c_double,
             D, C.c_int, D, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double])
        for name in ("destroy", "calculate_neighbors", "calculate_forces"):
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = None
        L.integrate.argtypes = [C.c_void_p, C.c_int]
        L.set_sample_observables.argtypes = [C.c_void_p, C.c_int]
        L.scalars.argtypes = [C.c_void_p, D]
        L.atoms.argtypes = [C.c_void_p, C.c_int, D]
        L.chain.argtypes = [C.c_void_p, C.c_int, D, D]
        L.chain.restype = C.c_int
        L.neighbors.argtypes = [C.c_void_p, I, I, C.c_long]
        L.neighbors.restype = C.c_long
        L.pair_correlation.argtypes = [C.c_void_p, C.c_int]
        L.gr.argtypes = [C.c_void_p, D, D]
        if which == "ref":
            L.eval.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, D]
        else:
            L.status.argtypes = [C.c_void_p]
            L.status.restype = C.c_uint
        _libs[which] = L
    return _libs[which]


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(D)


class RefDriver:
    """One reference MDDriver. ``tables`` is a ``mdelast_b200.potentials.SetflTables``
    (or any object with the same fields)."""

    which = "ref"

    def __init__(self, tables, positions, velocities, types, ensemble=0, coupling=0,
                 thermo=(300.0, [1e-30], [0.0], None), baro=(0.0, 1e-30, 0.0),
                 baro_thermo=(300.0, [1e-30], [0.0], 1.0), box=None, rg=None, Nf=None,
                 dt=1e-15, neighbors=False, r_skin=1.0, fatal_conservation=1e3,
                 interpolation="quintic", has_eam=True):
        L = lib(self.which)
        t = tables
        self.N = N = len(positions)
        self.ntypes = t.n_types
        keep = []

        def d(a):
            arr, p = _d(a)
            keep.append(arr)
            return p

        types = np.ascontiguousarray(types, dtype=np.uint32)
        keep.append(types)
        if box is None:
            raise ValueError("box (3x3, cm) required")
        if rg is None:
            rg = [(k + 0.5) * 0.01e-8 for k in range(10)]
        if Nf is None:
            Nf = 3.0 * N
        T, q, p_eta, nf_th = thermo
        if nf_th is None:
            nf_th = Nf
        P, w, p_eps = baro
        Tb, qb, p_eta_b, nf_b = baro_thermo
        self.h = L.create(
            t.n_types, interpolation.encode(), t.rcut, t.rmin_fatal, t.dr, t.n_r,
            d(t.phi), d(t.dphi), d(t.d2phi), int(has_eam), getattr(t, "eam_rcut", t.rcut),
            t.rhomax, t.drho, t.n_rho,
            d(t.rho), d(t.drho_dr), d(t.d2rho_dr2), d(t.F), d(t.dF), d(t.d2F),
            N, d(positions), d(velocities), types.ctypes.data_as(U), d(t.masses),
            int(ensemble), int(coupling),
            float(T), len(q), d(q), d(p_eta), float(nf_th),
            float(P), float(w), float(p_eps), float(Tb), len(qb), d(qb), d(p_eta_b), float(nf_b),
            d(np.asarray(box, dtype=float).reshape(9)), len(rg), d(rg), float(Nf), float(dt),
            int(bool(neighbors)), float(r_skin), float(fatal_conservation))
        if not self.h:
            raise ValueError("driver construction failed")
        self.n_rg = len(rg)
        self.nchain = (len(q), len(qb))

    def _L(self):
        return lib(self.which)

    def __del__(self):
        if getattr(self, "h", None):
            self._L().destroy(self.h)
            self.h = None

    def integrate(self, n=1):
        self._L().integrate(self.h, int(n))

    def calculate_neighbors(self):
        self._L().calculate_neighbors(self.h)

    def calculate_forces(self):
        self._L().calculate_forces(self.h)

    def set_sample_observables(self, flag):
        self._L().set_sample_observables(self.h, int(bool(flag)))

    def scalars(self) -> np.ndarray:
        out = np.zeros(N_SCALARS)
        self._L().scalars(self.h, out.ctypes.data_as(D))
        return out

    def scalar_dict(self) -> dict:
        s = self.scalars()
        out = {k: s[i] for i, k in enumerate(SCALAR_NAMES)}
        out["born_stress_tensor"] = s[16:22].copy()
        out["stress_tensor"] = s[22:28].copy()
        out["born_elasticity_tensor"] = s[28:64].reshape(6, 6).copy()
        out["box"] = s[64:73].reshape(3, 3).copy()
        out["baro_epsilon"], out["baro_p_epsilon"] = s[73], s[74]
        out["momentum_tot"] = s[75:78].copy()
        return out

    def atoms(self, field: str) -> np.ndarray:
        k = ATOM_FIELDS[field]
        out = np.zeros((self.N, 3) if k < 4 else self.N)
        self._L().atoms(self.h, k, out.ctypes.data_as(D))
        return out

    def chain(self, which=0):
        n = self.nchain[which]
        p, e = np.zeros(n), np.zeros(n)
        self._L().chain(self.h, which, p.ctypes.data_as(D), e.ctypes.data_as(D))
        return p, e

    def neighbors(self):
        point = np.zeros(self.N + 1, dtype=np.int32)
        cap = 1 << 26
        nb = np.zeros(cap, dtype=np.int32)
        total = self._L().neighbors(self.h, point.ctypes.data_as(I), nb.ctypes.data_as(I), cap)
        if total < 0:
            return None
        return point, nb[:total].copy()

    def pair_correlation(self, mode=0):
        self._L().pair_correlation(self.h, int(mode))
        gr = np.zeros(self.n_rg)
        npart = self.ntypes * (self.ntypes + 1) // 2
        grp = np.zeros((npart, self.n_rg))
        self._L().gr(self.h, gr.ctypes.data_as(D), grp.ctypes.data_as(D))
        return gr, grp

    def eval(self, what, k, x):
        o = np.zeros(3)
        self._L().eval(self.h, int(what), int(k), float(x), o.ctypes.data_as(D))
        return o


class OracleDriver(RefDriver):
    """The C restatement (``oracle/mdelast_oracle.c``) behind the same interface."""

    which = "oracle"

    def status(self) -> int:
        return int(self._L().status(self.h))
