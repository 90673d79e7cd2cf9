"""Record and replay the calls a script makes on ``md_driver_module``.

The reference's own callers (``molecular_dynamics.py``'s ``MolecularDynamics.run()``,
``benchmarks/smoke/run_smoke.py``, ``examples/cu_300k/run.py``) are run once, where the
reference's Python is available, against a module over the reference core
(``oracle/ref_module.py``) wrapped by :class:`Recorder`. The recorder logs, in order, every
object the script constructs on the module with its arguments, every attribute it reads on
those objects (with the value the reference returned), every attribute it sets and every
method it calls (with the result). :func:`replay` then drives another module through exactly
the same calls, with the same arguments, and hands each read and each result to a checker
beside the value the reference gave. So a replay on this package's ``md_driver_module`` is
the reference's run loop driving the GPU path, call for call.

Node arrays of ``TablePotential`` and ``EAM`` are recorded as sha256 digests (their files'
licences keep the tables out of the repository); the replay rebuilds them with this
package's reader, whose arrays are pinned bit for bit to the reference loader's
(``tests/test_readers.py``), and looks them up by digest.
"""

from __future__ import annotations

import enum
import io
import json
import types

import numpy as np

HANDLES = ("TablePotential", "EAM", "PotentialVector", "EAMVector", "Box", "Thermostat",
           "Barostat", "BarostatFlex", "MDDriver", "LennardJones", "Morse")
TABLE_CLASSES = ("TablePotential", "EAM")
PASS_THROUGH = ("Units", "Vector3d", "PotentialValue", "Potential")


def digest(a) -> str:
    import hashlib
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return hashlib.sha256(a.astype("<f8").tobytes()).hexdigest()


def _is_v3(x):
    return hasattr(x, "x") and hasattr(x, "y") and hasattr(x, "z") and not isinstance(x, np.ndarray)


def _kind(x):
    """The handle class name of an object of either module, or None."""
    n = type(x).__name__
    return n if n in ("Box", "Thermostat", "Barostat") else None


class _Store:
    def __init__(self, arrays=None):
        self.arrays = {} if arrays is None else arrays

    def put(self, a):
        k = f"a{len(self.arrays)}"
        self.arrays[k] = np.asarray(a)
        return k


def canon(v, store: _Store):
    """A JSON-able canonical form of a value read from either module; arrays go to
    ``store`` (small ones stay inline)."""
    if isinstance(v, enum.Enum) or type(v).__name__ in ("Ensamble", "ThermostatCoupling"):
        return {"enum": int(v)}
    if isinstance(v, (bool, np.bool_)):
        return bool(v)
    if isinstance(v, (int, np.integer)):
        return int(v)
    if isinstance(v, (float, np.floating)):
        return float(v)
    if v is None or isinstance(v, str):
        return v
    k = _kind(v)
    if k == "Box":
        return {"Box": {"h": canon(np.asarray(v.h, dtype=float), store)}}
    if k == "Thermostat":
        return {"Thermostat": {f: canon(np.asarray(getattr(v, f), dtype=float), store)
                               if f in ("q", "p_eta", "eta") else canon(getattr(v, f), store)
                               for f in ("temperature", "q", "p_eta", "eta", "nchain", "Nf")}}
    if k == "Barostat":
        return {"Barostat": {"pressure": float(v.pressure), "w": float(v.w),
                             "epsilon": float(v.epsilon), "p_epsilon": float(v.p_epsilon),
                             "thermostat": canon(v.thermostat, store)}}
    if _is_v3(v):
        return {"v3": [float(v.x), float(v.y), float(v.z)]}
    if isinstance(v, (list, tuple)) and v and all(_is_v3(x) for x in v):
        return {"V3": store.put(np.array([[x.x, x.y, x.z] for x in v], dtype=float))}
    a = np.asarray(v)
    if a.dtype.kind in "fiub" and a.size <= 8:
        return {"inline": a.astype(float).tolist(), "shape": list(a.shape)}
    if a.dtype.kind in "fiub":
        return {"arr": store.put(a.astype(float))}
    raise TypeError(f"cannot record a value of type {type(v).__name__}")


def uncanon(c, arrays):
    """The numpy/float form of a canonical value (for comparisons)."""
    if isinstance(c, dict):
        if "enum" in c:
            return int(c["enum"])
        if "inline" in c:
            return np.array(c["inline"], dtype=float).reshape(c["shape"])
        if "arr" in c:
            return arrays[c["arr"]]
        if "V3" in c:
            return arrays[c["V3"]]
        if "v3" in c:
            return np.array(c["v3"])
        (k, body), = c.items()
        return {kk: uncanon(vv, arrays) for kk, vv in body.items()}
    return c


class _Proxy:
    __slots__ = ("_rec", "_hid", "_obj")

    def __init__(self, rec, hid, obj):
        object.__setattr__(self, "_rec", rec)
        object.__setattr__(self, "_hid", hid)
        object.__setattr__(self, "_obj", obj)

    def __getattr__(self, name):
        rec, hid, obj = self._rec, self._hid, self._obj
        v = getattr(obj, name)
        if callable(v) and not isinstance(v, type) and _kind(v) is None \
                and not isinstance(v, (list, tuple, np.ndarray)):
            def call(*args):
                r = v(*[rec.unwrap(a) for a in args])
                ev = ["call", hid, name, [rec.enc(a, False) for a in args],
                      canon(r, rec.store)]
                rec.events.append(ev)
                return rec.wrap_result(r, ev)
            return call
        ev = ["get", hid, name, canon(v, rec.store)]
        rec.events.append(ev)
        return rec.wrap_result(v, ev)

    def __setattr__(self, name, value):
        rec = self._rec
        setattr(self._obj, name, rec.unwrap(value))
        rec.events.append(["set", self._hid, name, rec.enc(value, False)])

    def __iter__(self):
        return iter(self._obj)

    def __len__(self):
        return len(self._obj)


class Recorder:
    """Wraps a ``md_driver_module`` (``real``); :meth:`module` is the module to hand the
    script. ``events`` and ``store.arrays`` form the trace."""

    def __init__(self, real):
        self.real = real
        self.events = []
        self.store = _Store()
        self._n = 0

    def _hid(self):
        self._n += 1
        return self._n

    def unwrap(self, v):
        if isinstance(v, _Proxy):
            return v._obj
        if isinstance(v, list):
            return [self.unwrap(x) for x in v]
        if isinstance(v, tuple):
            return tuple(self.unwrap(x) for x in v)
        return v

    def enc(self, v, tables):
        """Encode a call argument."""
        if isinstance(v, _Proxy):
            return {"h": v._hid}
        if isinstance(v, enum.Enum) or type(v).__name__ in ("Ensamble", "ThermostatCoupling"):
            return {"enum": int(v)}
        if isinstance(v, (bool, np.bool_)):
            return bool(v)
        if isinstance(v, (int, np.integer)):
            return int(v)
        if isinstance(v, (float, np.floating)):
            return float(v)
        if v is None or isinstance(v, str):
            return v
        if _is_v3(v):
            return {"v3": [float(v.x), float(v.y), float(v.z)]}
        if isinstance(v, (list, tuple)) and v and all(_is_v3(x) for x in v):
            return {"V3": self.store.put(np.array([[x.x, x.y, x.z] for x in v], dtype=float))}
        if isinstance(v, (list, tuple)) and any(isinstance(x, _Proxy) for x in v):
            return {"list": [self.enc(x, tables) for x in v]}
        a = np.asarray(v)
        if tables and a.ndim == 1 and a.size > 8:
            return {"digest": digest(a), "n": int(a.size)}
        if isinstance(v, (list, tuple)):
            if a.dtype.kind in "iub":
                return {"ints": self.store.put(a.astype(np.int64))}
            return {"floats": self.store.put(a.astype(float))}
        return {"ndarray": self.store.put(a)}

    def wrap_result(self, v, ev):
        if _kind(v) is not None:
            hid = self._hid()
            ev.append(hid)
            return _Proxy(self, hid, v)
        return v

    def module(self):
        rec = self
        m = types.ModuleType("md_driver_module")
        for n in PASS_THROUGH:
            if hasattr(self.real, n):
                setattr(m, n, getattr(self.real, n))
        for n in HANDLES:
            if not hasattr(self.real, n):
                continue
            real_cls = getattr(self.real, n)

            def make(*args, _n=n, _c=real_cls):
                obj = _c(*[rec.unwrap(a) for a in args])
                hid = rec._hid()
                rec.events.append(["new", hid, _n, [rec.enc(a, _n in TABLE_CLASSES)
                                                    for a in args]])
                return _Proxy(rec, hid, obj)

            ns = {"__new__": staticmethod(lambda cls, *a, _m=make: _m(*a))}
            for attr in dir(real_cls):
                if attr.isupper() or attr in ("Ensamble", "ThermostatCoupling"):
                    ns[attr] = getattr(real_cls, attr)
            setattr(m, n, type(n, (), ns))
        return m

    def save(self, path, sessions):
        """``sessions``: {name: (events, arrays)} written to one npz file."""
        out = {}
        meta = {}
        for name, (events, arrays) in sessions.items():
            meta[name] = events
            for k, a in arrays.items():
                out[f"{name}/{k}"] = a
        out["events_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
        np.savez_compressed(path, **out)


def load(path):
    """{name: (events, arrays)} from a trace file."""
    z = np.load(path)
    meta = json.loads(bytes(z["events_json"]).decode())
    out = {}
    for name, events in meta.items():
        arrays = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}
        out[name] = (events, arrays)
    return out


def table_arrays(tables_list, interpolations=("quintic", "bspline")):
    """digest -> node array for every table array of the given SetflTables."""
    out = {}
    for t in tables_list:
        for arr in (t.phi, t.dphi, t.d2phi, t.rho, t.drho_dr, t.d2rho_dr2, t.F, t.dF, t.d2F):
            for row in arr:
                out[digest(row)] = np.asarray(row, dtype=float)
    return out


def replay(events, arrays, m, tables, check, on_new=None):
    """Drive module ``m`` through the recorded ``events``. ``tables``: digest -> array
    (:func:`table_arrays`). ``check(index, event, got)`` is called for every read and every
    call result, with ``got`` the canonical value (numpy form) ``m`` returned;
    ``on_new(hid, cls, obj)`` for every object constructed."""
    objs = {}
    store = _Store()

    def dec(c):
        if isinstance(c, dict):
            if "h" in c:
                return objs[c["h"]]
            if "enum" in c:
                return c["enum"]
            if "v3" in c:
                return m.Vector3d(*c["v3"])
            if "V3" in c:
                return [m.Vector3d(*r) for r in arrays[c["V3"]]]
            if "list" in c:
                return [dec(x) for x in c["list"]]
            if "digest" in c:
                return tables[c["digest"]]
            if "ints" in c:
                return [int(x) for x in arrays[c["ints"]]]
            if "floats" in c:
                return [float(x) for x in arrays[c["floats"]]]
            if "ndarray" in c:
                return arrays[c["ndarray"]]
        return c

    def fix_enums(cls, args):
        # the MDDriver constructor takes Ensamble and ThermostatCoupling at positions 4, 5
        if cls == "MDDriver":
            args[4] = m.MDDriver.Ensamble(args[4])
            args[5] = m.MDDriver.ThermostatCoupling(args[5])
        return args

    for i, ev in enumerate(events):
        kind = ev[0]
        if kind == "new":
            _, hid, cls, args = ev
            obj = getattr(m, cls)(*fix_enums(cls, [dec(a) for a in args]))
            objs[hid] = obj
            if on_new is not None:
                on_new(hid, cls, obj)
        elif kind == "get":
            obj = objs[ev[1]]
            v = getattr(obj, ev[2])
            check(i, ev, uncanon(canon(v, store), store.arrays))
            if len(ev) > 4:
                objs[ev[4]] = v
        elif kind == "set":
            setattr(objs[ev[1]], ev[2], dec(ev[3]))
        elif kind == "call":
            obj = objs[ev[1]]
            r = getattr(obj, ev[2])(*[dec(a) for a in ev[3]])
            check(i, ev, uncanon(canon(r, store), store.arrays))
            if len(ev) > 5:
                objs[ev[5]] = r
    return objs
