"""Generate tests/golden/dropin_traces.npz: every call the reference's own Python callers
make on ``md_driver_module``, recorded against the reference's C++ core.

The callers run unchanged from an mdelast checkout:

* ``benchmarks/smoke/run_smoke.py``'s ``run_dynamics`` (benchmark S Part B): the 500-atom
  Cu-6 at.% Zn cell through ``MolecularDynamics`` in NPT and NVT, whose ``run()`` loop
  (``molecular_dynamics.py:1240-1285``) samples observables every step, rebuilds the
  neighbour list every 20 steps, computes g(r) and partial g(r) every 100 steps after
  thermalisation, dumps XYZ frames, and ends in ``perform_thermal_average``; and NVE at
  dt = 1 fs, which drives ``integrate()`` directly. Shortened to a few hundred steps.
* ``run_smoke.py``'s ``run_ternary`` (Part C): the fixed 500-atom Ni-Al-Co cell.
* ``examples/cu_300k/run.py`` (configuration C1): pure Cu with the single-element Cu01
  tables through ``get_EAM_file`` and ``MolecularDynamics`` built from ``N_lattice_side``,
  NPT, 100 + 50 steps (g(r) every production step, the example's default stride).

The module they import is ``oracle/ref_module.py`` (the reference core, compiled from its
own sources) wrapped by ``tests/dropin.py``'s recorder. h5py and matplotlib, which the
callers import but whose output nothing here reads, are replaced by stand-ins when absent.

    python tests/golden/make_dropin_trace.py [path/to/mdelast]
"""

import importlib.util
import logging
import os
import sys
import tempfile
import types

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
ROOT = os.path.dirname(TESTS)
sys.path[:0] = [HERE, TESTS, ROOT]

from refroot import reference_root  # noqa: E402

SESSIONS = [
    # name, what, arguments
    ("smoke_npt_cuzn500", "dynamics", ("NPT", 2.0, 100, 200)),
    ("smoke_nvt_cuzn500", "dynamics", ("NVT", 2.0, 100, 200)),
    ("smoke_nve_cuzn500_dt1", "dynamics", ("NVE", 1.0, 50, 150)),
    ("smoke_ternary_nialco500", "ternary", ()),
    ("example_cu300k_cu01_500", "cu_example", (100, 50)),
]


class _H5File:
    """Stands in for h5py.File: accepts what MolecularDynamics.save_h5 writes."""

    def __init__(self, *a, **k):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def __setitem__(self, key, value):
        pass


class _PlotSeries:
    def __init__(self, *a, **k):
        pass

    def __getattr__(self, name):
        return lambda *a, **k: None


def stub_absent_modules():
    try:
        import h5py  # noqa: F401
    except ImportError:
        h5 = types.ModuleType("h5py")
        h5.File = _H5File
        sys.modules["h5py"] = h5
    try:
        import matplotlib  # noqa: F401
    except ImportError:
        mpl = types.ModuleType("matplotlib")
        mpl.use = lambda *a, **k: None
        sys.modules["matplotlib"] = mpl
    plot = types.ModuleType("plot")
    plot.PlotSeries = _PlotSeries
    sys.modules["plot"] = plot


def load_script(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    ref = reference_root(sys.argv[1] if len(sys.argv) > 1 else None)
    import dropin
    from oracle import ref_module
    rec = dropin.Recorder(ref_module)
    sys.modules["md_driver_module"] = rec.module()
    stub_absent_modules()
    sys.path.insert(0, os.path.join(ref, "src", "python"))
    import get_potential
    import molecular_dynamics as md_mod
    smoke = load_script(os.path.join(ref, "benchmarks", "smoke", "run_smoke.py"), "run_smoke")
    example = load_script(os.path.join(ref, "examples", "cu_300k", "run.py"), "cu_300k_run")
    logging.disable(logging.CRITICAL)
    mdm = sys.modules["md_driver_module"]
    tmp = tempfile.mkdtemp()
    sessions = {}
    for name, what, a in SESSIONS:
        rec.events, rec.store = [], dropin._Store()
        out = os.path.join(tmp, name)
        with _quiet():
            if what == "dynamics":
                ens = getattr(mdm.MDDriver, a[0])
                smoke.run_dynamics(mdm, md_mod, get_potential, out, ens, a[1], a[2], a[3])
            elif what == "ternary":
                smoke.run_ternary(mdm, get_potential)
            else:
                sys.argv = ["run.py", "--build-dir", tmp, "--python-dir",
                            os.path.join(ref, "src", "python"), "--output-dir", out,
                            "--cycles-thermalization", str(a[0]),
                            "--production-cycles", str(a[1]), "--velocity-seed", "0"]
                example.main()
        sessions[name] = (rec.events, rec.store.arrays)
        print(f"{name}: {len(rec.events)} calls, {len(rec.store.arrays)} arrays", file=sys.stderr)
    path = os.path.join(HERE, "dropin_traces.npz")
    rec.save(path, sessions)
    print("wrote", path, os.path.getsize(path), "bytes", file=sys.stderr)


class _quiet:
    """Silence C-level and Python stdout (the reference prints from its constructor)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.null)
        os.close(self.saved)
        return False


if __name__ == "__main__":
    main()
