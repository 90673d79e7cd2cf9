"""Generate tests/golden/fluct_estimator.npz: the reference's own thermal averaging
(molecular_dynamics.py:663-1173, MolecularDynamics.perform_thermal_average) run on seeded
synthetic sample series for NVT and NPT, with its inputs and the results the C_ij
estimator must reproduce (elasticity tensor, C11/C12/C44, bulk modulus, compressibility,
volumetric thermal expansion).

Run from the repository root, in a checkout where the reference sources and the built
md_driver_module are present (the reference's Python imports md_driver_module for its
enums and Units, and h5py, which is stubbed here because nothing is written):

    python tests/golden/make_fluct_golden.py /path/to/mdelast
"""

import logging
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def synthetic_series(rng, n, ensemble, N, V0):
    """Sample arrays with the magnitudes of the 13,500-atom Cu-Zn cell at 300 K (cgs)."""
    V_V0 = 1.0 + (0.002 * rng.standard_normal(n) if ensemble == 2 else np.zeros(n))
    V = V_V0 * V0
    mix = rng.standard_normal((6, 6)) * 0.3 + np.eye(6)
    sb = (np.array([1.0e9, 1.1e9, 0.9e9, 1e7, -2e7, 3e7])[:, None]
          + 5e8 * mix @ rng.standard_normal((6, n)))
    cb = np.zeros((6, 6, n))
    base = np.array([[2.0e12, 1.2e12, 1.2e12, 0, 0, 0], [0, 2.0e12, 1.2e12, 0, 0, 0],
                     [0, 0, 2.0e12, 0, 0, 0], [0, 0, 0, 0.9e12, 0, 0],
                     [0, 0, 0, 0, 0.9e12, 0], [0, 0, 0, 0, 0, 0.9e12]])
    for i in range(6):
        for j in range(i, 6):
            cb[i, j] = base[i, j] + 1e10 * rng.standard_normal(n)
    eV = 1.6021773e-12
    etot = -3.5 * eV + 0.01 * eV * rng.standard_normal(n) + 0.2 * eV * (V_V0 - 1.0)
    return dict(V_V0=V_V0, V=V, born_stress=sb, born_el=cb, etot_atom=etot,
                epot_atom=etot - 0.04 * eV, ekin_atom=np.full(n, 0.04 * eV),
                epot_eam_atom=etot * 0.5,
                temperature_kin=300.0 + 5.0 * rng.standard_normal(n),
                temperature_conf_inverse=1.0 / (300.0 + 5.0 * rng.standard_normal(n)),
                total_laplacian=1e5 + rng.standard_normal(n),
                total_force2=1e-3 + 1e-6 * rng.standard_normal(n),
                pressure=1e8 + 1e7 * rng.standard_normal(n),
                stress=1e8 + 1e7 * rng.standard_normal((6, n)),
                etot_cons=etot * N, etot_cons_err=np.abs(1e-7 * rng.standard_normal(n)))


def run_reference(ref_py, ensemble, s, N, V0, T, P, n_therm):
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    sys.path[:0] = [ref_py, os.path.join(ROOT, "mdelast_b200", "lib")]
    import md_driver_module as m
    import molecular_dynamics as md
    from series import Series
    logging.disable(logging.CRITICAL)

    class _Vol:
        def __init__(self, v):
            self.v = v

        def volume(self):
            return self.v

    drv = types.SimpleNamespace(
        ensamble=m.MDDriver.Ensamble(ensemble), time=1.0, cycle=len(s["V_V0"]),
        thermostat=types.SimpleNamespace(temperature=T),
        barostat=types.SimpleNamespace(pressure=P), box_initial=_Vol(V0))
    o = object.__new__(md.MolecularDynamics)
    o.driver = drv
    o.ensamble = drv.ensamble
    o.Nparticles = N
    o.volume = V0
    o.ndensity = N / V0
    o.temperature_thermostat = T
    o.pressure_barostat = P
    o.cycles_thermalization = n_therm
    o.sample_stride = 1
    o.samples_thermalization = n_therm
    o.thermalized = True
    o.gr_samples = 0
    o.gr_sum = np.zeros(4)
    o.gr_partial_sum = None
    o.rg = np.arange(4) + 0.5
    o.material = types.SimpleNamespace(eam=object(), atomic_weight=[1.0, 2.0])
    ser = Series()
    n = len(s["V_V0"])
    ser.time = list(range(n))
    for k, v in [("temperature_kin", "temperature_kin"),
                 ("temperature_conf_inverse", "temperature_conf_inverse"),
                 ("total_laplacian", "total_laplacian"), ("total_force2", "total_force2"),
                 ("pressure", "pressure"), ("etot_atom", "etot_atom"),
                 ("epot_atom", "epot_atom"), ("epot_eam_atom", "epot_eam_atom"),
                 ("ekin_atom", "ekin_atom"), ("etot_cons", "etot_cons"),
                 ("etot_cons_err", "etot_cons_err"), ("V_V0", "V_V0")]:
        getattr(ser, k).data = list(s[v])
    ser.L_L0.data = list(s["V_V0"] ** (1.0 / 3.0))
    for i in range(6):
        ser.stress_tensor.data[i].data = list(s["stress"][i])
        ser.born_stress_tensor.data[i].data = list(s["born_stress"][i])
        for j in range(6):
            ser.born_elasticity_tensor.data[i][j].data = list(s["born_el"][i, j])
    o.series = ser
    o.perform_thermal_average()
    tr = ser.thermal_results
    out = dict(C=np.array(tr.elasticity_tensor), C11=tr.elasticity_tensor_11,
               C12=tr.elasticity_tensor_12, C44=tr.elasticity_tensor_44,
               bulk_modulus=tr.bulk_modulus)
    if ensemble == 2:
        out.update(compressibility=tr.compressibility,
                   volume_thermal_expansion=tr.volume_thermal_expansion)
    return out


def main():
    sys.path.insert(0, HERE)
    from refroot import reference_root
    ref = reference_root(sys.argv[1] if len(sys.argv) > 1 else None)
    ref_py = os.path.join(ref, "src", "python")
    N, T, P = 13500, 300.0, 1e-10 * 1e10
    V0 = N / 4 * (3.6345e-8) ** 3
    n, n_therm = 300, 50
    arrays = {}
    for ens, name in [(1, "nvt"), (2, "npt")]:
        rng = np.random.RandomState(2026 + ens)
        s = synthetic_series(rng, n, ens, N, V0)
        res = run_reference(ref_py, ens, s, N, V0, T, P, n_therm)
        for k, v in s.items():
            arrays[f"{name}_in_{k}"] = np.asarray(v)
        for k, v in res.items():
            arrays[f"{name}_out_{k}"] = np.asarray(v)
    arrays.update(N=N, T=T, P=P, V0=V0, n_therm=n_therm)
    path = os.path.join(HERE, "fluct_estimator.npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, {k: np.asarray(v).shape for k, v in arrays.items() if "out" in k})


if __name__ == "__main__":
    main()
