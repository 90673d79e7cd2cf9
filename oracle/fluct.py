"""Test infrastructure (the oracle), not the product: a numpy restatement of the reference's
elastic-constant estimator on per-sample arrays, as MolecularDynamics.perform_thermal_average
computes it (src/python/molecular_dynamics.py:663-1000). Only the tests use it, as the
checker of the device sums and of mdelast_elastic_constants.

Pinned against tests/golden/fluct_estimator.npz, the reference's own perform_thermal_average
run on seeded sample series (tests/golden/make_fluct_golden.py).
"""

from __future__ import annotations

import numpy as np

K_BOLTZ = 1.38064852e-16  # units.hpp:6


def _mean_std(x):
    """averages.py:12-17: mean and population standard deviation (np.average)."""
    m = np.average(x)
    return m, np.sqrt(np.average((x - m) ** 2))


def elastic_constants(born_stress, born_el, V_V0, etot_atom, ensemble, N, V0, T, P, n_therm):
    """Per-sample arrays over the whole run (born_stress (6, n), born_el (6, 6, n) with zeros
    below the diagonal, V_V0 (n), etot_atom (n)); the production window starts at sample
    n_therm. Returns C (6 x 6), C11, C12, C44, bulk_modulus, compressibility,
    volume_thermal_expansion (the last two only for NPT, else 0)."""
    prod = slice(n_therm, None)
    kT = K_BOLTZ * T                                           # :773 kTth
    V_V0 = np.asarray(V_V0, dtype=float)
    vv_mean, vv_std = _mean_std(V_V0[prod])
    Vmean = vv_mean * V0                                       # :715-716
    rho = N / (V_V0 * V0)                                      # :717-722
    rho_mean = np.average(rho[prod])
    K = comp = vte = 0.0
    if ensemble == 2:                                          # :776-823
        comp = (vv_std * V0) ** 2 / (Vmean * kT)
        K = 1.0 / comp
        dV = V_V0 * V0 - Vmean
        e = np.asarray(etot_atom, dtype=float)
        dE = (e - np.average(e[prod])) * N
        vte = np.average((dV * (dE + P * dV) / (Vmean * K_BOLTZ * T ** 2))[prod])
    fluc = np.array(born_stress, dtype=float, copy=True)      # :826-841
    if ensemble == 2:
        fluc[:3, :] -= (rho * kT)[None, :]
    m = fluc[:, prod].mean(axis=1)
    V_all_mean = np.average((V_V0 * V0)[prod])                 # :893-898
    C = np.zeros((6, 6))
    for i in range(6):
        for j in range(6):
            sf = V_all_mean / kT * (fluc[i] * fluc[j] - m[i] * m[j])
            ck = rho * kT * ((2.0 if i < 3 else 1.0) if i == j else 0.0)
            bulk = K if (i < 3 and j < 3 and ensemble == 2) else 0.0
            C[i, j] = (np.average(np.asarray(born_el[i][j])[prod]) - np.average(sf[prod])
                       + np.average(ck[prod]) + bulk)          # :926-958
    C11 = (C[0, 0] + C[1, 1] + C[2, 2]) / 3.0                  # :984-999
    C12 = (C[0, 1] + C[0, 2] + C[1, 2]) / 3.0
    C44 = (C[3, 3] + C[4, 4] + C[5, 5]) / 3.0
    return dict(C=C, C11=C11, C12=C12, C44=C44, bulk_modulus=K, compressibility=comp,
                volume_thermal_expansion=vte)


def welford(x):
    """Running means and population co-moment sums of the rows of x (d, n), in the order
    the device folds samples in: returns (mean (d,), upper-triangle co-moments row by row)."""
    x = np.asarray(x, dtype=float)
    d, n = x.shape
    mean = np.zeros(d)
    M = np.zeros((d, d))
    for k in range(n):
        d0 = x[:, k] - mean
        mean = mean + d0 / (k + 1)
        d1 = x[:, k] - mean
        M += np.outer(d0, d1)
    iu = np.triu_indices(d)
    return mean, M[iu]
