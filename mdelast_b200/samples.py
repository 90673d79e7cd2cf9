"""Sample series from the device ring, in the reference's own containers.

The reference's run loop reads a dozen driver attributes after every sampled step and
appends them to its Series (molecular_dynamics.py:1218-1238, append_sample). With the
device ring, a run can go many steps without Python and then hand the whole stretch over
at once: ``drain_into_series`` appends every drained record exactly as append_sample would
have, so perform_thermal_average and the plotting code see the same series.
"""

from __future__ import annotations

import numpy as np

SCALARS = ["temperature_kin", "temperature_conf_inverse", "total_laplacian", "total_force2",
           "pressure", "etot_atom", "epot_atom", "epot_eam_atom", "ekin_atom", "etot_cons",
           "etot_cons_err"]


def drain_into_series(driver, series, V0: float, replica: int | None = None) -> int:
    """Drain `driver`'s ring (a replica of a BatchedMDDriver when `replica` is given) and
    append each record to `series` as molecular_dynamics.py:1218-1238 does; V0 is the
    initial box volume. Returns the number of records appended. Raises if records were
    lost to a full ring (a larger ring or more frequent drains avoid that)."""
    rec = driver.drain_samples() if replica is None else driver.drain_samples(replica)
    if rec["lost"]:
        raise RuntimeError(f"{rec['lost']} samples were overwritten before they were drained")
    n = len(rec["time"])
    for k in range(n):
        series.time.append(float(rec["time"][k]))
        for name in SCALARS:
            getattr(series, name).append(float(rec[name][k]))
        series.stress_tensor.append(np.copy(rec["stress_tensor"][k]))
        series.born_stress_tensor.append(np.copy(rec["born_stress_tensor"][k]))
        series.born_elasticity_tensor.append(np.copy(rec["born_elasticity_tensor"][k]))
        V_V0 = float(rec["volume"][k]) / V0
        series.V_V0.append(V_V0)
        series.L_L0.append(V_V0 ** (1.0 / 3.0))
    return n
