"""Learned warm start: a small MLP proposes the zero-pressure lattice constant and initial
C11, C12, C44 of a Cu-Zn FCC alloy from its Zn fraction and temperature, so that a run can
start in (nearly) the equilibrium box instead of equilibrating it by NPT.

* ``generate`` makes the training set with this package's own batched runs: short NPT
  runs of 8x8x8 (2,048-atom) cells over the composition and temperature box, each handed
  over to a short NVT run that estimates C_ij by the fluctuation formula.
* ``WarmStart.fit`` trains the network on the device (mdelast_b200.mlp, hand-written
  forward/backward/Adam kernels) on standardised inputs and targets.
* The same for the ternary Ni-Al-Co system (``generate_nialco``, ``system="nialco"``).
* ``WarmStart.propose`` evaluates it; ``judge`` is the acceptance test the production run
  applies: a proposal whose equilibrated pressure misses the tolerance gets one box
  correction from that pressure and the proposed bulk modulus, and if it still misses it
  is discarded and the plain NPT protocol runs instead (protocol.run_warm_start).

    python -m mdelast_b200.warmstart generate --runs 2048 --out data.npz
    python -m mdelast_b200.warmstart train --data data.npz --out model.npz
"""

from __future__ import annotations

import argparse
import os
import time

import numpy as np

from .protocol import Stages, run_protocol
from .systems import cuzn_cell, vegard_a

WIDTHS = [2, 64, 64, 64, 4]          # (x_Zn, T) -> (a, C11, C12, C44)
X_RANGE, T_RANGE = (0.0, 0.30), (5.0, 900.0)
GEN_STAGES = Stages(npt_therm=1500, npt_prod=1500, nvt_therm=500, nvt_prod=2500,
                    sample_stride=5, rebuild_every=20, checkpoint_every=2500)
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "models", "cuzn_warmstart.npz")

# The ternary Ni-Al-Co system of the bundled Mishin 2013 potential: compositions uniform on
# the simplex, T in [5, 900] K; (x_Ni, x_Al, T) -> (a, C11, C12, C44). Starting lattice
# constants of the pure FCC elements [A] for the linear guess the network replaces.
NIALCO_POTENTIAL = "Mishin_updated-Ni-Al-Co-2013.eam.alloy"
NIALCO_A0 = (3.52, 4.05, 3.54)
NIALCO_WIDTHS = [3, 64, 64, 64, 4]
NIALCO_MODEL = os.path.join(HERE, "models", "nialco_warmstart.npz")
# Chain masses proportional to kT (the reference's choice) make the barostat of a cell
# below ~15 K so light that a linear-guess box several GPa off equilibrium oscillates
# within a few steps and the run ends in NaN (the oracle does the same). The generator
# sets the masses for max(T, NIALCO_MASS_T): the ensemble (T, P) is unchanged, only the
# chains' time scales are.
NIALCO_MASS_T = 50.0


def nialco_guess_a(x, T):
    """Linear (Vegard) lattice constant of an FCC Ni-Al-Co solid solution [A], with a
    thermal expansion of 1.4e-5 / K about 300 K."""
    return float(np.dot(np.asarray(x, float), NIALCO_A0)) * (1.0 + 1.4e-5 * (T - 300.0))


def born_stable(C11, C12, C44):
    """Born's criteria for a cubic crystal: C11 - C12 > 0, C11 + 2 C12 > 0, C44 > 0. Runs
    that fail them (FCC cells of compositions this potential does not keep FCC, mostly
    Al-Co rich with little Ni) carry no meaningful lattice constant or C_ij and are left
    out of the fit."""
    C11, C12, C44 = (np.asarray(v, float) for v in (C11, C12, C44))
    return (C11 - C12 > 0) & (C11 + 2 * C12 > 0) & (C44 > 0)


def _nialco_guess(x, T):
    x = np.atleast_2d(np.asarray(x, float))
    T = np.broadcast_to(np.atleast_1d(np.asarray(T, float)), (len(x),))
    return np.array([nialco_guess_a(a, t) for a, t in zip(x, T)])


def nialco_features(x, T):
    x = np.atleast_2d(np.asarray(x, float))
    return np.concatenate([x[:, :2] * 2 - 1,
                           (np.atleast_1d(np.asarray(T, float)) / T_RANGE[1] * 2 - 1)[:, None]],
                          axis=1)


def generate_nialco(m, tables, n_runs=2048, nside=8, batch=64, seed=2027, stages=GEN_STAGES,
                    precision="mixed", log=None):
    """Training runs of the ternary system, as generate() for Cu-Zn."""
    from .systems import fcc_alloy_cell
    rs = np.random.RandomState(seed)
    out = {k: [] for k in ("x", "T", "a", "C11", "C12", "C44", "P_GPa")}
    done = 0
    while done < n_runs:
        k = min(batch, n_runs - done)
        xs = rs.dirichlet((1.0, 1.0, 1.0), size=k)
        Ts = rs.uniform(*T_RANGE, size=k)
        seeds = rs.randint(0, 2**31 - 1, size=(k, 3))
        a0 = [nialco_guess_a(x, T) for x, T in zip(xs, Ts)]
        cells = [fcc_alloy_cell(tables, nside, x, T=float(T), a_ang=a, ensemble=2,
                                placement_seed=int(s[0]), velocity_seed=int(s[1]),
                                mass_T=max(float(T), NIALCO_MASS_T))
                 for x, T, a, s in zip(xs, Ts, a0, seeds)]
        t0 = time.perf_counter()
        r = run_protocol(m, tables, cells, precision=precision, stages=stages,
                         nvt_seeds=[int(s[2]) for s in seeds], handoff="continue")
        for j in range(k):
            cnt = np.asarray(cells[j].meta["counts"], float)
            out["x"].append(cnt / cnt.sum())
            out["T"].append(float(Ts[j]))
            out["a"].append(a0[j] * r.V_V0[j] ** (1.0 / 3.0))
            for c in ("C11", "C12", "C44"):
                out[c].append(r.C_replicas[j][c])
            out["P_GPa"].append(r.npt_pressure_GPa[j])
        done += k
        if log:
            log(f"{done}/{n_runs} runs, batch of {k} in {time.perf_counter() - t0:.1f} s")
    return {k: np.asarray(v) for k, v in out.items()}


def generate(m, tables, n_runs=2048, nside=8, batch=64, seed=2026, stages=GEN_STAGES,
             precision="mixed", x_range=X_RANGE, T_range=T_RANGE, log=None):
    """Training runs: for each, the Zn fraction and temperature (uniform in the box), the
    NPT production-mean lattice constant [A] and the NVT fluctuation C11, C12, C44 [GPa]."""
    rs = np.random.RandomState(seed)
    out = {k: [] for k in ("x_zn", "T", "a", "C11", "C12", "C44", "P_GPa")}
    done = 0
    while done < n_runs:
        k = min(batch, n_runs - done)
        xs = rs.uniform(*x_range, size=k)
        Ts = rs.uniform(*T_range, size=k)
        seeds = rs.randint(0, 2**31 - 1, size=(k, 3))
        a0 = [vegard_a(x, T) for x, T in zip(xs, Ts)]
        cells = [cuzn_cell(tables, nside, x_zn=float(x), T=float(T), a_ang=a, ensemble=2,
                           placement_seed=int(s[0]), velocity_seed=int(s[1]))
                 for x, T, a, s in zip(xs, Ts, a0, seeds)]
        t0 = time.perf_counter()
        r = run_protocol(m, tables, cells, precision=precision, stages=stages,
                         nvt_seeds=[int(s[2]) for s in seeds], handoff="continue")
        for j in range(k):
            out["x_zn"].append(cells[j].meta["n_zn"] / cells[j].n_atoms)
            out["T"].append(float(Ts[j]))
            out["a"].append(a0[j] * r.V_V0[j] ** (1.0 / 3.0))
            for c in ("C11", "C12", "C44"):
                out[c].append(r.C_replicas[j][c])
            out["P_GPa"].append(r.npt_pressure_GPa[j])
        done += k
        if log:
            log(f"{done}/{n_runs} runs, batch of {k} in {time.perf_counter() - t0:.1f} s")
    return {k: np.asarray(v) for k, v in out.items()}


def features(x_zn, T):
    return np.stack([np.asarray(x_zn, float) / X_RANGE[1] * 2 - 1,
                     np.asarray(T, float) / T_RANGE[1] * 2 - 1], axis=-1)


class WarmStart:
    """The trained proposal network with its target scaling. `system` is "cuzn"
    (composition = the Zn fraction) or "nialco" (composition = (x_Ni, x_Al, x_Co))."""

    TARGETS = ("a", "C11", "C12", "C44")

    def __init__(self, params, y_mean, y_std, widths=WIDTHS, device=0, system="cuzn"):
        from .mlp import MLP
        self.widths = list(widths)
        self.system = system
        self.y_mean, self.y_std = np.asarray(y_mean, float), np.asarray(y_std, float)
        self.net = MLP(self.widths, seed=0, device=device)
        self.net.params = np.asarray(params, np.float32)

    def _features(self, x, T):
        if self.system == "nialco":
            return nialco_features(x, T)
        return features(np.atleast_1d(x), np.atleast_1d(T))

    @classmethod
    def fit(cls, data, steps=6000, lr=2e-3, seed=0, device=0, system="cuzn"):
        """Full-batch Adam on standardised targets. For "nialco" the lattice-constant
        target is the residual a / nialco_guess_a - 1 (a smooth, narrow function of the
        composition where a itself spans 3.5-4.1 A) and runs failing born_stable are
        dropped."""
        from .mlp import MLP
        nialco = system == "nialco"
        widths = NIALCO_WIDTHS if nialco else WIDTHS
        keep = (born_stable(data["C11"], data["C12"], data["C44"]) if nialco
                else np.ones(len(data["T"]), bool))
        d = {k: np.asarray(v)[keep] for k, v in data.items()}
        x = (nialco_features(d["x"], d["T"]) if nialco
             else features(d["x_zn"], d["T"])).astype(np.float32)
        y = np.stack([d[k] for k in cls.TARGETS], axis=1)
        if nialco:
            y[:, 0] = d["a"] / _nialco_guess(d["x"], d["T"]) - 1.0
        mu, sd = y.mean(axis=0), y.std(axis=0) + 1e-12
        net = MLP(widths, seed=seed, device=device)
        loss = net.train(x, ((y - mu) / sd).astype(np.float32), steps, lr)
        ws = cls(net.params, mu, sd, widths, device, system)
        ws.train_loss = loss
        ws.n_train = int(keep.sum())
        return ws

    def propose(self, x, T) -> dict:
        y = self.net(self._features(x, T).astype(np.float32))
        y = y.astype(np.float64) * self.y_std + self.y_mean
        out = {k: y[:, j] for j, k in enumerate(self.TARGETS)}
        if self.system == "nialco":
            out["a"] = (out["a"] + 1.0) * _nialco_guess(x, T)
        out["B"] = (out["C11"] + 2.0 * out["C12"]) / 3.0
        return out

    def save(self, path):
        np.savez(path, params=self.net.params, y_mean=self.y_mean, y_std=self.y_std,
                 widths=np.asarray(self.widths), system=np.asarray(self.system))

    @classmethod
    def load(cls, path=DEFAULT_MODEL, device=0):
        z = np.load(path)
        system = str(z["system"]) if "system" in z else "cuzn"
        return cls(z["params"], z["y_mean"], z["y_std"], [int(w) for w in z["widths"]], device,
                   system)


def judge(p_GPa, tol_GPa=0.2) -> bool:
    """Accept a proposed box when the run's equilibrated mean pressure is within tol."""
    return abs(p_GPa) <= tol_GPa


def _main():
    import sys
    sys.path[:0] = [os.path.join(HERE, "lib")]
    import md_driver_module as m
    from .potentials import find_potential, read_setfl
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["generate", "train"])
    ap.add_argument("--system", choices=["cuzn", "nialco"], default="cuzn")
    ap.add_argument("--runs", type=int, default=2048)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--data", default=os.path.join(HERE, "models", "cuzn_warmstart_data.npz"))
    ap.add_argument("--out", default=None)
    ap.add_argument("--steps", type=int, default=6000)
    a = ap.parse_args()
    os.makedirs(os.path.join(HERE, "models"), exist_ok=True)
    nialco = a.system == "nialco"
    if a.cmd == "generate":
        if nialco:
            t = read_setfl(find_potential(NIALCO_POTENTIAL))
            d = generate_nialco(m, t, n_runs=a.runs, batch=a.batch, log=print)
        else:
            t = read_setfl(find_potential("ZnCu.eam.alloy"))
            d = generate(m, t, n_runs=a.runs, batch=a.batch, log=print)
        np.savez(a.out or a.data, **d)
    else:
        d = dict(np.load(a.data))
        ws = WarmStart.fit(d, steps=a.steps, system=a.system)
        ws.save(a.out or (NIALCO_MODEL if nialco else DEFAULT_MODEL))
        print("train loss (standardised)", ws.train_loss)


if __name__ == "__main__":
    _main()
