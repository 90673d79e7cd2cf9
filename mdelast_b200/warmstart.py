"""Learned warm start: a small MLP proposes the zero-pressure lattice constant and initial
C11, C12, C44 of a Cu-Zn FCC alloy from its Zn fraction and temperature, so that a run can
start in (nearly) the equilibrium box instead of equilibrating it by NPT.

* ``generate`` makes the training set with this package's own batched runs: short NPT
  runs of 8x8x8 (2,048-atom) cells over the composition and temperature box, each handed
  over to a short NVT run that estimates C_ij by the fluctuation formula.
* ``WarmStart.fit`` trains the network on the device (mdelast_b200.mlp, hand-written
  forward/backward/Adam kernels) on standardised inputs and targets.
* ``WarmStart.propose`` evaluates it; ``judge`` is the acceptance test the production run
  applies: a proposal whose equilibrated pressure misses the tolerance is discarded and
  the plain NPT protocol runs instead (protocol.run_warm_start).

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
    """The trained proposal network with its target scaling."""

    TARGETS = ("a", "C11", "C12", "C44")

    def __init__(self, params, y_mean, y_std, widths=WIDTHS, device=0):
        from .mlp import MLP
        self.widths = list(widths)
        self.y_mean, self.y_std = np.asarray(y_mean, float), np.asarray(y_std, float)
        self.net = MLP(self.widths, seed=0, device=device)
        self.net.params = np.asarray(params, np.float32)

    @classmethod
    def fit(cls, data, steps=6000, lr=2e-3, seed=0, device=0):
        from .mlp import MLP
        x = features(data["x_zn"], data["T"]).astype(np.float32)
        y = np.stack([data[k] for k in cls.TARGETS], axis=1)
        mu, sd = y.mean(axis=0), y.std(axis=0) + 1e-12
        net = MLP(WIDTHS, seed=seed, device=device)
        loss = net.train(x, ((y - mu) / sd).astype(np.float32), steps, lr)
        ws = cls(net.params, mu, sd, WIDTHS, device)
        ws.train_loss = loss
        return ws

    def propose(self, x_zn, T) -> dict:
        y = self.net(features(np.atleast_1d(x_zn), np.atleast_1d(T)).astype(np.float32))
        y = y.astype(np.float64) * self.y_std + self.y_mean
        return {k: y[:, j] for j, k in enumerate(self.TARGETS)}

    def save(self, path):
        np.savez(path, params=self.net.params, y_mean=self.y_mean, y_std=self.y_std,
                 widths=np.asarray(self.widths))

    @classmethod
    def load(cls, path=DEFAULT_MODEL, device=0):
        z = np.load(path)
        return cls(z["params"], z["y_mean"], z["y_std"], [int(w) for w in z["widths"]], device)


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
    ap.add_argument("--runs", type=int, default=2048)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--data", default=os.path.join(HERE, "models", "cuzn_warmstart_data.npz"))
    ap.add_argument("--out", default=None)
    ap.add_argument("--steps", type=int, default=6000)
    a = ap.parse_args()
    os.makedirs(os.path.join(HERE, "models"), exist_ok=True)
    if a.cmd == "generate":
        t = read_setfl(find_potential("ZnCu.eam.alloy"))
        d = generate(m, t, n_runs=a.runs, batch=a.batch, log=print)
        np.savez(a.out or a.data, **d)
    else:
        d = dict(np.load(a.data))
        ws = WarmStart.fit(d, steps=a.steps)
        ws.save(a.out or DEFAULT_MODEL)
        print("train loss (standardised)", ws.train_loss)


if __name__ == "__main__":
    _main()
