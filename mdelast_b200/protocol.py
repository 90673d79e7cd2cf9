"""The elastic-constant protocol of the reference's sample case on the device, for one cell
or a batch of replicas, with running estimates for time-to-solution measurements.

The reference (sample_case/run.py:200-300) runs an NPT stage (thermalisation, then a
production window whose mean V/V0 it keeps), hands the final NPT snapshot over to an NVT
stage scaled by that mean (V/V0)^(1/3) with fresh velocities, and estimates C_ij from the
NVT production window by the fluctuation formula (molecular_dynamics.py:826-958). Here the
same stages run on BatchedMDDriver: samples stay on the device (mdelast_driver_fluct_*),
the handoff takes the snapshot from device state, and the NVT production is cut into
checkpoints at which every replica's C_ij estimate is read, so that the wall time to reach
a given accuracy can be measured. With several replicas the estimate is the mean of the
replicas' estimates.

The reference's handoff multiplies the snapshot's positions by (V/V0)^(1/3), but those
positions are already in the expanded NPT box; handoff="box" (the default) places the
snapshot's scaled coordinates in the mean box instead, and handoff="reference" keeps the
reference's arithmetic (see _nvt_cells).
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field, replace

import numpy as np

from .dump import handoff_positions
from .lattice import initial_state
from .systems import Cell, make_batch
from .units import Units as U

RING = 1024  # records per replica in the device sample ring (the driver's default)


@dataclass
class Stages:
    npt_therm: int = 10_000
    npt_prod: int = 10_000
    nvt_therm: int = 10_000
    nvt_prod: int = 90_000
    sample_stride: int = 1
    rebuild_every: int = 20
    checkpoint_every: int = 5_000


@dataclass
class ProtocolResult:
    precision: str
    replicas: int
    atoms_per_replica: int
    stages: Stages
    V_V0: list                  # NPT production mean per replica
    npt_pressure_GPa: list      # NPT production mean pressure per replica
    C: dict                     # final C11, C12, C44 [GPa], mean over replicas
    C_replicas: list            # per replica
    checkpoints: list = field(default_factory=list)  # (nvt prod steps, wall s, C11, C12, C44)
    wall_s: float = 0.0
    wall_npt_s: float = 0.0
    accepted_start: bool = True
    corrections: int = 0        # box corrections of a warm start before it was accepted


def _nvt_cells(tables, cells, positions, coordinates, V_V0, seeds, handoff):
    """Cells of the NVT stage in the NPT production-mean box L0 (V/V0)^(1/3).

    handoff "reference": the snapshot's positions times (V/V0)^(1/3), as
    sample_case/run.py:273-279 does, wrapped into the mean box as
    benchmarks/l12_cuzn3_5K/run.py:127-140 does; the snapshot's positions are already in the NPT box,
    so the lattice is stretched a second time and squeezed at the periodic boundary (a
    misfit that takes the NVT stage tens of picoseconds to anneal). "box": the snapshot's
    scaled coordinates placed in the mean box. Both draw fresh velocities and chain
    momenta from the seed, as the reference's NVT stage does. "continue": like "box", with
    the NPT stage's velocities, thermostat momenta and thermostat masses carried over."""
    out = []
    for k, (c, v, seed) in enumerate(zip(cells, V_V0, seeds)):
        scale = v ** (1.0 / 3.0)
        L = c.box * scale
        if handoff == "reference":
            # scaled, then wrapped into the mean box as benchmarks/l12_cuzn3_5K/run.py:127-140
            # does (x >= L/2 moves down by L, x < -L/2 up by L)
            pos, _ = handoff_positions(positions[k][0], v)
            pos = pos - L * np.floor((pos + 0.5 * L) / L)
        else:
            u = np.asarray(coordinates[k], dtype=float)
            pos = (u - np.floor(u + 0.5)) * L
        mass = np.array(tables.masses)[c.types]
        st = initial_state(mass, c.T, c.T, 5e-14, 5e-13, random_seed=seed)
        vel, p_eta, q = st.velocities, st.thermo_p_eta, st.thermo_q
        if handoff == "continue":
            vel, p_eta, q = positions[k][1], positions[k][2], c.thermo_q
        out.append(replace(c, positions=pos, velocities=np.asarray(vel), box=L, ensemble=1,
                           thermo_q=np.asarray(q), thermo_p_eta=np.asarray(p_eta),
                           baro_q=st.baro_q, baro_p_eta=st.baro_p_eta, baro_w=st.baro_w,
                           baro_p_eps=st.baro_p_eps, Nf=st.Nf))
    return out


def run_protocol(m, tables, cells: list[Cell], precision="fp64", stages: Stages | None = None,
                 nvt_seeds=None, judge=None, autotune=True, npt_fallback: Stages | None = None,
                 handoff="box") -> ProtocolResult:
    """NPT -> handoff -> NVT on all `cells` at once. `judge(V_V0, p_GPa)` (optional) decides,
    after the NPT stage, whether each replica's equilibrated box and pressure are within
    tolerance; if any is not, the NPT stage is rerun with `npt_fallback` stages from the
    original cells (the plain method as fallback). `handoff` is "reference", "box" or
    "continue" (see _nvt_cells). Returns the result with checkpoints of the running C_ij
    estimate; wall times include driver creation and every readout."""
    st = stages or Stages()
    seeds = list(nvt_seeds) if nvt_seeds is not None else [1000 + k for k in range(len(cells))]
    t0 = time.perf_counter()
    accepted = True

    def npt_stage(s):
        b = make_batch(m, tables, [replace(c, ensemble=2) for c in cells], r_skin=1.2,
                       precision=precision)
        if autotune:
            b.autotune(2)
        b.run(s.npt_therm, s.rebuild_every, s.sample_stride, False)
        for r in range(b.n_replicas):
            b.drain_samples(r)
        b.fluctuation_start()
        # production in chunks the sample ring holds, pressures drained after each
        psum = np.zeros(b.n_replicas)
        pn = np.zeros(b.n_replicas)
        done = 0
        while done < s.npt_prod:
            n = min(RING * s.sample_stride, s.npt_prod - done)
            b.run(n, s.rebuild_every, s.sample_stride, False)
            done += n
            for r in range(b.n_replicas):
                rec = b.drain_samples(r)
                psum[r] += float(np.sum(rec["pressure"]))
                pn[r] += len(rec["pressure"])
        V_V0 = [float(b.fluctuations(r)["mean"][7]) / float(np.prod(c.box))
                for r, c in enumerate(cells)]
        p = [psum[r] / max(pn[r], 1.0) / U.GPa for r in range(b.n_replicas)]
        snap = [(np.asarray(b.atoms(r, m.ATOM_POSITIONS)),
                 np.asarray(b.atoms(r, m.ATOM_VELOCITIES)), b.chain(r, 0)[1])
                for r in range(b.n_replicas)]
        crd = [np.asarray(b.atoms(r, m.ATOM_COORDINATES)) for r in range(b.n_replicas)]
        del b
        return V_V0, p, snap, crd

    V_V0, p_npt, snap, crd = npt_stage(st)
    if judge is not None and not all(judge(v, p) for v, p in zip(V_V0, p_npt)):
        accepted = False
        V_V0, p_npt, snap, crd = npt_stage(npt_fallback or Stages())
    t_npt = time.perf_counter() - t0

    nvt = _nvt_cells(tables, cells, snap, crd, V_V0, seeds, handoff)
    b = make_batch(m, tables, nvt, r_skin=1.2, precision=precision)
    if autotune:
        b.autotune(2)
    b.set_sample_ring(0)  # the fluctuation sums are all this stage reads
    b.run(st.nvt_therm, st.rebuild_every, st.sample_stride, False)
    b.fluctuation_start()
    done, checkpoints, Cr = 0, [], []
    while done < st.nvt_prod:
        n = min(st.checkpoint_every, st.nvt_prod - done)
        b.run(n, st.rebuild_every, st.sample_stride, False)
        done += n
        Cr = [b.elastic_constants(r) for r in range(b.n_replicas)]
        C = [float(np.mean([c[k] for c in Cr])) / U.GPa for k in ("C11", "C12", "C44")]
        checkpoints.append((done, time.perf_counter() - t0, *C))
    wall = time.perf_counter() - t0
    C_rep = [{k: c[k] / U.GPa for k in ("C11", "C12", "C44")} for c in Cr]
    C = {k: float(np.mean([c[k] for c in C_rep])) for k in ("C11", "C12", "C44")}
    return ProtocolResult(precision=precision, replicas=len(cells),
                          atoms_per_replica=cells[0].n_atoms, stages=st, V_V0=V_V0,
                          npt_pressure_GPa=p_npt, C=C, C_replicas=C_rep,
                          checkpoints=checkpoints, wall_s=wall, wall_npt_s=t_npt,
                          accepted_start=accepted)


def time_to_within(result: ProtocolResult, target: dict, tol: float = 0.02):
    """Wall time (s) of the first checkpoint from which C11, C12 and C44 all stay within
    `tol` (relative) of `target` to the end of the run, or None."""
    ok_from = None
    for (_, wall, c11, c12, c44) in result.checkpoints:
        good = all(abs(v / target[k] - 1.0) <= tol
                   for v, k in ((c11, "C11"), (c12, "C12"), (c44, "C44")))
        if good and ok_from is None:
            ok_from = wall
        elif not good:
            ok_from = None
    return ok_from


def _corrected_cells(m, b, cells, p_GPa, bulk_GPa):
    """The batch's current states in boxes scaled by 1 + p / (3 B) per edge (one Newton
    step of p(V) = -B ln(V / V_eq)): scaled coordinates, velocities and thermostat
    momenta carried over."""
    out = []
    for r, c in enumerate(cells):
        L = c.box * (1.0 + p_GPa[r] / (3.0 * bulk_GPa[r]))
        u = np.asarray(b.atoms(r, m.ATOM_COORDINATES), dtype=float)
        out.append(replace(c, positions=(u - np.floor(u + 0.5)) * L, box=L,
                           velocities=np.asarray(b.atoms(r, m.ATOM_VELOCITIES)),
                           thermo_p_eta=np.asarray(b.chain(r, 0)[1])))
    return out


def run_warm_start(m, tables, cells: list[Cell], precision="mixed",
                   stages: Stages | None = None, judge=None, check_steps=1000,
                   fallback: Stages | None = None, autotune=True, bulk_GPa=None,
                   max_corrections=1) -> ProtocolResult:
    """The production run started in a proposed equilibrium box (`cells`, NVT, built at
    the proposed lattice constant), with no NPT stage: NVT thermalisation, then production
    whose first `check_steps` steps also serve as the acceptance window. If `judge(p_GPa)`
    rejects any replica's mean pressure over that window and the proposal's bulk moduli
    `bulk_GPa` are given, every box is corrected from its window pressure
    (_corrected_cells) and thermalisation (half as long) and window rerun, up to
    `max_corrections` times; a proposal still rejected is discarded and the plain protocol
    (run_protocol with `fallback` stages) runs from the original cells."""
    st = stages or Stages(npt_therm=0, npt_prod=0, nvt_therm=1000, nvt_prod=2000,
                          sample_stride=5, checkpoint_every=500)
    t0 = time.perf_counter()
    work = [replace(c, ensemble=1) for c in cells]
    n = min(check_steps, st.nvt_prod)
    corrections, therm = 0, st.nvt_therm
    while True:
        b = make_batch(m, tables, work, r_skin=1.2, precision=precision)
        if autotune:
            b.autotune(2)
        b.run(therm, st.rebuild_every, st.sample_stride, False)
        for r in range(b.n_replicas):
            b.drain_samples(r)
        b.fluctuation_start()
        b.run(n, st.rebuild_every, st.sample_stride, False)
        p = [float(np.mean(b.drain_samples(r)["pressure"])) / U.GPa
             for r in range(b.n_replicas)]
        if judge is None or all(judge(x) for x in p):
            break
        if bulk_GPa is None or corrections >= max_corrections:
            del b
            res = run_protocol(m, tables, cells, precision=precision,
                               stages=fallback or Stages(), autotune=autotune)
            res.accepted_start = False
            res.corrections = corrections
            res.wall_s = time.perf_counter() - t0
            return res
        work = _corrected_cells(m, b, work, p, bulk_GPa)
        del b
        corrections += 1
        therm = st.nvt_therm // 2
    b.set_sample_ring(0)
    done, checkpoints, Cr = n, [], []
    while True:
        if done % st.checkpoint_every == 0 or done >= st.nvt_prod:
            Cr = [b.elastic_constants(r) for r in range(b.n_replicas)]
            C = [float(np.mean([c[k] for c in Cr])) / U.GPa for k in ("C11", "C12", "C44")]
            checkpoints.append((done, time.perf_counter() - t0, *C))
        if done >= st.nvt_prod:
            break
        k = min(st.checkpoint_every - done % st.checkpoint_every, st.nvt_prod - done)
        b.run(k, st.rebuild_every, st.sample_stride, False)
        done += k
    wall = time.perf_counter() - t0
    C_rep = [{k: c[k] / U.GPa for k in ("C11", "C12", "C44")} for c in Cr]
    C = {k: float(np.mean([c[k] for c in C_rep])) for k in ("C11", "C12", "C44")}
    res = ProtocolResult(precision=precision, replicas=len(cells),
                         atoms_per_replica=cells[0].n_atoms, stages=st,
                         V_V0=[float(np.prod(w.box) / np.prod(c.box)) for w, c in zip(work, cells)],
                         npt_pressure_GPa=p, C=C, C_replicas=C_rep,
                         checkpoints=checkpoints, wall_s=wall, wall_npt_s=0.0,
                         accepted_start=True, corrections=corrections)
    return res
