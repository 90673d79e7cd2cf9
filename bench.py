#!/usr/bin/env python
"""Benchmark of the EAM force-and-stress step (one MD step of mdelast's integrate()).

Workload (default, one GPU): the Cu-6 at.% Zn FCC cell of 15x15x15 unit cells (13,500
atoms, 810 Zn placed by RandomState(42)), Cu-Zn EAM (ZnCu.eam.alloy), NVT at 300 K with
dt = 2 fs, a 10-link Nose-Hoover chain, neighbour list with r_skin = 1.2 rebuilt every 20
steps, and the Born tensor / Laplacian sampled every step - the production protocol of
the reference's sample case at the size of its 13,500-atom configuration. Positions come
from the FCC builder and Maxwell-Boltzmann velocities from the seeded stream; no dataset.

A step = one integrate() (with the list rebuild on every 20th). value = atom-steps/s over
all ranks, timed on the device with CUDA events, L2 flushed before every timed step.
e2e = the same metric through the public API (md_driver_module, the reference's plugin
interface): driver created from host arrays, integrate() plus the per-step observable
reads of molecular_dynamics.py's append_sample, final positions and velocities read back;
wall-clock time of all of it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--replicas R] [--precision fp64|mixed]

--impl reference times the reference's own C++ core (compiled in place by oracle/Makefile)
on the host's cores on the same workload: one process per core, each timing a bounded
sample of steps (including one O(N^2) list rebuild, amortised over the 20-step cadence).
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "mdelast_b200", "lib")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "atom-steps/s"
WORKLOAD = "cuzn6_fcc15_13500_nvt300"
NSIDE, N_ZN, T_K, DT, SKIN, REBUILD = 15, 810, 300.0, 2e-15, 1.2, 20
L2_FLUSH_BYTES = 512 << 20


# ----------------------------------------------------------------------------- inputs
def make_case():
    """Positions, types, velocities and thermostat state of the workload (cgs)."""
    import numpy as np

    from mdelast_b200.lattice import fcc_lattice, initial_state, substitute
    from mdelast_b200.potentials import find_potential, read_setfl
    from mdelast_b200.units import Units as U

    path = find_potential("ZnCu.eam.alloy")
    if path is None:
        raise SystemExit("ZnCu.eam.alloy not found (make -C oracle potentials)")
    t = read_setfl(path)
    names = [e[0] for e in t.elements]
    pos, L = fcc_lattice(NSIDE, 3.6345 * U.angstrom)
    typ = substitute(len(pos), N_ZN, 42, names.index("Cu"), names.index("Zn"))
    mass = np.array(t.masses)[typ]
    st = initial_state(mass, T_K, T_K, 5e-14, 5e-13, random_seed=0)
    drg = 3.6345 * U.angstrom / 500
    rg = [(k + 0.5) * drg for k in range(int(L / 2 / drg))]
    return dict(tables=t, positions=pos, velocities=st.velocities, types=typ, L=L, st=st, rg=rg)


def make_driver(m, c, precision, device=0):
    import numpy as np

    from mdelast_b200.potentials import make_objects
    from mdelast_b200.units import Units as U

    t, st = c["tables"], c["st"]
    _, pots, eams = make_objects(m, t)
    P = [m.Vector3d(*p) for p in c["positions"]]
    V = [m.Vector3d(*v) for v in c["velocities"]]
    th = m.Thermostat(T_K, list(st.thermo_q), list(st.thermo_p_eta), st.Nf)
    baro = m.Barostat(1e-10 * U.GPa, st.baro_w, st.baro_p_eps,
                      m.Thermostat(T_K, list(st.baro_q), list(st.baro_p_eta), 1.0))
    return m.MDDriver(P, V, m.PotentialVector(pots), m.EAMVector(eams), m.MDDriver.NVT,
                      m.MDDriver.THERMOSTAT_KINETIC, th, baro, m.Box(np.diag([c["L"]] * 3)),
                      c["rg"], st.Nf, list(t.masses), [int(x) for x in c["types"]], DT, True,
                      SKIN, 1e3, precision=precision, device=device)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, n in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- ours
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    import md_driver_module as m

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    c = make_case()
    N = len(c["positions"])
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    drivers = [make_driver(m, c, args.precision, local_rank) for _ in range(args.replicas)]
    for d in drivers:  # warm-up: graphs captured, clocks up
        d.run(max(args.warmup, 1), REBUILD, 1, False)
        d.synchronize()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # timed region: K steps, L2 flushed before each
    barrier()
    total_ms = 0.0
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            for d in drivers:
                total_ms += d.run(1, REBUILD, 1, True)
    barrier()
    clocks = clk.summary()
    t_dev = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_dev, op=dist.ReduceOp.MAX)
    ms_total = float(t_dev.item())
    atoms_all = N * args.replicas * world
    value = atoms_all * args.steps / (ms_total * 1e-3)

    # per-kernel device times (same flushing), for the roofline of the dominant kernel
    d0 = drivers[0]
    kt = np.zeros(6)
    nk = max(3, min(args.steps, 20))
    for _ in range(nk):
        flush.zero_()
        torch.cuda.synchronize()
        kt += np.array(d0.kernel_times(1))
    kt /= nk
    point, _ = d0.neighbor_list()
    nbar = float(point[-1]) / N  # half-list entries per atom (the reference's point[N]/N)
    bytes_force = N * (4.0 * nbar + 108.0)  # list indices + own record + F' + kick r/w + force
    names = ["k_pre", "k_kick_drift", "k_density", "k_force", "k_post", "k_nbr_build"]
    kshare = {n: float(t) for n, t in zip(names, kt)}
    hbm = peaks.get("hbm_gbs")
    achieved = bytes_force / (kt[3] * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": "k_force", "achieved": achieved,
            "peak": hbm if hbm else 6650.0, "unit": "GB/s",
            "peak_source": "measured" if hbm else "fallback",
            "frac": achieved / (hbm if hbm else 6650.0),
            "traffic": TRAFFIC_PER_LAUNCH.get((args.precision, "k_force")),
            "algorithmic_bytes_per_launch": bytes_force, "half_list_nbar": nbar,
            "kernel_ms": kshare}

    # e2e through the public API, host wall clock (rank's own work, max over ranks)
    e2e_steps = max(args.steps, REBUILD)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dd = [make_driver(m, c, args.precision, local_rank) for _ in range(args.replicas)]
    for s in range(e2e_steps):
        for d in dd:
            if s % REBUILD == 0:
                d.calculate_neighbors()
            d.sample_observables = True
            d.integrate()
            _ = (d.time, d.temperature_kin, d.temperature_conf_inverse, d.total_laplacian,
                 d.total_force2, d.pressure, np.copy(d.stress_tensor), d.etot_atom, d.epot_atom,
                 d.epot_eam_atom, d.ekin_atom, d.etot_cons, d.etot_cons_err,
                 np.copy(d.born_stress_tensor), np.copy(d.born_elasticity_tensor),
                 d.box.volume())
    for d in dd:
        _ = (d.atoms_array(m.ATOM_POSITIONS), d.atoms_array(m.ATOM_VELOCITIES))
    t_e2e = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    e2e_value = atoms_all * e2e_steps / float(t_e2e.item())
    h2d = args.replicas * (N * (6 * 8 + 4) + c["tables"].phi.size * 3 * 8 +
                           c["tables"].rho.size * 3 * 8 + c["tables"].F.size * 3 * 8)
    d2h_obs = 78 * 8 + 8
    d2h = args.replicas * (e2e_steps * d2h_obs + 2 * N * 24)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(c, max_seconds=20.0)
    launches = args.steps * args.replicas * 5 + (args.steps // REBUILD + 1) * args.replicas * 3
    line = {
        "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32 pair math, f64 sums",
        "data": "synthetic (seeded FCC lattice, Maxwell-Boltzmann velocities)",
        "config": {"workload": WORKLOAD, "atoms_per_replica": N, "replicas_per_gpu": args.replicas,
                   "potential": "ZnCu.eam.alloy", "ensemble": "NVT 300 K", "dt_fs": 2,
                   "neighbor_list": f"r_skin {SKIN}, rebuilt every {REBUILD} steps",
                   "sample_observables": "every step", "precision": args.precision,
                   "l2": "flushed (512 MiB write) before every timed step",
                   "parallelism": f"replicas only, dp{world}"},
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "atom-steps/s",
                "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
                "steps": e2e_steps, "api": "md_driver_module.MDDriver"},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    del drivers, dd
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_force launch of this workload
# (profiles/k_force_cuzn6_13500.md); None until captured
TRAFFIC_PER_LAUNCH: dict = {}


# ----------------------------------------------------------------------------- reference
def _ref_worker(args):
    """One host process: the reference's C++ core on the workload; returns s/step."""
    sys.path.insert(0, ROOT)
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)  # the reference prints from C++
    import numpy as np

    from oracle.ref import RefDriver
    c = make_case()
    st = c["st"]
    from mdelast_b200.units import Units as U
    n_steps = args
    d = RefDriver(c["tables"], c["positions"], c["velocities"], c["types"], ensemble=1,
                  thermo=(T_K, st.thermo_q, st.thermo_p_eta, st.Nf),
                  baro=(1e-10 * U.GPa, st.baro_w, st.baro_p_eps),
                  baro_thermo=(T_K, st.baro_q, st.baro_p_eta, 1.0),
                  box=np.diag([c["L"]] * 3), rg=c["rg"], Nf=st.Nf, dt=DT, neighbors=True,
                  r_skin=SKIN)
    t0 = time.perf_counter()
    d.calculate_neighbors()
    t_list = time.perf_counter() - t0
    t0 = time.perf_counter()
    d.integrate(n_steps)
    t_steps = (time.perf_counter() - t0) / n_steps
    return t_steps + t_list / REBUILD


def cpu_sample(c, max_seconds=20.0, n_steps=8):
    """The reference's C++ core (oracle/_ref) on one core: list build + n steps."""
    from oracle import ref
    if not ref.available("ref"):
        return None
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        per_step = pool.map(_ref_worker, [n_steps])[0]
    N = len(c["positions"])
    return {"value": N / per_step, "unit": "atom-steps/s", "cores": 1, "kind": "reference",
            "sample": f"{N}-atom workload cell: one list build + {n_steps} sampled steps, "
                      f"list cost amortised over {REBUILD} steps; {per_step * 1e3:.1f} ms/step"}


def run_reference(args, rank):
    if rank != 0:
        return
    from oracle import ref
    if not ref.available("ref"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libmdelast_ref.so not built (make -C oracle ref)"}))
        return
    cores = os.cpu_count() or 1
    n_steps = max(1, min(args.steps, 10))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        per_step = pool.map(_ref_worker, [n_steps] * cores)
    wall = time.perf_counter() - t0
    N = NSIDE**3 * 4
    value = sum(N / t for t in per_step)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atom-steps/s",
        "n_gpus": 0, "steps": n_steps, "warmup": 0,
        "ms_per_step": statistics.mean(per_step) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "atoms_per_replica": N, "replicas": cores,
                   "parallelism": f"{cores} independent single-thread processes"},
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": cores,
                         "kind": "reference",
                         "sample": f"per process: one O(N^2) list build + {n_steps} steps of "
                                   f"the {N}-atom cell (list amortised over {REBUILD}); "
                                   f"wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--replicas", type=int, default=1)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
