#!/usr/bin/env python
"""Benchmark of the EAM force-and-stress step (one MD step of mdelast's integrate()).

Workload: the Cu-6 at.% Zn FCC cell of 15x15x15 unit cells (13,500 atoms, 810 Zn placed by
RandomState(42)), Cu-Zn EAM (ZnCu.eam.alloy), NVT at 300 K, dt = 2 fs, 10-link
Nose-Hoover chain, neighbour list with r_skin = 1.2 rebuilt every 20 steps, Born tensor
and Laplacian sampled every step - the production protocol of the reference's sample case
at the size of its 13,500-atom configuration. Positions from the FCC builder, velocities
Maxwell-Boltzmann from seeded streams; no dataset.

Timed: R replicas of that cell (default 16, mixed precision, velocity seeds 0..R-1)
advanced together by BatchedMDDriver; a step = one integrate() of every replica (the
list rebuild on every 20th). Setup (untimed): 400 equilibration steps from the lattice,
launch shapes chosen on real steps (autotune_steps), then the W warm-up steps. value = atom-steps/s over all ranks from CUDA events around
the K timed steps; the replicas' state is larger than the L2, so no flush is needed. The
plain path (one FP64 cell, L2 flushed before every timed step) is reported beside it.
e2e = the same batched metric through the public API: the batch created from host arrays,
every step the per-replica observables molecular_dynamics.py's append_sample reads, the
final positions and velocities read back; wall-clock time of all of it (the batch's
destruction afterwards is reported in e2e.phases, not timed).
e2e_long: the same through a 1,000-step session, which amortises the batch's creation.
dropin_run_loop: one cell driven through MDDriver with the calls the reference's own run
loop makes per step (integrate() and the 17 reads of append_sample), wall clock.
time_to_cij (rank 0, --no-cij skips it): wall time to C11/C12/C44 within 2 % of the FP64
plain protocol's result, the plain protocol (one FP64 cell, NPT then NVT as the reference's
sample case, 120k steps) against 4 mixed-precision replicas started in the box the trained
warm-start network proposes, and against the same replicas without the network
(ablation_no_network; see time_to_cij). The same comparison runs for the 108,000-atom
Ni-Al-Co cell and the ternary network (time_to_cij_nialco; --no-cij-nialco skips it).
mixed_vs_fp64 (--no-precision-report skips it): the mixed path's error against FP64 on
the workload cell, per quantity over a same-seed window and for C_ij over paired replicas.
other_configs: 64 uneven replicas, the 32,000-atom L1_2 cell and configuration C1 (pure
Cu, single-element Cu01 tables, 500 atoms, FP64).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--replicas R] [--precision fp64|mixed]

--impl reference times the reference's own C++ core (compiled in place by oracle/Makefile)
on the host's cores on the same cell: one process per core, each timing a bounded sample
of steps (including one O(N^2) list rebuild, amortised over the 20-step cadence).
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
E2E_LONG = 1000
TUNE_STEPS = 3  # steps per candidate launch shape (autotune_steps)
# Untimed steps from the lattice start before tuning and timing. Near the perfect lattice
# the pair distances fall on few table intervals and the pair passes run up to 30 % faster
# than in the thermalised cell a production run spends its time in; 400 steps (0.8 ps)
# reach the thermalised cost.
EQUIL_STEPS = 400


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, period_ms=20):
        self.gpu = gpu_index
        self.period_ms = period_ms
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
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
                "reasons": sorted(reasons), "samples": len(sm),
                "window": "warm-up and timed steps, every 20 ms"}


# ----------------------------------------------------------------------------- ours
KERNELS = ["k_pre", "k_kick_drift", "k_density", "k_force", "k_post", "k_nbr_build"]


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    import md_driver_module as m
    from mdelast_b200.systems import make_batch, make_driver

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    t, base = make_cells(1, workload=args.workload)
    cells = make_cells(args.replicas, seed0=1000 * rank, workload=args.workload)[1]
    N = base[0].n_atoms
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # --- batched replicas: the timed workload. Its state (list, tables, atoms) is far
    # larger than the 126 MB L2 for 16 replicas, so steps run back to back unflushed.
    b = make_batch(m, t, cells, dt=DT, r_skin=SKIN, precision=args.precision,
                   device=local_rank)
    # equilibration from the lattice (untimed), then the launch shapes of the pair passes
    # timed on this workload and kept, or the shapes given by --launch
    b.run(EQUIL_STEPS, REBUILD, 1, False)
    if args.launch:
        tpa_d, tpa_f, blk_d, blk_f = (int(v) for v in args.launch.split(","))
        b.set_launch(tpa_d, tpa_f, blk_d, blk_f)
        if args.force_tables != "auto" and b.force_staging is not None:
            b.force_staging = args.force_tables == "shared"
        tune = {"tpa_density": tpa_d, "tpa_force": tpa_f, "blocks_density": blk_d,
                "blocks_force": blk_f, "given": True, "force_staged": bool(b.force_staging)}
    else:
        # shapes chosen on real steps (the state advances)
        tune = b.autotune_steps(TUNE_STEPS, REBUILD)
    # the sampler starts before the warm-up steps so that a short timed region still has
    # samples (the timed steps follow the warm-up back to back)
    with ClockSampler(local_rank) as clk:
        time.sleep(0.1)
        b.run(args.warmup, REBUILD, 1, False)
        b.synchronize()
        barrier()
        ms_total = b.run(args.steps, REBUILD, 1, True)
        barrier()
    clocks = clk.summary()
    t_dev = torch.tensor([ms_total], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_dev, op=dist.ReduceOp.MAX)
    ms_total = float(t_dev.item())
    atoms_all = b.n_atoms * world
    value = atoms_all * args.steps / (ms_total * 1e-3)
    status_ok = all((b.observables(r)["status"] & 0xff) == 0 for r in range(b.n_replicas))

    # per-kernel device times of the batched step (events between kernels, sampled steps)
    kt = np.array(b.kernel_times(max(3, min(args.steps, 10))))
    nbar = half_list_nbar(m, t, base[0])
    bytes_force = b.n_atoms * (4.0 * nbar + 108.0)
    hbm = peaks.get("hbm_gbs")
    peak = hbm if hbm else 6650.0
    achieved = bytes_force / (kt[3] * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": "k_force" + ("_mx" if args.precision == "mixed" else ""),
            "achieved": achieved, "peak": peak, "unit": "GB/s",
            "peak_source": "measured" if hbm else "fallback", "frac": achieved / peak,
            "traffic": TRAFFIC_PER_LAUNCH.get((args.precision, args.replicas,
                                               bool(tune.get("force_staged"))))
            if args.workload == WORKLOAD else None,
            "traffic_source": "ncu single-pass capture at 16 replicas, caches not flushed",
            "force_tables": "shared memory" if tune.get("force_staged") else "L1",
            "algorithmic_bytes_per_launch": bytes_force, "half_list_nbar": nbar,
            "kernel_ms": {n: float(x) for n, x in zip(KERNELS, kt)}}
    del b

    # --- the plain path for comparison: one FP64 cell, L2 flushed before every timed step
    plain = None
    if not args.no_plain:
        flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        d = make_driver(m, t, base[0], dt=DT, r_skin=SKIN, precision="fp64", device=local_rank)
        d.run(EQUIL_STEPS, REBUILD, 1, False)
        tune_plain = d.autotune_steps(TUNE_STEPS, REBUILD)
        d.run(args.warmup, REBUILD, 1, False)
        d.synchronize()
        ms = 0.0
        n_plain = min(args.steps, 100)
        for _ in range(n_plain):
            flush.zero_()
            torch.cuda.synchronize()
            ms += d.run(1, REBUILD, 1, True)
        plain = {"value": N * n_plain / (ms * 1e-3), "unit": "atom-steps/s",
                 "ms_per_step": ms / n_plain, "precision": "fp64", "replicas": 1,
                 "l2": "flushed before every timed step", "launch": tune_plain}
        del d, flush

    # --- e2e through the public API: batch created from host arrays, every step the
    # per-replica observables that append_sample reads, final positions/velocities back
    e2e_steps = max(args.steps, REBUILD)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    phases = {}
    if not args.no_e2e:
        bb = make_batch(m, t, cells, dt=DT, r_skin=SKIN, precision=args.precision,
                        device=local_rank)
        # the shapes tuned above for this workload, reused as a caller would
        bb.set_launch(tune["tpa_density"], tune["tpa_force"], tune["blocks_density"],
                      tune["blocks_force"])
        t1 = time.perf_counter()
        for s in range(e2e_steps):
            bb.run(1, REBUILD, 1, False)
            _ = bb.observables_all()
        t2 = time.perf_counter()
        for r in range(bb.n_replicas):
            _ = (bb.atoms(r, m.ATOM_POSITIONS), bb.atoms(r, m.ATOM_VELOCITIES))
        t3 = time.perf_counter()
        del bb
        t4 = time.perf_counter()
        phases = {"create_s": t1 - t0, "steps_s": t2 - t1, "readback_s": t3 - t2,
                  "destroy_s": t4 - t3}
    # creation (host arrays up), the steps with every step's observables down, and the
    # final readback; the batch's destruction (freeing its device memory, 7-120 ms from one
    # run to the next) is reported in phases but not timed
    t_end = t0 + sum(phases[k] for k in ("create_s", "steps_s", "readback_s")) if phases \
        else time.perf_counter()
    t_e2e = torch.tensor([t_end - t0], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    e2e_value = atoms_all * e2e_steps / float(t_e2e.item())
    # the same session over E2E_LONG steps: creation amortised, the per-step API cost shows
    e2e_long = None
    if not args.no_e2e:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bb = make_batch(m, t, cells, dt=DT, r_skin=SKIN, precision=args.precision,
                        device=local_rank)
        bb.set_launch(tune["tpa_density"], tune["tpa_force"], tune["blocks_density"],
                      tune["blocks_force"])
        t1 = time.perf_counter()
        for s in range(E2E_LONG):
            bb.run(1, REBUILD, 1, False)
            _ = bb.observables_all()
        t2 = time.perf_counter()
        for r in range(bb.n_replicas):
            _ = (bb.atoms(r, m.ATOM_POSITIONS), bb.atoms(r, m.ATOM_VELOCITIES))
        t3 = time.perf_counter()
        del bb
        tl = torch.tensor([t3 - t0], dtype=torch.float64, device="cuda")
        if dist is not None:
            dist.all_reduce(tl, op=dist.ReduceOp.MAX)
        e2e_long = {"value": atoms_all * E2E_LONG / float(tl.item()), "unit": "atom-steps/s",
                    "steps": E2E_LONG,
                    "phases": {"create_s": t1 - t0, "steps_s": t2 - t1, "readback_s": t3 - t2}}
    tb = t.phi.size + t.rho.size + t.F.size
    h2d = args.replicas * N * (6 * 8 + 4) + 3 * 8 * tb
    d2h = e2e_steps * args.replicas * (78 * 8 + 8) + args.replicas * 2 * N * 24

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == WORKLOAD:
        cpu = cpu_sample(N)
    cij = None
    if rank == 0 and not args.no_cij:
        cij = time_to_cij(m, t, cpu)
    cij_nialco = None
    if rank == 0 and not args.no_cij and not args.no_cij_nialco:
        cij_nialco = time_to_cij_nialco(m)
    precision_report = None
    if rank == 0 and not args.no_precision_report and args.workload == WORKLOAD:
        precision_report = mixed_vs_fp64(m, t)
    run_loop = None
    if rank == 0 and not args.no_e2e and args.workload == WORKLOAD:
        run_loop = dropin_run_loop(m, t)
    others = None if args.no_configs else other_configs(m, t, local_rank, peak=peak)
    # per step: k_pre, k_kick_drift, k_sublist, density, force, k_reduce, k_post; per list
    # rebuild: k_cell_bin, k_cell_sort, k_nbr_cells, k_nbr_build, k_sub_invalidate
    n_rebuilds = (args.steps + REBUILD - 1) // REBUILD
    launches = args.steps * 7 + n_rebuilds * 5
    line = {
        "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32 pair math, f64 sums and integrator",
        "data": "synthetic (seeded FCC lattice and Zn placement, Maxwell-Boltzmann velocities)",
        "config": {"workload": args.workload, "atoms_per_replica": N,
                   "replicas_per_gpu": args.replicas, "atoms_per_gpu": N * args.replicas,
                   "potential": "ZnCu.eam.alloy", "ensemble": WORKLOADS[args.workload],
                   "dt_fs": 2,
                   "neighbor_list": f"r_skin {SKIN}, rebuilt every {REBUILD} steps",
                   "sample_observables": "every step", "precision": args.precision,
                   "l2": ("inputs larger than L2 (replica state > 126 MB)"
                          if args.replicas >= 8 else "replica state smaller than L2"),
                   "parallelism": f"replicas only, dp{world}", "fatal_status_clear": status_ok,
                   "launch": tune},
        "plain_fp64_single_cell": plain,
        "time_to_cij": cij,
        "time_to_cij_nialco_108000": cij_nialco,
        "mixed_vs_fp64": precision_report,
        "other_configs": others,
        "roofline": roof,
        "roofline_step": step_roofline(value / world, nbar, peak),
        "cpu_baseline": cpu,
        "e2e": None if args.no_e2e else {
            "value": e2e_value, "unit": "atom-steps/s",
            "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
            "steps": e2e_steps, "api": "md_driver_module.BatchedMDDriver",
            "phases": phases},
        "e2e_long": e2e_long,
        "dropin_run_loop": run_loop,
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def step_roofline(value, nbar, peak, sampled=True):
    """Whole-step HBM roofline: B = 8 nbar + 144 bytes per atom-step (list indices read by
    both pair passes, positions, types, F', velocities, positions written), plus 152 on
    sampled steps (g, h and F''), with nbar the reference's half-list entries per atom."""
    b = 8.0 * nbar + 144.0 + (152.0 if sampled else 0.0)
    achieved = value * b / 1e9
    return {"bound": "hbm", "bytes_per_atom_step": b, "half_list_nbar": nbar,
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak}


def batch_nbar(b):
    """Half-list entries per atom over all replicas of a batch (its current list)."""
    tot = n = 0
    for r in range(b.n_replicas):
        point, _ = b.neighbor_list(r)
        tot += int(point[-1])
        n += len(point) - 1
    return tot / n


def other_configs(m, t, device, steps=50, warmup=5, peak=6650.0):
    """Atom-steps/s of the other batched and single-cell workloads, mixed precision,
    observables every step, list rebuilt every 20 steps, autotuned, CUDA-event timed:
    64 uneven replicas (4 n^3 atoms, n uniform in [4, 20], x_Zn in [0, 0.3], T in [5, 900] K,
    from RandomState(2026)) and the 32,000-atom L1_2 CuZn3 cell at 5 K."""
    from mdelast_b200.systems import l12_cell, make_batch, uneven_replicas
    out = {}
    for name, cells in [("batched_uneven_64", uneven_replicas(t, 64)),
                        ("l12_cuzn3_20x20x20_5K", [l12_cell(t, 20, T=5.0, ensemble=1)])]:
        b = make_batch(m, t, cells, dt=DT, r_skin=SKIN, precision="mixed", device=device)
        b.run(EQUIL_STEPS, REBUILD, 1, False)
        tune = b.autotune_steps(TUNE_STEPS, REBUILD)
        b.run(warmup, REBUILD, 1, False)
        ms = b.run(steps, REBUILD, 1, True)
        value = b.n_atoms * steps / (ms * 1e-3)
        out[name] = {"value": value, "unit": "atom-steps/s",
                     "atoms": b.n_atoms, "replicas": b.n_replicas, "steps": steps,
                     "ms_per_step": ms / steps, "launch": tune,
                     "roofline_step": step_roofline(value, batch_nbar(b), peak)}
        del b
    out[C1_NAME] = c1_config(m, device, peak)
    return out


C1_NAME = "cu01_fcc5_500_nvt300_fp64"


def c1_config(m, device, peak, steps=1000, warmup=20, replicas=64):
    """Configuration C1: pure Cu, the single-element Mishin Cu01 tables (10,000 nodes per
    function), the pure-Cu example's 5x5x5 FCC cell (500 atoms) at the file's lattice
    constant, NVT 300 K, dt 1 fs, FP64, observables every step, list (r_skin 1.2) every 20
    steps. One cell through MDDriver (the configuration as stated), and the same cell in
    64 replicas through BatchedMDDriver; CUDA-event timed, autotuned. The reference core
    runs the same cell on one host core for comparison (200 steps, list included)."""
    from mdelast_b200.potentials import find_potential, read_setfl
    from mdelast_b200.systems import make_batch, make_driver, pure_cell
    path = find_potential("Cu01.eam.alloy.txt")
    if path is None:
        return {"unavailable": "Cu01.eam.alloy.txt not staged"}
    t = read_setfl(path)
    cell = pure_cell(t, 5, T=300.0, ensemble=1, velocity_seed=0)
    d = make_driver(m, t, cell, dt=1e-15, r_skin=SKIN, precision="fp64", device=device)
    d.run(EQUIL_STEPS, REBUILD, 1, False)
    tune = d.autotune_steps(TUNE_STEPS, REBUILD)
    d.run(warmup, REBUILD, 1, False)
    ms = d.run(steps, REBUILD, 1, True)
    point, _ = d.neighbor_list()
    nbar = float(point[-1]) / cell.n_atoms
    value = cell.n_atoms * steps / (ms * 1e-3)
    out = {"value": value, "unit": "atom-steps/s", "atoms": cell.n_atoms, "replicas": 1,
           "steps": steps, "ms_per_step": ms / steps, "precision": "fp64", "dt_fs": 1,
           "potential": "Cu01.eam.alloy.txt", "launch": tune,
           "roofline_step": step_roofline(value, nbar, peak)}
    del d
    cells = [pure_cell(t, 5, T=300.0, ensemble=1, velocity_seed=k) for k in range(replicas)]
    b = make_batch(m, t, cells, dt=1e-15, r_skin=SKIN, precision="fp64", device=device)
    b.run(EQUIL_STEPS, REBUILD, 1, False)
    tune_b = b.autotune_steps(TUNE_STEPS, REBUILD)
    b.run(warmup, REBUILD, 1, False)
    ms_b = b.run(200, REBUILD, 1, True)
    vb = b.n_atoms * 200 / (ms_b * 1e-3)
    out["batched"] = {"value": vb, "unit": "atom-steps/s", "replicas": replicas,
                      "atoms": b.n_atoms, "steps": 200, "ms_per_step": ms_b / 200,
                      "precision": "fp64", "launch": tune_b,
                      "roofline_step": step_roofline(vb, nbar, peak)}
    del b
    from oracle import ref
    if ref.available("ref"):
        ctx = mp.get_context("spawn")
        with ctx.Pool(1) as pool:
            per_step = pool.map(_ref_c1_worker, [200])[0]
        out["reference_cpu_1core"] = {
            "value": cell.n_atoms / per_step, "unit": "atom-steps/s", "cores": 1,
            "kind": "reference", "ms_per_step": per_step * 1e3,
            "sample": "200 steps of the same cell, list rebuilt every 20 steps (included)"}
    return out


def _ref_c1_worker(n_steps):
    """The reference core on the C1 cell: n_steps with the 20-step list cadence."""
    sys.path.insert(0, ROOT)
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    import numpy as np

    from mdelast_b200.potentials import find_potential, read_setfl
    from mdelast_b200.systems import pure_cell, rg_bins
    from oracle.ref import RefDriver
    t = read_setfl(find_potential("Cu01.eam.alloy.txt"))
    c = pure_cell(t, 5, T=300.0, ensemble=1, velocity_seed=0)
    d = RefDriver(t, c.positions, c.velocities, c.types, ensemble=1,
                  thermo=(c.T, c.thermo_q, c.thermo_p_eta, c.Nf),
                  baro=(c.pressure, c.baro_w, c.baro_p_eps),
                  baro_thermo=(c.T, c.baro_q, c.baro_p_eta, 1.0),
                  box=np.diag(c.box), rg=rg_bins(c, 3.615), Nf=c.Nf, dt=1e-15,
                  neighbors=True, r_skin=SKIN)
    t0 = time.perf_counter()
    for k in range(n_steps):
        if k % REBUILD == 0:
            d.calculate_neighbors()
        d.integrate()
    return (time.perf_counter() - t0) / n_steps


WORKLOADS = {WORKLOAD: "NVT 300 K", "l12_cuzn3_20x20x20_32000_nvt5": "NVT 5 K"}


def make_cells(replicas, seed0=0, workload=WORKLOAD):
    """The workload cell in `replicas` copies that differ in their velocity seed: the
    15x15x15 Cu-6 at.% Zn cell (default), or the ordered L1_2 CuZn3 20x20x20 cell at
    5 K."""
    from mdelast_b200.potentials import find_potential, read_setfl
    from mdelast_b200.systems import cuzn_cell, l12_cell
    path = find_potential("ZnCu.eam.alloy")
    if path is None:
        raise SystemExit("ZnCu.eam.alloy not found (make -C oracle potentials)")
    t = read_setfl(path)
    if workload == WORKLOAD:
        cells = [cuzn_cell(t, NSIDE, n_zn=N_ZN, T=T_K, ensemble=1, placement_seed=42,
                           velocity_seed=seed0 + k) for k in range(replicas)]
    else:
        cells = [l12_cell(t, 20, T=5.0, ensemble=1, velocity_seed=500 + seed0 + k)
                 for k in range(replicas)]
    return t, cells


# ----------------------------------------------------------------------------- time to C_ij
CIJ_TOL = 0.02
PLAIN_STAGES = dict(npt_therm=10000, npt_prod=10000, nvt_therm=10000, nvt_prod=90000,
                    sample_stride=1, rebuild_every=REBUILD, checkpoint_every=2500)
WARM_REPLICAS = 4
WARM_LONG_PROD = 20000  # production steps of the long-horizon check of the warm start
WARM_STAGES = dict(npt_therm=0, npt_prod=0, nvt_therm=500, nvt_prod=3000, sample_stride=5,
                   rebuild_every=REBUILD, checkpoint_every=250)


def time_to_cij(m, t, cpu):
    """Wall time to C11/C12/C44 of the workload cell at 300 K.

    plain: the reference's protocol in FP64 on the GPU, one cell: 20k NPT steps (10k
    thermalisation + 10k production for the mean box), handoff into the mean box, 100k NVT
    steps (10k + 90k production, sampled every step); its final C_ij is the target.
    warm start: the trained network proposes the zero-pressure lattice constant; 4 replicas
    of the cell in that box, mixed precision, no NPT stage, 500 NVT thermalisation steps,
    production sampled every 5th step with the running estimate read every 250 steps;
    accepted because the first 500 production steps' mean pressure passes the judge (else
    it would fall back to NPT). Its time counts from loading the network (driver creation,
    autotuning and every readout included) to the first checkpoint from which all three
    constants stay within 2 % of the plain result until the end of its run."""
    from mdelast_b200.protocol import Stages, run_protocol, run_warm_start, time_to_within
    from mdelast_b200.systems import cuzn_cell
    from mdelast_b200.warmstart import WarmStart, judge
    base = dict(n_zn=N_ZN, T=T_K, placement_seed=42)
    plain = run_protocol(m, t, [cuzn_cell(t, NSIDE, ensemble=2, velocity_seed=0, **base)],
                         precision="fp64", stages=Stages(**PLAIN_STAGES), nvt_seeds=[1])
    target = plain.C
    t0 = time.perf_counter()
    ws = WarmStart.load()
    prop = ws.propose(N_ZN / NSIDE**3 / 4, T_K)
    a = float(prop["a"][0])
    cells = [cuzn_cell(t, NSIDE, a_ang=a, ensemble=1, velocity_seed=200 + k, **base)
             for k in range(WARM_REPLICAS)]
    setup = time.perf_counter() - t0
    warm = run_warm_start(m, t, cells, precision="mixed", stages=Stages(**WARM_STAGES),
                          judge=judge, check_steps=500)
    t_warm = time_to_within(warm, target, CIJ_TOL)
    t_warm = None if t_warm is None else setup + t_warm
    t_plain_self = time_to_within(plain, target, CIJ_TOL)
    # the same warm start followed for 20,000 production steps: its time to 2 % then
    # counts only from a checkpoint after which the estimate stays within 2 % for the
    # whole longer run, so an estimate that wanders out later is caught
    t1 = time.perf_counter()
    prop_l = ws.propose(N_ZN / NSIDE**3 / 4, T_K)
    cells_l = [cuzn_cell(t, NSIDE, a_ang=float(prop_l["a"][0]), ensemble=1,
                         velocity_seed=200 + k, **base) for k in range(WARM_REPLICAS)]
    setup_l = time.perf_counter() - t1
    long_stages = dict(WARM_STAGES, nvt_prod=WARM_LONG_PROD)
    warm_l = run_warm_start(m, t, cells_l, precision="mixed", stages=Stages(**long_stages),
                            judge=judge, check_steps=500)
    t_long = time_to_within(warm_l, target, CIJ_TOL)
    devs = [max(abs(c[2 + q] / target[k] - 1.0) for q, k in enumerate(("C11", "C12", "C44")))
            for c in warm_l.checkpoints]
    ablation = ablation_no_network(m, t, target)
    out = {
        "metric": f"wall time to C11/C12/C44 within {CIJ_TOL:.0%} of the FP64 plain result",
        "unit": "s", "cell": WORKLOAD, "tolerance": CIJ_TOL,
        "plain_fp64": {"wall_s": plain.wall_s, "C_GPa": plain.C, "steps": 120000,
                       "replicas": 1, "stages": PLAIN_STAGES,
                       "own_time_to_within_s": t_plain_self,
                       "npt_mean_box_V_V0": plain.V_V0[0]},
        "warm_start_mixed": {"time_to_within_s": t_warm, "wall_s": setup + warm.wall_s,
                             "C_GPa": warm.C,
                             "rel_err_vs_plain": {k: warm.C[k] / target[k] - 1 for k in target},
                             "replicas": WARM_REPLICAS, "stages": WARM_STAGES,
                             "proposal": {k: float(v[0]) for k, v in prop.items()},
                             "accepted": warm.accepted_start,
                             "window_pressure_GPa": warm.npt_pressure_GPa},
        "speedup_vs_plain_protocol": (plain.wall_s / t_warm) if t_warm else None,
        "speedup_vs_plain_time_to_within": (t_plain_self / t_warm)
        if (t_warm and t_plain_self) else None,
        "warm_start_long_horizon": {
            "production_steps": WARM_LONG_PROD,
            "time_to_within_s": None if t_long is None else setup_l + t_long,
            "wall_s": setup_l + warm_l.wall_s,
            "C_GPa": warm_l.C,
            "rel_err_vs_plain": {k: warm_l.C[k] / target[k] - 1 for k in target},
            "largest_deviation_after_3500_steps": max(
                (d for (n, *_), d in zip(warm_l.checkpoints, devs) if n >= 3500), default=None)},
        "ablation_no_network": ablation,
        "network_gain_vs_ablation": (ablation["time_to_within_s"] / t_warm)
        if (t_warm and ablation.get("time_to_within_s")) else None,
    }
    if cpu and cpu.get("value"):
        # the reference core's measured per-step time on this host, times the plain protocol
        ms_step = 1e3 * NSIDE**3 * 4 / cpu["value"]
        est = 120000 * ms_step * 1e-3
        out["reference_cpu_estimated_s"] = est
        out["reference_cpu_basis"] = (f"{ms_step:.1f} ms/step measured for the reference core "
                                      f"(1 core, cpu_baseline) x 120,000 steps; not run")
        if t_warm:
            out["speedup_vs_reference_cpu_estimated"] = est / t_warm
    return out


ABLATION_STAGES = dict(npt_therm=1000, npt_prod=1000, nvt_therm=500, nvt_prod=3000,
                       sample_stride=5, rebuild_every=REBUILD, checkpoint_every=250)


def ablation_no_network(m, t, target):
    """The warm start without its network: the same 4 mixed-precision replicas (same
    seeds, same NVT stages and checkpoints) started at the linear (Vegard) lattice constant
    with a short NPT stage (1,000 + 1,000 steps) to find the box. Its time to within 2 % of
    the plain result, set against the warm start's, is what the network contributes."""
    from mdelast_b200.protocol import Stages, run_protocol, time_to_within
    from mdelast_b200.systems import cuzn_cell, vegard_a
    x = N_ZN / NSIDE**3 / 4
    a = vegard_a(x, T_K)
    cells = [cuzn_cell(t, NSIDE, n_zn=N_ZN, T=T_K, a_ang=a, ensemble=2, placement_seed=42,
                       velocity_seed=200 + k) for k in range(WARM_REPLICAS)]
    res = run_protocol(m, t, cells, precision="mixed", stages=Stages(**ABLATION_STAGES),
                       nvt_seeds=[300 + k for k in range(WARM_REPLICAS)])
    tw = time_to_within(res, target, CIJ_TOL)
    return {"time_to_within_s": tw, "wall_s": res.wall_s, "wall_npt_s": res.wall_npt_s,
            "C_GPa": res.C, "rel_err_vs_plain": {k: res.C[k] / target[k] - 1 for k in target},
            "a_start": a, "npt_mean_V_V0": res.V_V0, "stages": ABLATION_STAGES,
            "replicas": WARM_REPLICAS}


NIALCO_NSIDE = 30  # 108,000 atoms
NIALCO_SEED = 5    # composition: RandomState(5).dirichlet((2, 2, 2))


def time_to_cij_nialco(m):
    """Wall time to C11/C12/C44 of a random Ni-Al-Co FCC 30^3 cell (108,000 atoms) at
    300 K, composition one Dirichlet(2, 2, 2) draw, bundled Mishin 2013 potential.

    plain: the same FP64 protocol as the Cu-Zn comparison, started at the linear (Vegard)
    lattice constant; its final C_ij is the target. warm start: the ternary network
    proposes the lattice constant and the bulk modulus; one cell in the proposed box, mixed
    precision, 500 NVT thermalisation steps, production sampled every 5th step; its first
    500 production steps are the judge's window (0.2 GPa), with at most one box correction
    from the window pressure and the proposed bulk modulus before the plain protocol takes
    over. Times as in time_to_cij."""
    import numpy as np

    from mdelast_b200.potentials import find_potential, read_setfl
    from mdelast_b200.protocol import Stages, run_protocol, run_warm_start, time_to_within
    from mdelast_b200.systems import fcc_alloy_cell
    from mdelast_b200.warmstart import (NIALCO_MODEL, NIALCO_POTENTIAL, WarmStart, judge,
                                        nialco_guess_a)
    t = read_setfl(find_potential(NIALCO_POTENTIAL))
    x = np.random.RandomState(NIALCO_SEED).dirichlet((2.0, 2.0, 2.0))
    a_lin = nialco_guess_a(x, T_K)
    kw = dict(T=T_K, placement_seed=11)
    plain = run_protocol(m, t, [fcc_alloy_cell(t, NIALCO_NSIDE, x, a_ang=a_lin, ensemble=2,
                                               velocity_seed=0, **kw)],
                         precision="fp64", stages=Stages(**PLAIN_STAGES), nvt_seeds=[1])
    target = plain.C
    t0 = time.perf_counter()
    ws = WarmStart.load(NIALCO_MODEL)
    prop = ws.propose(x, T_K)
    cells = [fcc_alloy_cell(t, NIALCO_NSIDE, x, a_ang=float(prop["a"][0]), ensemble=1,
                            velocity_seed=200, **kw)]
    setup = time.perf_counter() - t0
    warm = run_warm_start(m, t, cells, precision="mixed", stages=Stages(**WARM_STAGES),
                          judge=judge, check_steps=500, bulk_GPa=[float(prop["B"][0])])
    t_warm = time_to_within(warm, target, CIJ_TOL)
    t_warm = None if t_warm is None else setup + t_warm
    t_plain_self = time_to_within(plain, target, CIJ_TOL)
    a_npt = a_lin * plain.V_V0[0] ** (1.0 / 3.0)
    return {
        "unit": "s", "cell": f"nialco_fcc{NIALCO_NSIDE}_{4 * NIALCO_NSIDE**3}_npt300",
        "fractions_ni_al_co": x.tolist(), "tolerance": CIJ_TOL,
        "plain_fp64": {"wall_s": plain.wall_s, "C_GPa": plain.C, "steps": 120000,
                       "own_time_to_within_s": t_plain_self, "a_npt": a_npt,
                       "a_linear_guess": a_lin},
        "warm_start_mixed": {"time_to_within_s": t_warm, "wall_s": setup + warm.wall_s,
                             "C_GPa": warm.C,
                             "rel_err_vs_plain": {k: warm.C[k] / target[k] - 1 for k in target},
                             "proposal": {k: float(v[0]) for k, v in prop.items()},
                             "a_rel_err_vs_npt": float(prop["a"][0]) / a_npt - 1,
                             "accepted": warm.accepted_start, "corrections": warm.corrections,
                             "window_pressure_GPa": warm.npt_pressure_GPa},
        "speedup_vs_plain_protocol": (plain.wall_s / t_warm) if t_warm else None,
        "speedup_vs_plain_time_to_within": (t_plain_self / t_warm)
        if (t_warm and t_plain_self) else None,
    }


A_EQ_300K = 3.66683  # [A] FP64 NPT production mean of the 13,500-atom cell at 300 K


def mixed_vs_fp64(m, t, window=200, replicas=4, therm=2000, prod=20000):
    """Error of the mixed-precision path against the FP64 path on the timed workload cell.

    same_seed_window: one cell (velocity seed 0) run in both precisions from the same
    state for `window` steps, observables sampled every step; per quantity the largest
    deviation of the mixed run from the FP64 run over the first 10, 50 and `window` steps
    (relative for energies and temperatures, in GPa for pressure and stresses, which pass
    through zero). Trajectories that differ by rounding diverge exponentially, so the
    short windows measure the arithmetic and the long one the start of the divergence.

    cij: `replicas` cells at the FP64 NPT mean lattice constant of this cell at 300 K
    (A_EQ_300K), velocity seeds 100.., run in both precisions (NVT 300 K,
    `therm` steps, then C11/C12/C44 by the fluctuation formula over `prod` steps sampled
    every step). Reported: each precision's mean over replicas with its standard error, and
    the paired difference mixed - FP64 with its standard error (the trajectories decorrelate
    long before the end of production, so the pairs are independent samples)."""
    import numpy as np

    from mdelast_b200.systems import cuzn_cell, make_batch, make_driver
    from mdelast_b200.units import Units as U
    cell = cuzn_cell(t, NSIDE, n_zn=N_ZN, T=T_K, ensemble=1, placement_seed=42, velocity_seed=0)
    recs = {}
    for prec in ("fp64", "mixed"):
        d = make_driver(m, t, cell, dt=DT, r_skin=SKIN, precision=prec)
        d.run(window, REBUILD, 1, False)
        recs[prec] = d.drain_samples()
        del d
    a, b = recs["mixed"], recs["fp64"]
    eV = U.ev
    quantities = {
        "epot_atom": ("rel", a["epot_atom"], b["epot_atom"]),
        "etot_cons": ("rel", a["etot_cons"], b["etot_cons"]),
        "temperature_kin": ("rel", a["temperature_kin"], b["temperature_kin"]),
        "temperature_conf": ("rel", 1.0 / a["temperature_conf_inverse"],
                             1.0 / b["temperature_conf_inverse"]),
        "pressure_GPa": ("abs", a["pressure"] / U.GPa, b["pressure"] / U.GPa),
        "born_stress_GPa": ("abs", a["born_stress_tensor"] / U.GPa,
                            b["born_stress_tensor"] / U.GPa),
        "born_elasticity_GPa": ("abs", a["born_elasticity_tensor"] / U.GPa,
                                b["born_elasticity_tensor"] / U.GPa),
    }
    win = {}
    for name, (kind, x, y) in quantities.items():
        x, y = np.asarray(x), np.asarray(y)
        dev = np.abs(x - y)
        if kind == "rel":
            dev = dev / np.abs(y)
        dev = dev.reshape(len(dev), -1).max(axis=1)
        win[name] = {f"max_first_{n}": float(dev[:n].max()) for n in (10, 50, window)}
        win[name]["kind"] = "relative" if kind == "rel" else "absolute"
    win["epot_atom_eV_first_step"] = [float(a["epot_atom"][0] / eV), float(b["epot_atom"][0] / eV)]

    cells = [cuzn_cell(t, NSIDE, n_zn=N_ZN, T=T_K, a_ang=A_EQ_300K, ensemble=1,
                       placement_seed=42, velocity_seed=100 + k) for k in range(replicas)]
    C = {}
    wall = {}
    for prec in ("fp64", "mixed"):
        t0 = time.perf_counter()
        bt = make_batch(m, t, cells, dt=DT, r_skin=SKIN, precision=prec)
        bt.autotune(2)
        bt.set_sample_ring(0)
        bt.run(therm, REBUILD, 1, False)
        bt.fluctuation_start()
        bt.run(prod, REBUILD, 1, False)
        C[prec] = np.array([[bt.elastic_constants(r)[k] / U.GPa for k in ("C11", "C12", "C44")]
                            for r in range(replicas)])
        wall[prec] = time.perf_counter() - t0
        del bt
    diff = C["mixed"] - C["fp64"]
    se = lambda x: (x.std(axis=0, ddof=1) / np.sqrt(len(x))).tolist()  # noqa: E731
    names = ("C11", "C12", "C44")
    cij = {"replicas": replicas, "thermalisation_steps": therm, "production_steps": prod,
           "sample_every": 1, "unit": "GPa", "wall_s": wall}
    for prec in ("fp64", "mixed"):
        cij[prec] = {k: {"mean": float(C[prec][:, i].mean()), "se": float(se(C[prec])[i])}
                     for i, k in enumerate(names)}
    cij["mixed_minus_fp64"] = {k: {"mean": float(diff[:, i].mean()), "se": float(se(diff)[i]),
                                   "rel": float(diff[:, i].mean() / C["fp64"][:, i].mean())}
                               for i, k in enumerate(names)}
    return {"cell": WORKLOAD, "same_seed_window": win, "window_steps": window, "cij": cij}


def run_loop_calls(d, steps, rebuild=REBUILD):
    """The calls MolecularDynamics.run() makes on its driver per step, in its order
    (molecular_dynamics.py:1240-1285, observables sampled every step): the cycle checks,
    the list rebuild every `rebuild` steps, sample_observables, integrate(), then the reads
    of append_sample (molecular_dynamics.py:1218-1238)."""
    import numpy as np
    for _ in range(steps):
        c = d.cycle
        if c % rebuild == 0:
            d.calculate_neighbors()
        d.sample_observables = True
        d.integrate()
        _ = (d.time, d.temperature_kin, d.temperature_conf_inverse, d.total_laplacian,
             d.total_force2, d.pressure, np.copy(d.stress_tensor), d.etot_atom, d.epot_atom,
             d.epot_eam_atom, d.ekin_atom, d.etot_cons, d.etot_cons_err,
             np.copy(d.born_stress_tensor), np.copy(d.born_elasticity_tensor),
             d.box.volume() / d.box_initial.volume(), d.cycle)


def dropin_run_loop(m, t, steps=200, warmup=20):
    """Atom-steps/s of the workload cell driven the way the reference's run loop drives
    its driver (run_loop_calls): one MDDriver, one integrate() per step and 17 attribute
    reads after it, wall-clock time; FP64 and mixed precision."""
    from mdelast_b200.systems import cuzn_cell, make_driver
    cell = cuzn_cell(t, NSIDE, n_zn=N_ZN, T=T_K, ensemble=1, placement_seed=42, velocity_seed=0)
    out = {"api": "md_driver_module.MDDriver, the calls of molecular_dynamics.py:1240-1285",
           "atoms": cell.n_atoms, "steps": steps, "unit": "atom-steps/s"}
    for prec in ("fp64", "mixed"):
        d = make_driver(m, t, cell, dt=DT, r_skin=SKIN, precision=prec)
        d.autotune(2)
        run_loop_calls(d, warmup)
        d.synchronize()
        t0 = time.perf_counter()
        run_loop_calls(d, steps)
        wall = time.perf_counter() - t0
        out[prec] = {"value": cell.n_atoms * steps / wall, "ms_per_step": 1e3 * wall / steps}
        del d
    return out


def half_list_nbar(m, t, cell):
    """Half-list entries per atom of the reference's list at this cell (point[N]/N)."""
    from mdelast_b200.systems import make_driver
    d = make_driver(m, t, cell, dt=DT, r_skin=SKIN)
    point, _ = d.neighbor_list()
    return float(point[-1]) / cell.n_atoms


# ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_force_mx launch, keyed by
# (precision, replicas, staged tables): single-pass captures of the bench command at 16
# replicas without cache flushing (the launches of timed-region steps, so the L2 holds
# what the preceding kernels of the step left in it), mean over the captured launches;
# profiles/launches_bench_mixed_16x13500.md has the capture. None where not captured.
TRAFFIC_PER_LAUNCH: dict = {("mixed", 16, False): 82.38e6 + 1.11e6,
                            ("mixed", 16, True): 78.89e6 + 0.77e6}


# ----------------------------------------------------------------------------- reference
def _ref_worker(args):
    """One host process: the reference's C++ core on the workload cell, n_warm untimed
    steps then one list build and n_steps timed steps; returns s/step (list amortised)."""
    n_steps, n_warm = args
    sys.path.insert(0, ROOT)
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)  # the reference prints from C++
    import numpy as np

    from mdelast_b200.systems import rg_bins
    from oracle.ref import RefDriver
    t, cells = make_cells(1)
    c = cells[0]
    d = RefDriver(t, c.positions, c.velocities, c.types, ensemble=1,
                  thermo=(c.T, c.thermo_q, c.thermo_p_eta, c.Nf),
                  baro=(c.pressure, c.baro_w, c.baro_p_eps),
                  baro_thermo=(c.T, c.baro_q, c.baro_p_eta, 1.0),
                  box=np.diag(c.box), rg=rg_bins(c), Nf=c.Nf, dt=DT, neighbors=True, r_skin=SKIN)
    if n_warm > 0:
        d.integrate(n_warm)
    t0 = time.perf_counter()
    d.calculate_neighbors()
    t_list = time.perf_counter() - t0
    t0 = time.perf_counter()
    d.integrate(n_steps)
    t_steps = (time.perf_counter() - t0) / n_steps
    return t_steps + t_list / REBUILD


def cpu_sample(N, n_steps=8):
    """The reference's C++ core (oracle/_ref) on one core: list build + n steps."""
    from oracle import ref
    if not ref.available("ref"):
        return None
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        per_step = pool.map(_ref_worker, [(n_steps, 0)])[0]
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
    # a bounded sample per process: at most 10 timed steps after at most 10 warm-up steps
    n_steps = max(1, min(args.steps, 10))
    n_warm = max(0, min(args.warmup, 10))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        per_step = pool.map(_ref_worker, [(n_steps, n_warm)] * cores)
    wall = time.perf_counter() - t0
    N = NSIDE**3 * 4
    value = sum(N / x for x in per_step)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atom-steps/s",
        "n_gpus": 0, "steps": n_steps, "warmup": n_warm,
        "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": statistics.mean(per_step) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "atoms_per_replica": N, "replicas": cores,
                   "parallelism": f"{cores} independent single-thread processes"},
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": cores,
                         "kind": "reference",
                         "sample": f"per process: {n_warm} warm-up steps, then one O(N^2) list "
                                   f"build + {n_steps} timed steps of the {N}-atom cell (list "
                                   f"amortised over {REBUILD}); wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--replicas", type=int, default=16)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="mixed")
    ap.add_argument("--launch", default=None, metavar="TPA_D,TPA_F,BLOCKS_D,BLOCKS_F",
                    help="launch shapes of the density and force passes instead of the "
                         "autotuner's (lanes per atom, target block count)")
    ap.add_argument("--force-tables", choices=("auto", "l1", "shared"), default="auto",
                    help="with --launch: the force pass reads its tables through the L1 or "
                         "from the staged shared-memory copy (default: as the driver has it)")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default=WORKLOAD,
                    help="the timed batch's cell (the C_ij comparisons always use the "
                         "Cu-Zn cell)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other workloads (64 uneven replicas, L1_2 32k cell)")
    ap.add_argument("--no-cij", action="store_true",
                    help="skip the time-to-C_ij comparison (plain FP64 protocol vs warm start)")
    ap.add_argument("--no-cij-nialco", action="store_true",
                    help="skip the C_ij timing of the 108,000-atom Ni-Al-Co cell (plain FP64 "
                         "protocol vs the ternary warm start; about 3 minutes)")
    ap.add_argument("--no-precision-report", action="store_true",
                    help="skip the mixed-vs-FP64 error report (about 30 s)")
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
