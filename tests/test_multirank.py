"""Replicas across ranks (CPU, gloo, world size 2): the shards cover every replica once,
each rank advances its own replicas (the oracle stands in for a GPU here), and the gathered
per-replica results equal a single-process run."""

import os
import socket

import numpy as np
import pytest

from mdelast_b200.sharding import shard_replicas


def test_shards_cover_and_balance():
    sizes = [256, 500, 864, 2048, 4000, 256, 108, 32000]
    for world in (1, 2, 3, 4):
        sh = shard_replicas(sizes, world)
        flat = sorted(k for s in sh for k in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[k] for k in s) for s in sh]
        assert max(loads) - min(loads) <= max(sizes)
    assert shard_replicas(sizes, 2) == shard_replicas(sizes, 2)


def _cells():
    from helpers import tables
    from mdelast_b200.systems import cuzn_cell
    t = tables()
    return t, [cuzn_cell(t, n, x_zn=x, T=T, velocity_seed=k)
               for k, (n, x, T) in enumerate([(3, 0.1, 300.0), (4, 0.05, 600.0),
                                               (3, 0.2, 100.0)])]


def _advance(t, cell, steps=3):
    from mdelast_b200.systems import rg_bins
    from oracle.ref import OracleDriver
    d = OracleDriver(t, cell.positions, cell.velocities, cell.types, ensemble=cell.ensemble,
                     thermo=(cell.T, cell.thermo_q, cell.thermo_p_eta, cell.Nf),
                     baro=(cell.pressure, cell.baro_w, cell.baro_p_eps),
                     baro_thermo=(cell.T, cell.baro_q, cell.baro_p_eta, 1.0),
                     box=np.diag(cell.box), rg=rg_bins(cell), Nf=cell.Nf, dt=2e-15)
    d.integrate(steps)
    s = d.scalar_dict()
    return {"etot_cons": s["etot_cons"], "pressure": s["pressure"]}


def _rank_main(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [here, os.path.dirname(here)]
    import torch.distributed as dist
    from datetime import timedelta
    from mdelast_b200.sharding import gather_observables
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    t, cells = _cells()
    mine = shard_replicas([c.n_atoms for c in cells], world)[rank]
    local = {k: _advance(t, cells[k]) for k in mine}
    allres = gather_observables(local)
    if rank == 0:
        q.put(allres)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gather_every_replica():
    import multiprocessing as mp
    from oracle import ref
    if not ref.available("oracle"):
        pytest.skip("oracle not built")
    t, cells = _cells()
    serial = {k: _advance(t, c) for k, c in enumerate(cells)}
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(got) == sorted(serial)
    for k in serial:
        assert got[k]["etot_cons"] == serial[k]["etot_cons"]
        assert got[k]["pressure"] == serial[k]["pressure"]
