"""Sharding of independent systems across ranks: the partition, and the world-size-2 gather over gloo on CPU
(the evaluator here is the oracle; on GPUs every rank runs its systems through the engine's batched launch)."""

import os
import socket

import numpy as np
import pytest

from conftest import PKG, ROOT, oracle_settings, oracle_topology


def shard():
    import pgm_md_b200.shard as sh
    return sh


def test_partition_balanced_and_complete():
    rng = np.random.default_rng(0)
    counts = rng.integers(24, 1537, size=1024)
    for world in (1, 2, 3, 8):
        parts = shard().partition(counts, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(1024))
        loads = [int(counts[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= counts.max()
        assert parts == shard().partition(counts, world)   # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    from oracle import pgm_oracle as O
    import pgm_md_b200.shard as sh
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    systems = pkg.systems.water_batch(nsys=6, seed=9, nmin=8, nmax=24, tol=1e-8)
    parts = sh.partition([s.n for s in systems], world)
    mine = parts[rank]
    rows = []
    for k in mine:
        S = systems[k]
        e = O.Engine(O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength),
                     O.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-8, max_iter=500, peek=0.0,
                                predictor=0, ke=pkg.systems.KE_DEFAULT))
        E = e.compute(S.pos, S.box, want_forces=False)
        rows.append([E, e.iterations])
    allE = sh.gather_energies(mine, np.array(rows).reshape(len(mine), 2), len(systems))
    if rank == 0:
        q.put(allE.tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_gather_world_size_2_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    allE = np.array(q.get(timeout=300))
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    from oracle import pgm_oracle as O
    systems = PKG.systems.water_batch(nsys=6, seed=9, nmin=8, nmax=24, tol=1e-8)
    for k, S in enumerate(systems):
        e = O.Engine(oracle_topology(S), oracle_settings(S, tol=1e-8)).compute(S.pos, S.box, want_forces=False)
        assert abs(allE[k, 0] - e) <= 1e-12 * abs(e)
