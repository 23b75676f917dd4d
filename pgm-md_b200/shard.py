"""Sharding of independent systems across ranks (one process per GPU).

A batch of independent periodic systems needs no exchange during an evaluation: every rank evaluates its own
systems in one batched launch, and the per-system results are gathered once at the end.  Systems go to ranks
by atom count, largest first, each to the rank with the fewest atoms so far (longest-processing-time
scheduling), so every rank computes the same partition without communication.
"""

from __future__ import annotations

import numpy as np


def partition(atom_counts, world):
    """Lists of system indices per rank (balanced by atoms, deterministic)."""
    counts = np.asarray(atom_counts, dtype=np.int64)
    order = sorted(range(len(counts)), key=lambda k: (-int(counts[k]), k))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += int(counts[k])
    return [sorted(p) for p in parts]


def gather_energies(local_index, local_energies, nsys, group=None):
    """All-gathers per-system energy rows (any width) from every rank into an (nsys, width) array ordered by
    system index.  Uses torch.distributed (NCCL on GPUs, gloo on CPU) when it is initialised."""
    import torch
    import torch.distributed as dist

    local_energies = np.asarray(local_energies, dtype=np.float64).reshape(len(local_index), -1)
    width = local_energies.shape[1]
    if not (dist.is_available() and dist.is_initialized()):
        out = np.zeros((nsys, width))
        out[np.asarray(local_index, dtype=np.int64)] = local_energies
        return out
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    world = dist.get_world_size(group)
    # fixed-size exchange: every rank sends nsys rows (its own rows filled, a mask column marks them)
    buf = torch.zeros((nsys, width + 1), dtype=torch.float64, device=dev)
    idx = torch.as_tensor(np.asarray(local_index, dtype=np.int64), device=dev)
    if len(local_index):
        buf[idx, :width] = torch.as_tensor(local_energies, device=dev)
        buf[idx, width] = 1.0
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = torch.zeros((nsys, width), dtype=torch.float64, device=dev)
    for p in parts:
        mask = p[:, width] > 0
        out[mask] = p[mask, :width]
    return out.cpu().numpy()
