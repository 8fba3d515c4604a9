"""Molecule sharding across GPUs (one process per GPU, torch.distributed for the plumbing).

The batched single points are independent molecules, so the path shards without any exchange
in the compute: every rank takes a size-balanced bin of molecules (longest-processing-time
order on the dense-algebra cost (n_AO + 32)^3, the cost model the engine's team plan uses within
a GPU), runs them in one Batch on its own GPU, and the per-molecule results are gathered
afterwards (an all-gather of small result arrays; energies are nmol doubles, gradients 3 natoms).
"""
from __future__ import annotations

import heapq

import numpy as np


def molecule_cost(numbers) -> float:
    from .calculator import basis_size

    return (float(basis_size(numbers)[1]) + 32.0) ** 3


def shard_indices(costs, world: int) -> list[list[int]]:
    """Deterministic LPT partition of molecule indices into `world` bins (each bin sorted)."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    bins: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        bins[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(b) for b in bins]


def gather(local: np.ndarray, indices, nmol: int, group=None) -> np.ndarray:
    """All-gather per-molecule rows (local[k] belongs to molecule indices[k]) into a (nmol, ...)
    array in the original molecule order, on every rank."""
    import torch
    import torch.distributed as dist

    local = np.asarray(local, dtype=np.float64)
    row = local.shape[1:] if local.ndim > 1 else ()
    payload = torch.as_tensor(np.concatenate([np.asarray(indices, dtype=np.float64)[:, None],
                                              local.reshape(len(indices), -1)], axis=1))
    world = dist.get_world_size(group)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([payload.shape[0]], dtype=torch.int64), group=group)
    width = payload.shape[1]
    nmax = int(max(s.item() for s in sizes))
    padded = torch.zeros((nmax, width), dtype=torch.float64)
    padded[: payload.shape[0]] = payload
    parts = [torch.zeros((nmax, width), dtype=torch.float64) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    out = np.zeros((nmol,) + tuple(row))
    for p, s in zip(parts, sizes):
        p = p[: int(s.item())].numpy()
        for rec in p:
            out[int(rec[0])] = rec[1:].reshape(row) if row else rec[1]
    return out


def run_sharded(molecules, gradient: bool = True, group=None, **options):
    """Every rank runs its bin of `molecules` on its current GPU; returns (energies (nmol,),
    statuses (nmol,), gradients: list of (nat, 3) arrays or None) on every rank."""
    import torch.distributed as dist

    from .calculator import Batch

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    bins = shard_indices([molecule_cost(m[0]) for m in molecules], world)
    mine = bins[rank]
    res = Batch([molecules[i] for i in mine], **options).run(gradient=gradient) if mine else []
    nmol = len(molecules)
    energy = gather(np.array([r.energy for r in res]), mine, nmol, group)
    status = gather(np.array([r.status for r in res], dtype=np.float64), mine, nmol, group).astype(int)
    grads = None
    if gradient:
        nat = np.array([len(m[0]) for m in molecules])
        width = 3 * int(nat.max())
        loc = np.zeros((len(mine), width))
        for k, r in enumerate(res):
            loc[k, : r.gradient.size] = r.gradient.reshape(-1)
        full = gather(loc, mine, nmol, group)
        grads = [full[i, : 3 * nat[i]].reshape(-1, 3) for i in range(nmol)]
    return energy, status, grads
