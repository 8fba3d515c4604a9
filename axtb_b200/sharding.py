"""Molecule sharding across GPUs (one process per GPU, torch.distributed for the plumbing).

The batched single points are independent molecules, so the path shards without any exchange
in the compute: every rank takes a size-balanced bin of molecules (longest-processing-time
order on the dense-algebra cost (n_AO + 32)^3, the cost model the engine's team plan uses within
a GPU), runs them in one Batch on its own GPU, and the per-molecule results are gathered
afterwards (an all-gather of small result arrays; energies are nmol doubles, gradients 3 natoms).
With the NCCL backend the gathered arrays live on the rank's current CUDA device (NCCL moves
device memory only); with gloo they stay in host memory.
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


def _device(group):
    """Where collective payloads must live for the group's backend."""
    import torch
    import torch.distributed as dist

    if str(dist.get_backend(group)).lower() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather(local: np.ndarray, indices, nmol: int, group=None) -> np.ndarray:
    """All-gather per-molecule rows (local[k] belongs to molecule indices[k]) into a (nmol, ...)
    array in the original molecule order, on every rank."""
    import torch
    import torch.distributed as dist

    dev = _device(group)
    local = np.asarray(local, dtype=np.float64)
    row = local.shape[1:] if local.ndim > 1 else ()
    width = 1 + int(np.prod(row)) if row else 2
    payload = np.zeros((len(indices), width))
    if len(indices):
        payload[:, 0] = np.asarray(indices, dtype=np.float64)
        payload[:, 1:] = local.reshape(len(indices), -1)
    world = dist.get_world_size(group)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([payload.shape[0]], dtype=torch.int64, device=dev), group=group)
    counts = [int(s.item()) for s in sizes]
    nmax = max(max(counts), 1)
    padded = torch.zeros((nmax, width), dtype=torch.float64, device=dev)
    if payload.shape[0]:
        padded[: payload.shape[0]] = torch.from_numpy(payload).to(dev)
    parts = [torch.zeros((nmax, width), dtype=torch.float64, device=dev) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    out = np.zeros((nmol,) + tuple(row))
    for p, c in zip(parts, counts):
        for rec in p[:c].cpu().numpy():
            out[int(rec[0])] = rec[1:].reshape(row) if row else rec[1]
    return out


def _default_batch(molecules, **options):
    from .calculator import Batch

    return Batch(molecules, **options)


class ShardedBatch:
    """A list of molecules split over the ranks of `group`: each rank builds one engine Batch of
    its bin once (on its current GPU) and every ``run`` gathers the results of all molecules on
    every rank. ``batch_factory(molecules, **options)`` makes the per-rank batch (default: the
    engine's ``Batch``); anything with ``run(positions, gradient)`` returning results with
    ``energy``, ``status`` and ``gradient`` serves."""

    def __init__(self, molecules, group=None, batch_factory=None, **options):
        import torch.distributed as dist

        self.group = group
        self.nmol = len(molecules)
        self.natoms = np.array([len(m[0]) for m in molecules])
        distributed = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if distributed else 0
        self.world = dist.get_world_size(group) if distributed else 1
        self.bins = shard_indices([molecule_cost(m[0]) for m in molecules], self.world)
        self.mine = self.bins[self.rank]
        factory = batch_factory or _default_batch
        self.local = factory([molecules[i] for i in self.mine], **options) if self.mine else None

    def run(self, positions=None, gradient: bool = True):
        """(energies (nmol,), statuses (nmol,), gradients: list of (nat, 3) arrays or None) on
        every rank; `positions` is None (the set-up geometries) or one (nat, 3) array per
        molecule of the whole list."""
        mypos = None if positions is None else [positions[i] for i in self.mine]
        res = self.local.run(mypos, gradient=gradient) if self.local is not None else []
        if self.world == 1:
            energy = np.array([r.energy for r in res])
            status = np.array([r.status for r in res], dtype=int)
            grads = [np.asarray(r.gradient).reshape(-1, 3) for r in res] if gradient else None
            return energy, status, grads
        energy = gather(np.array([r.energy for r in res]), self.mine, self.nmol, self.group)
        status = gather(np.array([r.status for r in res], dtype=np.float64), self.mine, self.nmol,
                        self.group).astype(int)
        grads = None
        if gradient:
            width = 3 * int(self.natoms.max())
            loc = np.zeros((len(self.mine), width))
            for k, r in enumerate(res):
                g = np.asarray(r.gradient).reshape(-1)
                loc[k, : g.size] = g
            full = gather(loc, self.mine, self.nmol, self.group)
            grads = [full[i, : 3 * self.natoms[i]].reshape(-1, 3) for i in range(self.nmol)]
        return energy, status, grads

    def close(self):
        if self.local is not None and hasattr(self.local, "close"):
            self.local.close()


def run_sharded(molecules, gradient: bool = True, group=None, batch_factory=None, **options):
    """Every rank runs its bin of `molecules` on its current GPU; returns (energies (nmol,),
    statuses (nmol,), gradients: list of (nat, 3) arrays or None) on every rank."""
    sb = ShardedBatch(molecules, group=group, batch_factory=batch_factory, **options)
    try:
        return sb.run(gradient=gradient)
    finally:
        sb.close()
