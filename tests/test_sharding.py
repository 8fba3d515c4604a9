"""Molecule sharding across ranks (CPU: gloo, world size 2; no GPU, no engine call).

Checks the size-balanced partition (every molecule exactly once, balanced cost) and the result
gather back into molecule order, run as two gloo processes on 127.0.0.1."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from axtb_b200.sharding import shard_indices


def test_partition_covers_every_molecule_once_and_balances():
    rng = np.random.default_rng(0)
    costs = (rng.integers(30, 600, 4096).astype(float) + 32.0) ** 3
    for world in (1, 2, 3, 8):
        bins = shard_indices(costs, world)
        flat = sorted(i for b in bins for i in b)
        assert flat == list(range(len(costs)))
        loads = np.array([costs[b].sum() for b in bins])
        assert loads.max() <= loads.mean() + costs.max()  # LPT bound
    assert shard_indices([5.0, 1.0], 4)[2:] == [[], []]


def test_partition_is_deterministic():
    costs = [3.0, 3.0, 2.0, 7.0, 1.0, 1.0]
    assert shard_indices(costs, 2) == shard_indices(list(costs), 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from axtb_b200.sharding import gather, shard_indices

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nmol = 37
        costs = [float((i * 7919) % 101 + 1) for i in range(nmol)]
        mine = shard_indices(costs, world)[rank]
        # stand-in per-molecule results: energy = -index, gradient row = index * (1, 2, 3)
        e = gather(np.array([-float(i) for i in mine]), mine, nmol)
        g = gather(np.array([[i, 2 * i, 3 * i] for i in mine], dtype=float), mine, nmol)
        out[rank] = (e.tolist(), g.tolist())
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_gather_two_gloo_ranks():
    ctx = tmp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs)
    for r in range(2):
        e, g = out[r]
        assert e == [-float(i) for i in range(37)]
        assert g == [[i, 2 * i, 3 * i] for i in range(37)]


class _OracleBatch:
    """CPU stand-in for the engine's Batch in the sharding test: the oracle's single points."""

    def __init__(self, molecules, **options):
        self.mols = molecules
        self.options = options

    def run(self, positions=None, gradient=True):
        from types import SimpleNamespace

        from oracle import oracle as O

        out = []
        for k, (z, x) in enumerate(self.mols):
            xx = x if positions is None else positions[k]
            r = O.singlepoint(z, xx, accuracy=self.options.get("accuracy", 1.0), gradient=gradient)
            out.append(SimpleNamespace(energy=r["energy"], status=0, gradient=r["gradient"]))
        return out


def _small_molecules():
    from axtb_b200 import structures as S

    return [S.water_cluster(n, seed=n) for n in (2, 3, 4)] + [S.alkane(k, seed=k) for k in (2, 3, 5)]


def _sharded_worker(rank, world, port, out):
    import torch.distributed as dist

    from axtb_b200.sharding import ShardedBatch

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mols = _small_molecules()
        sb = ShardedBatch(mols, batch_factory=_OracleBatch, accuracy=1e-6)
        e, st, g = sb.run(gradient=True)
        # a second run on displaced geometries through the same per-rank batches
        moved = [x + 0.01 for _, x in mols]
        e2, _, g2 = sb.run(moved, gradient=True)
        out[rank] = (sb.mine, e.tolist(), st.tolist(), [a.tolist() for a in g], e2.tolist(),
                     [a.tolist() for a in g2])
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_run_sharded_two_gloo_ranks_matches_single_process():
    """The sharded run (LPT bins, one batch per rank, results all-gathered in molecule order)
    gives every rank what one process computes alone, with the oracle as the per-rank engine."""
    from oracle import oracle as O

    O.build()
    ctx = tmp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
    assert all(p.exitcode == 0 for p in procs)
    mols = _small_molecules()
    ref = [O.singlepoint(z, x, accuracy=1e-6) for z, x in mols]
    ref2 = [O.singlepoint(z, x + 0.01, accuracy=1e-6) for z, x in mols]
    assert sorted(out[0][0] + out[1][0]) == list(range(len(mols)))
    for r in range(2):
        _, e, st, g, e2, g2 = out[r]
        assert st == [0] * len(mols)
        assert e == [x["energy"] for x in ref]
        assert all(np.array_equal(np.array(a), x["gradient"]) for a, x in zip(g, ref))
        assert e2 == [x["energy"] for x in ref2]
        assert all(np.array_equal(np.array(a), x["gradient"]) for a, x in zip(g2, ref2))
