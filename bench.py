#!/usr/bin/env python3
"""Benchmark of the batched GFN2-xTB energy + gradient (one JSON line on rank 0).

Workload: the mixed batch of 4096 molecules (half water clusters (H2O)n, n ~ U{5..100}, lattice
rule; half alkanes CkH2k+2, k ~ U{5..60}, dihedrals 70 % anti / 30 % gauche), per-molecule SCC
convergence at 1e-7 Eh (accuracy 0.1), FP64. A step is one energy + gradient pass over the whole
batch. Multi-GPU (torchrun): the job is nmol molecules per rank, split over the ranks in
size-balanced bins (axtb_b200.sharding; weak scaling) with no collective on the data path; the
time is the maximum over ranks, and the e2e leg all-gathers every molecule's results.

* value: molecules/s with positions resident in HBM (axtb_gpu_batch_run_device), CUDA events on
  the engine's stream, L2 flushed (256 MB write) between timed steps;
* e2e: the same through the public API with host arrays (Batch.run: pinned host->device copy of
  the positions and device->host read of energies, gradients and moments inside the timed step);
* roofline: the dominant kernel's live CUDA-event time against its algorithmic FLOPs (or bytes);
* cpu_baseline: the C++ oracle (CPU restatement of axtb's algorithm, not axtb itself) on an
  interleaved sample of 256 molecules of the same batch, one molecule per host core, from a
  process pool made before the timing.

``--impl reference`` times that CPU restatement alone on the host cores (the reference is Rust
and cannot be built in this image), rank 0 only: W short warm-up steps, then K steps of 256
molecules each (a different interleaved sample per step).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "GFN2 E+grad mol/s batched; s/point at 3000 atoms; vs FP64 plain at |dE|<1e-6 Eh"
WORKLOAD = ("mixed batch of 4096: half (H2O)n n~U{5..100} (3.1 A lattice, 0.2 A jitter), half CkH2k+2 "
            "k~U{5..60} (70/30 anti/gauche); SCC at 1e-7 Eh; FP64")


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------------------ CPU baseline
def _oracle_init():
    from oracle import oracle as O

    O.enable_lapack()
    O.lib()


def _oracle_one(args):
    z, x, acc = args
    from oracle import oracle as O

    r = O.singlepoint(z, x, accuracy=acc, lapack=True, lapack_threads=1)
    return r["energy"]


CPU_SAMPLE = 256  # molecules per CPU step: every (nmol / 256)-th molecule of the batch


def interleaved(mols, size, offset):
    """A fixed sample of `size` molecules spread evenly over the batch (stride nmol / size from
    `offset`, every other pick one further on): the batch alternates water clusters and alkanes,
    so an even stride alone would sample one kind only; this keeps both kinds and their sizes."""
    n = len(mols)
    stride = max(1, n // size)
    idx = [(offset + k * stride + (k & 1)) % n for k in range(min(size, n))]
    return [mols[i] for i in idx]


class CpuPool:
    """The oracle (C++ restatement of axtb, not axtb itself; OpenBLAS eigensolver) on every host
    core: a spawned process pool made once, outside any timed interval, one molecule per
    process at a time (axtb's own throughput mode)."""

    def __init__(self, cores=None):
        import multiprocessing as mp

        from oracle import oracle as O

        O.build()
        self.cores = cores or os.cpu_count() or 1
        self.pool = mp.get_context("spawn").Pool(self.cores, initializer=_oracle_init)
        self.pool.map(_oracle_one, [(np.array([1, 1], dtype=np.int32), np.array([[0, 0, 0], [0, 0, 1.4]]), 1.0)]
                      * self.cores)

    def time(self, sample, acc):
        t0 = time.perf_counter()
        self.pool.map(_oracle_one, [(z, x, acc) for z, x in sample], chunksize=1)
        return time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_rate(mols, acc, pool, steps, warmup):
    """Oracle throughput (mol/s) on the host cores: `warmup` untimed steps of 32 molecules, then
    `steps` timed steps of 256, each an interleaved sample of the batch from its own offset (the
    same procedure for the reference arm and for the baseline beside the GPU line); returns the
    rate, the molecules timed and the seconds."""
    done, total = 0, 0.0
    for step in range(warmup + steps):
        sample = interleaved(mols, 32 if step < warmup else CPU_SAMPLE, step)
        dt = pool.time(sample, acc)
        if step >= warmup:
            done += len(sample)
            total += dt
    return done / total, done, total


def cpu_baseline(mols, acc, pool):
    """Oracle throughput (mol/s) on the host cores: one warm-up step and one timed step."""
    v, done, dt = cpu_rate(mols, acc, pool, steps=1, warmup=1)
    return {"value": v, "unit": "mol/s", "cores": pool.cores, "kind": "port",
            "sample": f"{done} molecules, an interleaved sample of the same batch (half of each kind; "
                      f"{dt:.1f} s on {pool.cores} processes made and warmed up before timing; C++ restatement "
                      f"of axtb with OpenBLAS eigensolver, not axtb itself)"}


def cpu_point(z, x, acc, threads):
    """Seconds per single point of one large molecule through the oracle with `threads` LAPACK
    threads (the reference runs single large points multi-threaded, capped at 8 threads)."""
    from oracle import oracle as O

    O.enable_lapack()
    t0 = time.perf_counter()
    r = O.singlepoint(z, x, accuracy=acc, lapack=True, lapack_threads=threads)
    return time.perf_counter() - t0, r


# ------------------------------------------------------------------------------ GPU helpers
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"axtb_clocks_{os.getpid()}.csv"

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def fp64_peak_tflops(dev):
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


# ------------------------------------------------------------------------------ main
def large_point(device):
    """s/point of (H2O)1000 (3000 atoms, 6000 AOs; 10x10x10 lattice rule, seed 0) through the
    public API (host positions in, energy and gradient out), FP64 and split precision, after one
    warm-up point each; the split run's |dE| and max |dG| against the FP64 one."""
    import torch

    from axtb_b200 import Batch, structures

    z, x = structures.water_cluster(1000, seed=0, dims=(10, 10, 10))
    res = {}
    for prec in ("fp64", "split"):
        b = Batch([(z, x)], accuracy=1.0, precision=prec, device=device)
        b.run([x], gradient=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = b.run([x], gradient=True)[0]
        torch.cuda.synchronize()
        res[prec] = (r, time.perf_counter() - t0)
        b.close()
    (r64, t64), (rsp, tsp) = res["fp64"], res["split"]
    out = {"system": "(H2O)1000: 3000 atoms, 6000 AOs (10x10x10 lattice rule, seed 0), accuracy 1",
           "s_per_point": t64, "iterations": r64.iterations, "status": r64.status, "energy": r64.energy,
           "split": {"s_per_point": tsp, "iterations": rsp.iterations, "abs_dE": abs(rsp.energy - r64.energy),
                     "max_abs_dG": float(np.abs(rsp.gradient - r64.gradient).max()),
                     "speedup_vs_fp64": t64 / tsp}}
    # the other large single points of the workload set, FP64
    for name, (z, x) in large_molecules().items():
        if name == "(H2O)1000":
            continue
        b = Batch([(z, x)], accuracy=1.0, device=device)
        b.run([x], gradient=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = b.run([x], gradient=True)[0]
        torch.cuda.synchronize()
        out[name] = {"s_per_point": time.perf_counter() - t0, "atoms": len(z), "iterations": r.iterations,
                     "status": r.status, "energy": r.energy}
        b.close()
    return out


def large_molecules():
    from axtb_b200 import structures

    return {"(H2O)500": structures.water_cluster(500, seed=0, dims=(10, 10, 5)),
            "C200H402": structures.alkane(200, seed=0, gauche=0.1),
            "(H2O)1000": structures.water_cluster(1000, seed=0, dims=(10, 10, 10))}


def cpu_points(names):
    """s/point of the oracle (C++ restatement of axtb, OpenBLAS LAPACK eigensolver) on large
    single points, accuracy 1, with every host core and with 8 threads (the reference's cap for
    one calculation, crates/driver/src/lib.rs:164-169)."""
    mols = large_molecules()
    cores = os.cpu_count() or 1
    out = {}
    for name in names:
        z, x = mols[name]
        row = {"atoms": len(z)}
        for label, th in (("all_cores", cores), ("8_threads", 8)):
            dt, r = cpu_point(z, x, 1.0, th)
            row[label] = {"s_per_point": dt, "threads": th, "energy": r["energy"]}
        out[name] = row
    out["kind"] = "port: C++ restatement of axtb with OpenBLAS eigensolver, not axtb itself"
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nmol", type=int, default=4096)
    ap.add_argument("--accuracy", type=float, default=0.1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-large", action="store_true", help="skip the large single points")
    ap.add_argument("--cpu-large", action="store_true", help="also time the CPU restatement on (H2O)500 (minutes)")
    ap.add_argument("--band-max-nao", type=int, default=None,
                    help="schedule: two-stage tridiagonal reduction below this many AOs (default: the engine's)")
    args = ap.parse_args()
    rank, world, local = rank_info()

    from axtb_b200 import structures

    if args.impl == "reference":
        if rank != 0:
            return
        mols = structures.mixed_batch(args.nmol, seed=0)
        pool = CpuPool()
        v, done, total = cpu_rate(mols, args.accuracy, pool, args.steps, args.warmup)
        pool.close()
        per = done // max(1, args.steps)
        cb = {"value": v, "unit": "mol/s", "cores": pool.cores, "kind": "port",
              "sample": f"{args.steps} steps of {per} molecules (interleaved samples of the batch, half of each "
                        f"kind, from a per-step offset), {total:.1f} s on {pool.cores} processes made and warmed up "
                        f"before timing; C++ restatement of axtb with OpenBLAS eigensolver, not axtb itself"}
        out = {"metric": METRIC, "value": v, "unit": "mol/s", "n_gpus": args.gpus, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": args.nmol / v * 1e3, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
               "config": {"workload": WORKLOAD, "nmol": args.nmol, "accuracy": args.accuracy,
                          "sample_per_step": per,
                          "ms_per_step": "the whole batch at the sampled rate"},
               "cpu_baseline": cb, "e2e": {"value": v, "unit": "mol/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out), flush=True)
        return

    import torch

    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    from axtb_b200.sharding import ShardedBatch

    t0 = time.time()
    # the whole job: nmol molecules per rank, split over the ranks in size-balanced bins (weak
    # scaling); each rank times its own bin and the e2e leg gathers every result on every rank
    allmols = structures.mixed_batch(args.nmol * world, seed=0)
    log(f"[rank {rank}] built {len(allmols)} molecules in {time.time() - t0:.1f} s")
    t0 = time.time()
    sched = {} if args.band_max_nao is None else {"band_max_nao": args.band_max_nao}
    sharded = ShardedBatch(allmols, accuracy=args.accuracy, device=local, **sched)
    batch = sharded.local
    mols = [allmols[i] for i in sharded.mine]
    log(f"[rank {rank}] engine set-up {time.time() - t0:.1f} s ({len(mols)} molecules)")
    natT = int(batch.natoms.sum())
    pos = torch.tensor(np.concatenate([x.reshape(-1) for _, x in mols]), dtype=torch.float64, device=dev)
    energy = torch.zeros(len(mols), dtype=torch.float64, device=dev)
    grad = torch.zeros(natT * 3, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(batch.stream, device=dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    def step():
        st = batch.run_device(pos.data_ptr(), energy.data_ptr(), grad.data_ptr(), gradient=True)
        return st

    for w in range(args.warmup):
        t0 = time.time()
        st = step()
        torch.cuda.synchronize()
        log(f"[rank {rank}] warmup {w}: {time.time() - t0:.2f} s, failed molecules {int((st != 0).sum())}")
    peaks = measured_peaks()
    fp64 = fp64_peak_tflops(dev)
    batch.set_profiling(True)
    barrier()
    total = 0.0
    launches = 0
    with Clocks(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
            st = step()
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1) / 1e3
            launches += batch.launches
    barrier()
    prof = batch.profile()
    batch.set_profiling(False)
    t = torch.tensor([total], dtype=torch.float64, device=dev)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tmax = float(t.item())
    value = args.nmol * world * args.steps / tmax
    fails = int((st != 0).sum())

    # e2e through the public API with host arrays
    e2e = None
    if not args.no_e2e:
        hostpos = [x for _, x in allmols]
        sharded.run(hostpos, gradient=True)  # warm-up of the API path
        batch.set_profiling(True)
        tt = 0.0
        nst = max(1, min(args.steps, 2))
        for k in range(nst):
            flush.fill_(float(k))
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
            sharded.run(hostpos, gradient=True)
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize()
            tt += e0.elapsed_time(e1) / 1e3
        p2 = batch.profile()
        batch.set_profiling(False)
        te = torch.tensor([tt], dtype=torch.float64, device=dev)
        if world > 1:
            import torch.distributed as dist

            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": args.nmol * world * nst / float(te.item()), "unit": "mol/s",
               "h2d_bytes_per_step": p2["h2d_bytes"] // nst, "d2h_bytes_per_step": p2["d2h_bytes"] // nst}

    if rank == 0:
        kern = prof["kernels"]
        top = max(kern.items(), key=lambda kv: kv[1]["ms"])
        name, kd = top
        tot_ms = sum(v["ms"] for v in kern.values())
        if kd["flops"] > 0:
            ach = kd["flops"] / (kd["ms"] / 1e3) / 1e12
            roof = {"kernel": name, "bound": "tensor", "achieved": ach, "peak": fp64, "unit": "TFLOP/s",
                    "frac": ach / fp64, "traffic": None, "share": kd["ms"] / tot_ms,
                    "note": "FP64 dense algebra; achieved = algorithmic FLOPs n^3 (reduction to standard form) + "
                            "4/3 n^3 (tridiagonalisation) + 4 n^2 k (back-transform, L^-T, density) per molecule "
                            "and eigen phase / CUDA-event time of the phase (k_team, then k_chase and k_team again "
                            "when the bulge chasing of the two-stage reduction runs on chip); peak = torch "
                            "float64 8192^3 GEMM measured on this GPU in this run (the pool's measured peaks hold "
                            "HBM and bf16 only); traffic: ncu DRAM bytes are not measured inside the bench run"}
        else:
            ach = kd["bytes"] / (kd["ms"] / 1e3) / 1e9
            roof = {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": ach / peaks["hbm_gbs"], "traffic": None, "share": kd["ms"] / tot_ms}
        # the HBM-bound matrix passes: algorithmic bytes / CUDA-event time against measured HBM
        hbm = {}
        for kname in ("fock", "mulliken", "integrals"):
            v = kern.get(kname)
            if v and v["bytes"] > 0 and v["ms"] > 0:
                gbs = v["bytes"] / (v["ms"] / 1e3) / 1e9
                hbm[kname] = {"achieved_gbs": gbs, "frac": gbs / peaks["hbm_gbs"], "share": v["ms"] / tot_ms}
        # whole-step roofline: sum over kernels of max(FLOPs / FP64 peak, bytes / HBM), against the
        # measured step (kernels without an algorithmic count contribute no roofline time)
        t_roof = sum(max(v["flops"] / (fp64 * 1e12), v["bytes"] / (peaks["hbm_gbs"] * 1e9)) for v in kern.values())
        step_roof = {"t_roof_ms": t_roof * 1e3 / args.steps, "t_step_ms": tmax / args.steps * 1e3,
                     "frac": t_roof / tmax}
        large = None
        if not args.no_large and world == 1:
            large = large_point(local)
        cb = None
        cpu_large = None
        if not args.no_cpu:
            pool = CpuPool()
            cb = cpu_baseline(allmols, args.accuracy, pool)
            pool.close()
            if world == 1:
                cpu_large = cpu_points(["C200H402"] + (["(H2O)500"] if args.cpu_large else []))
        out = {"metric": METRIC, "value": value, "unit": "mol/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": tmax / args.steps * 1e3, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": WORKLOAD, "nmol": args.nmol, "atoms": natT, "accuracy": args.accuracy,
                          "l2": "flushed between timed steps (256 MB write)", "parallelism": f"molecule-sharded x{world}",
                          "failed_molecules": fails, **sched},
               "e2e": e2e, "gpu_launches": launches, "roofline": roof, "hbm_kernels": hbm,
               "step_roofline": step_roof,
               "large_point": large, "cpu_baseline": cb, "cpu_large_point": cpu_large,
               "clocks": clk.summary(), "kernel_ms": {k: round(v["ms"], 3) for k, v in kern.items()}}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
