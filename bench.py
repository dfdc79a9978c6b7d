#!/usr/bin/env python
"""Throughput benchmark of the exhaustive third-order K2 epistasis search on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: "plain-large" -- 4096 SNPs x 16384 samples (8192 cases / 8192 controls),
seeded Hardy-Weinberg genotypes with one planted triplet (synthetic: the reference
benchmarks on no public dataset).  Metric: triplet*samples/s, one unit = one SNP
triplet scored over one sample.

A step scans one shard of the triplet space: the first SNP index i is cut into
`--shards` contiguous ranges of equal work (C(M-1-i, 2) triplets per i); step t of
rank r scans shard (t*N + r) mod shards, so K = shards steps on one GPU cover every
triplet once.  Per-GPU work is fixed as N grows ("weak" scaling; the only exchange
of a sharded search is the final argmin, which is outside the timed steps).

Our arm ("value") runs with the dataset resident in HBM; "e2e" repeats the steps
through the public one-call entry point (epik2_scan_u8) from pinned host buffers, so
each step includes the host->device upload, GPU encoding and the result read-back.
The reference arm (--impl reference) times the reference's own OpenMP CPU search
(v4_popc_avx512, built from the reference sources by oracle/Makefile) on the host
cores, each step a bounded sample of the same matrix (its first M' SNPs, all samples).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cross-dpc-episdet_b200"))

METRIC = "triplet*samples/s"
UNIT = "triplet*samples/s"


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def shard_bounds(m, parts):
    """Cut first indices [0, m) into `parts` contiguous ranges of near-equal triplet count."""
    work = [((m - 1 - i) * (m - 2 - i)) // 2 for i in range(m)]
    total = sum(work)
    bounds, acc, lo = [], 0, 0
    for i in range(m):
        acc += work[i]
        if len(bounds) < parts - 1 and acc >= total * (len(bounds) + 1) / parts:
            bounds.append((lo, i + 1))
            lo = i + 1
    bounds.append((lo, m))
    while len(bounds) < parts:
        bounds.append((m, m))
    return bounds


def triplets_in(m, lo, hi):
    return sum(((m - 1 - i) * (m - 2 - i)) // 2 for i in range(lo, hi))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, pci_bus=None):
        self.bus = pci_bus  # PCI bus number of the benchmarked GPU (int), or None
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        def bus_of(r):
            try:
                return int(r[1].split(":")[1], 16)
            except (IndexError, ValueError):
                return None
        if len({r[1] for r in rows}) > 1 and self.bus is not None:
            rows = [r for r in rows if bus_of(r) == self.bus] or rows
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        under_load = [x for x in sm if x > 600] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[6 + q].lower() == "active"})
        pw = [float(r[4]) for r in rows if r[4].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(under_load) if under_load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows),
                "power_w_max": max(pw) if pw else None}


def cpu_reference_step(g, p, m_sub, threads=None):
    """One bounded run of the reference's CPU search on the first m_sub SNPs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    binary = oracle.best_ref_binary()
    if binary is None:
        return None
    sub = np.ascontiguousarray(g[:, :m_sub])
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "geno.bin")
        oracle.write_geno_file(path, sub, p)
        r = oracle.run_ref_file(binary, path, sub.shape[0], m_sub, 64, 16, threads=threads, timeout=600)
    ts = m_sub * (m_sub - 1) * (m_sub - 2) // 6 * sub.shape[0]
    return {"value": ts / r["wall_search_s"], "wall_s": r["wall_search_s"], "threads": r["threads"],
            "binary": binary, "ijk": r["ijk"], "triplet_samples": ts}


def cpu_sample_snps():
    """SNP count of one bounded CPU step: ~5-15 s of reference work on this host."""
    cores = os.cpu_count() or 1
    rate = 1.2e10 * cores  # triplet*samples/s per core of the reference's AVX-512 search (measured on a 8-core host)
    for m_sub in (1024, 768, 640, 512):
        if m_sub * (m_sub - 1) * (m_sub - 2) / 6 * 16384 / rate <= 12.0:
            return m_sub
    return 384


def run_reference(args, rank, world):
    from epik2 import workloads as W
    import epik2
    if rank != 0:
        return 0
    cfg = W.PLAIN_LARGE
    g, p = W.generate(cfg)
    m_sub = cpu_sample_snps()
    for _ in range(args.warmup):
        r = cpu_reference_step(g, p, min(m_sub, 256))
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU harness not built"}))
            return 0
    walls, ts_total, thr = [], 0, None
    for _ in range(args.steps):
        r = cpu_reference_step(g, p, m_sub)
        walls.append(r["wall_s"])
        ts_total += r["triplet_samples"]
        thr = r["threads"]
    value = ts_total / sum(walls)
    sample = (f"{cfg['name']}: first {m_sub} SNPs x {cfg['n_samples']} samples per step "
              f"({r['binary']} search, C({m_sub},3) triplets)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(walls) / len(walls),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Hardy-Weinberg, planted triplet)",
            "config": {"workload": cfg["name"], "form": "plain", "sample_snps": m_sub, "step": "bounded CPU sample",
                       "parallelism": "OpenMP host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import epik2
    from epik2 import workloads as W

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    cfg = W.CONFIGS[args.workload]
    g, p = W.generate(cfg)
    S, M = g.shape
    ctx = epik2.Context(local_rank)
    ext = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local_rank))
    did = ctx.load(g, p)
    info = ctx.info(did)
    words = (info["n_samples"] - info["n_cases"] + 31) // 32 + (info["n_cases"] + 31) // 32
    parts = max(args.shards, world)
    shards = shard_bounds(M, parts)
    peaks = epik2.probe_int_peaks(local_rank)
    flush = torch.empty(args.flush_mb << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")

    def shard_of(t):
        return shards[(t * world + rank) % parts]

    def step(t):
        lo, hi = shard_of(t)
        with torch.cuda.stream(ext):
            flush.zero_()
        return ctx.scan(did, snp_begin=lo, snp_end=hi)

    for t in range(args.warmup):
        step(t)
    torch.cuda.synchronize()
    barrier()
    pci = None
    try:
        pci = torch.cuda.get_device_properties(local_rank).pci_bus_id
    except Exception:
        pass
    sampler = ClockSampler(pci) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.reset_stats()
    ev0.record(ext)
    kernel_ms, step_trip, bests = [], [], []
    for t in range(args.warmup, args.warmup + args.steps):
        b = step(t)
        st = ctx.stats()
        kernel_ms.append(st["last_scan_kernel_ms"])
        step_trip.append(st["last_scan_triplets"])
        bests.append((b.score, b.ijk))
    ev1.record(ext)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop() if sampler else None
    launches = ctx.stats()["kernel_launches"]
    elapsed_ms = ev0.elapsed_time(ev1)
    ts_local = sum(step_trip) * S
    popc_local = sum(step_trip) * words * 8
    stats_t = torch.tensor([elapsed_ms, ts_local, popc_local, sum(kernel_ms)], dtype=torch.float64,
                           device=f"cuda:{local_rank}")
    if dist is not None:
        mx = stats_t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = stats_t.clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        elapsed_max, ts_total = float(mx[0]), float(sm[1])
    else:
        elapsed_max, ts_total = elapsed_ms, ts_local
    value = ts_total / (elapsed_max / 1e3)

    # roofline of the search kernel: algorithmic popcounts (8 per triplet per 32-sample
    # class word) over the kernel's own event-timed duration, against the measured POPC rate
    achieved_popc = popc_local / (sum(kernel_ms) / 1e3)
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))["k_scan_int"]
        if tr["workload"] == cfg["name"]:
            traffic = tr["dram_bytes_per_triplet"] * sum(step_trip) / len(step_trip)
    except (OSError, KeyError, ValueError):
        pass
    ref_form_popc = sum(step_trip) * words * 27 / (sum(kernel_ms) / 1e3)

    # end to end through the one-call entry point, pinned host buffers
    e2e = None
    if not args.no_e2e:
        gh = torch.empty(g.shape, dtype=torch.uint8, pin_memory=True)
        ph = torch.empty(p.shape, dtype=torch.uint8, pin_memory=True)
        gh.numpy()[...] = g
        ph.numpy()[...] = p
        gn, pn = gh.numpy(), ph.numpy()
        ctx.unload(did)
        torch.cuda.synchronize()
        barrier()
        ctx.reset_stats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        e_trip = 0
        for t in range(args.warmup, args.warmup + args.steps):
            lo, hi = shard_of(t)
            b = ctx.scan_u8(gn, pn, snp_begin=lo, snp_end=hi)
            e_trip += ctx.stats()["last_scan_triplets"]
        e1.record(ext)
        torch.cuda.synchronize()
        barrier()
        st = ctx.stats()
        e_ms = e0.elapsed_time(e1)
        et = torch.tensor([e_ms, e_trip * S], dtype=torch.float64, device=f"cuda:{local_rank}")
        if dist is not None:
            a = et.clone()
            dist.all_reduce(a, op=dist.ReduceOp.MAX)
            c = et.clone()
            dist.all_reduce(c, op=dist.ReduceOp.SUM)
            e_ms, e_ts = float(a[0]), float(c[1])
        else:
            e_ts = e_trip * S
        e2e = {"value": e_ts / (e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": st["h2d_bytes"] // args.steps,
               "d2h_bytes_per_step": st["d2h_bytes"] // args.steps, "gpu_launches": st["kernel_launches"],
               "entry_point": "epik2_scan_u8"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        m_sub = cpu_sample_snps()
        r = cpu_reference_step(g, p, m_sub)
        if r is not None:
            cpu = {"value": r["value"], "unit": UNIT, "cores": r["threads"], "kind": "reference",
                   "sample": f"first {m_sub} SNPs x {S} samples of the same matrix, {r['binary']} "
                             f"(reference OpenMP search), {r['wall_s']:.2f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Hardy-Weinberg genotypes, planted triplet (17,203,411) at effect 0.8)",
            "config": {"workload": cfg["name"], "form": "plain", "n_snps": M, "n_samples": S,
                       "n_cases": info["n_cases"], "step": f"1/{parts} of the triplet space (first-index shard)",
                       "l2": f"flushed before every step ({args.flush_mb} MiB write)",
                       "parallelism": f"{world} GPU(s), shard-parallel", "engine": "integer (LOP3+POPC)"},
            "roofline": {"bound": "popc", "achieved": achieved_popc / 1e9, "peak": peaks["popc_per_s"] / 1e9,
                         "unit": "Gpopc/s", "frac": achieved_popc / peaks["popc_per_s"], "traffic": traffic,
                         "traffic_source": "ncu dram bytes per triplet (profiles/traffic.json) x triplets per launch",
                         "peak_source": "measured live by epik2_probe_int_peaks on this GPU",
                         "algorithmic_popc_per_triplet_word": 8,
                         "reference_form_frac": ref_form_popc / peaks["popc_per_s"],
                         "kernel_ms_per_step": sum(kernel_ms) / len(kernel_ms)},
            "clocks": clocks,
            "gpu_launches": launches,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "scan_latency_ms": {"p50": float(np.percentile(kernel_ms, 50)), "p99": float(np.percentile(kernel_ms, 99)),
                                "what": "device time of one step's search kernel"},
            "best_in_last_step": {"score": bests[-1][0], "ijk": list(bests[-1][1])},
        }
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain-large", choices=["plain-large", "plain-small", "precision"])
    ap.add_argument("--shards", type=int, default=8)
    ap.add_argument("--flush-mb", type=int, default=256)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank, world, local_rank = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
