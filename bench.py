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
triplet once.  Per-GPU work is fixed as N grows ("weak" scaling).  The one exchange of
a sharded search, the argmin over ranks (two MIN all-reduces of one int64), closes every
step when N > 1.

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


def _oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def cpu_reference_step(g, p, m_sub, threads=None, block=(64, 16)):
    """One bounded run of the reference's CPU search on the first m_sub SNPs."""
    import numpy as np
    oracle = _oracle_module()
    binary = oracle.best_ref_binary()
    if binary is None:
        return None
    sub = np.ascontiguousarray(g[:, :m_sub])
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "geno.bin")
        oracle.write_geno_file(path, sub, p)
        r = oracle.run_ref_file(binary, path, sub.shape[0], m_sub, block[0], block[1], threads=threads, timeout=600)
    ts = m_sub * (m_sub - 1) * (m_sub - 2) // 6 * sub.shape[0]
    return {"value": ts / r["wall_search_s"], "wall_s": r["wall_search_s"], "threads": r["threads"],
            "binary": binary, "ijk": r["ijk"], "triplet_samples": ts, "block": list(block), "m_sub": m_sub}


# block_pac x block_snp of the reference's blocked search (CPU/v4_popc_avx512.cpp:4600-4601)
CPU_BLOCKS = [(32, 16), (32, 32), (64, 16), (64, 32), (128, 16), (128, 32)]


def cpu_baseline_protocol(g, p, threads=None):
    """The reference's CPU search timed by a bounded protocol: sweep the six block shapes on
    the first 512 SNPs, then time the best shape on the first 512, 768 and 1024 SNPs to check
    that triplet*samples/s is flat in the subset size (the rate the full search would have).
    Returns None when no reference binary is built."""
    sweep = []
    for blk in CPU_BLOCKS:
        r = cpu_reference_step(g, p, 512, threads, blk)
        if r is None:
            return None
        sweep.append(r)
    best = max(sweep, key=lambda r: r["value"])
    flat = [best] + [cpu_reference_step(g, p, m, threads, tuple(best["block"])) for m in (768, 1024)]
    rates = [r["value"] for r in flat]
    return {"best": max(flat, key=lambda r: r["value"]), "block": best["block"],
            "block_sweep_m512": {f"{r['block'][0]}/{r['block'][1]}": r["value"] for r in sweep},
            "flatness": {str(r["m_sub"]): r["value"] for r in flat},
            "flatness_spread": (max(rates) - min(rates)) / max(rates), "threads": best["threads"],
            "binary": best["binary"], "rate": max(rates),
            "wall_s": sum(r["wall_s"] for r in sweep + flat[1:])}


def reference_matrix(cfg):
    """The workload's matrix from the oracle's restatement of the seeded generator (no product
    library is loaded by the reference arm), checked against the recorded digest."""
    import hashlib
    import numpy as np
    oracle = _oracle_module()
    g, p = oracle.gen_hwe(cfg["seed"], cfg["n_samples"], cfg["n_snps"], cfg["n_cases"], cfg["maf"], cfg["planted"],
                          cfg["effects"])
    try:
        rec = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_best.json")))
        for v in rec.values():
            if v["seed"] == cfg["seed"] and v["n_snps"] == cfg["n_snps"] and v["n_samples"] == cfg["n_samples"]:
                assert hashlib.sha256(np.ascontiguousarray(g).tobytes()).hexdigest() == v["geno_sha256"]
                break
    except OSError:
        pass
    return g, p


def run_reference(args, rank, world):
    sys.path.insert(0, os.path.join(ROOT, "cross-dpc-episdet_b200", "epik2"))
    import workloads as W  # the workload table only; the product library is not loaded
    if rank != 0:
        return 0
    cfg = W.PLAIN_LARGE
    g, p = reference_matrix(cfg)
    proto = cpu_baseline_protocol(g, p)  # block sweep + flatness check; also warms the host
    if proto is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU harness not built"}))
        return 0
    # each step: the first m_sub SNPs (the rate is flat in the subset size, see "flatness"),
    # sized to about 3 s of host work so that --steps K ends within minutes
    m_sub = 512
    for m in (640, 768, 1024):
        if m * (m - 1) * (m - 2) / 6 * cfg["n_samples"] / proto["rate"] <= 3.0:
            m_sub = m
    for _ in range(max(0, args.warmup - 1)):
        cpu_reference_step(g, p, 256, block=tuple(proto["block"]))
    walls, ts_total, thr = [], 0, None
    for _ in range(args.steps):
        r = cpu_reference_step(g, p, m_sub, block=tuple(proto["block"]))
        walls.append(r["wall_s"])
        ts_total += r["triplet_samples"]
        thr = r["threads"]
    value = ts_total / sum(walls)
    sample = (f"{cfg['name']}: first {m_sub} SNPs x {cfg['n_samples']} samples per step "
              f"({r['binary']} search, C({m_sub},3) triplets, block {proto['block'][0]}/{proto['block'][1]}, "
              f"the best of the 6-shape sweep)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(walls) / len(walls),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Hardy-Weinberg, planted triplet)",
            "config": {"workload": cfg["name"], "form": "plain", "sample_snps": m_sub, "step": "bounded CPU sample",
                       "parallelism": "OpenMP host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "reference", "sample": sample,
                             "block_sweep_m512": proto["block_sweep_m512"], "flatness": proto["flatness"],
                             "flatness_spread": proto["flatness_spread"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import epik2
    from epik2 import sharding as SH
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
    shards = SH.shard_bounds(M, parts)
    peaks = epik2.probe_int_peaks(local_rank)
    tune = ctx.autotune(did)  # AUTO-engine scans below use this choice
    if args.engine != "auto":  # a pinned engine (profiling runs): report it as the choice
        ctx.set_engine({"int": epik2.ENGINE_INT, "tc": epik2.ENGINE_TC, "fp4": epik2.ENGINE_TC_FP4}[args.engine])
        tune = dict(tune, engine={"int": epik2.ENGINE_INT, "tc": epik2.ENGINE_TC, "fp4": epik2.ENGINE_TC_FP4}[args.engine])
    if args.stage_words:
        ctx.set_stage_words(args.stage_words)
        tune = dict(tune, stage_words=args.stage_words)
    if args.pair_tile:
        ctx.set_pair_tile(args.pair_tile)
        tune = dict(tune, pair_tile=args.pair_tile)
    if args.overlap:
        ctx.set_overlap(args.overlap)
        tune = dict(tune, overlap=1 if args.overlap == 2 else 0)
    engine_tc = tune["engine"] in (epik2.ENGINE_TC, epik2.ENGINE_TC_FP4)
    engine_fp4 = tune["engine"] == epik2.ENGINE_TC_FP4
    flush = torch.empty(args.flush_mb << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")

    def shard_of(t):
        return shards[(t * world + rank) % parts]

    def exchange(b):
        # the one exchange step of the sharded search: lowest (score, index) over ranks
        if dist is None:
            return b.score, b.ijk
        return SH.exchange_best(b.score, b.ijk)

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
        bests.append(exchange(b))
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

    # roofline of the search kernel over its own event-timed duration.  Tensor-core engine:
    # algorithmic int8 ops = 2 x 8 multiply-accumulates (the 8 counted cells) per triplet
    # per sample, against the measured dense int8 tcgen05 rate.  Integer engine: 8 POPC per
    # triplet per 32-sample class word, against the measured POPC rate.
    kernel_s = sum(kernel_ms) / 1e3
    achieved_popc = popc_local / kernel_s
    ref_form_popc = sum(step_trip) * words * 27 / kernel_s
    kernel_name = ("k_scan_pipe" if tune.get("overlap") else "k_scan_tc") if engine_tc else "k_scan_int"
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))[kernel_name]
        if tr["workload"] == cfg["name"]:
            traffic = tr["dram_bytes_per_triplet"] * sum(step_trip) / len(step_trip)
    except (OSError, KeyError, ValueError):
        pass
    peak_key = "tc_fp4_mac_per_s" if engine_fp4 else "tc_i8_mac_per_s"
    if engine_tc and peak_key in peaks:
        # 8 counted cells per triplet and sample = 8 multiply-accumulates = 16 operations
        ops = 16.0 * ts_local / kernel_s
        roof = {"bound": "tensor", "achieved": ops / 1e12, "peak": 2 * peaks[peak_key] / 1e12,
                "unit": "TOPS (fp4)" if engine_fp4 else "TOPS (int8)", "frac": ops / (2 * peaks[peak_key]),
                "peak_source": ("measured live by epik2_probe_tc_fp4 on this GPU (dense tcgen05 kind::mxf4, "
                                "M128 N224 K64)" if engine_fp4 else
                                "measured live by epik2_probe_tc_i8 on this GPU (dense tcgen05 kind::i8)"),
                "algorithmic_ops_per_triplet_sample": 16}
    else:
        roof = {"bound": "popc", "achieved": achieved_popc / 1e9, "peak": peaks["popc_per_s"] / 1e9,
                "unit": "Gpopc/s", "frac": achieved_popc / peaks["popc_per_s"],
                "peak_source": "measured live by epik2_probe_int_peaks on this GPU",
                "algorithmic_popc_per_triplet_word": 8}
    roof.update({"traffic": traffic, "traffic_source": "ncu dram bytes per triplet (profiles/traffic.json) x triplets "
                 "per launch", "kernel": kernel_name, "kernel_ms_per_step": sum(kernel_ms) / len(kernel_ms),
                 "popc_equivalent_frac": achieved_popc / peaks["popc_per_s"],
                 "reference_form_popc_frac": ref_form_popc / peaks["popc_per_s"]})

    # end to end through the one-call entry point, pinned host buffers
    e2e = None
    if not args.no_e2e:
        gh = torch.empty(g.shape, dtype=torch.uint8, pin_memory=True)
        ph = torch.empty(p.shape, dtype=torch.uint8, pin_memory=True)
        gh.numpy()[...] = g
        ph.numpy()[...] = p
        gn, pn = gh.numpy(), ph.numpy()
        ctx.unload(did)
        for t in range(args.warmup):  # untimed, like the device-resident leg
            lo, hi = shard_of(t)
            exchange(ctx.scan_u8(gn, pn, snp_begin=lo, snp_end=hi))
        torch.cuda.synchronize()
        barrier()
        ctx.reset_stats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        e_trip = 0
        parts_ms = {"load_wall": 0.0, "upload_device": 0.0, "encode_margins_device": 0.0, "scan_wall": 0.0,
                    "search_kernel_device": 0.0}
        for t in range(args.warmup, args.warmup + args.steps):
            lo, hi = shard_of(t)
            b = ctx.scan_u8(gn, pn, snp_begin=lo, snp_end=hi)
            st1 = ctx.stats()
            e_trip += st1["last_scan_triplets"]
            parts_ms["load_wall"] += st1["last_load_ms"]
            parts_ms["upload_device"] += st1["last_upload_ms"]
            parts_ms["encode_margins_device"] += st1["last_prepare_ms"]
            parts_ms["scan_wall"] += st1["last_scan_wall_ms"]
            parts_ms["search_kernel_device"] += st1["last_scan_kernel_ms"]
            exchange(b)
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
        breakdown = {k: v / args.steps for k, v in parts_ms.items()}
        breakdown["step"] = e_ms / args.steps
        breakdown["other"] = breakdown["step"] - breakdown["load_wall"] - breakdown["scan_wall"]
        e2e = {"value": e_ts / (e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": st["h2d_bytes"] // args.steps,
               "d2h_bytes_per_step": st["d2h_bytes"] // args.steps, "gpu_launches": st["kernel_launches"],
               "entry_point": "epik2_scan_u8", "breakdown_ms_per_step": breakdown,
               "what": "load_wall = upload + encode + pair margins (host wall); scan_wall = tile list, search, "
                       "reduction, read-back (host wall); other = the rest of the call (unload) and the loop"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        proto = cpu_baseline_protocol(g, p)
        if proto is not None:
            b = proto["best"]
            cpu = {"value": proto["rate"], "unit": UNIT, "cores": proto["threads"], "kind": "reference",
                   "sample": (f"first M' SNPs x {S} samples of the same matrix, {proto['binary']} (reference "
                              f"OpenMP search): block_pac/block_snp swept over {len(CPU_BLOCKS)} shapes at M'=512, "
                              f"best {proto['block'][0]}/{proto['block'][1]} timed at M' = 512, 768, 1024; value = "
                              f"the highest rate ({b['m_sub']} SNPs), {proto['wall_s']:.1f} s of CPU runs"),
                   "block_sweep_m512": proto["block_sweep_m512"], "flatness": proto["flatness"],
                   "flatness_spread": proto["flatness_spread"]}

    ctx.close()
    forms = None
    if rank == 0 and world == 1 and not args.no_forms:
        # the other forms, bounded (about 1.5 minutes together), after the timed region:
        # precision, batched, replicates and serving
        forms = {}
        for name, fn in (("precision", precision_form), ("batched", batched_form), ("replicates", replicates_form),
                         ("serving", serving_form)):
            t0 = time.perf_counter()
            try:
                forms[name] = fn()
            except Exception as e:  # a form that fails is reported, not fatal to the plain line
                forms[name] = {"error": f"{type(e).__name__}: {e}"}
            forms[name]["bench_wall_s"] = time.perf_counter() - t0
        if "value" in forms.get("batched", {}):
            forms["batched"]["speedup_vs_plain_large"] = forms["batched"]["value"] / value

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Hardy-Weinberg genotypes, planted triplet (17,203,411) at effect 0.8)",
            "config": {"workload": cfg["name"], "form": "plain", "n_snps": M, "n_samples": S,
                       "n_cases": info["n_cases"], "step": f"1/{parts} of the triplet space (first-index shard)",
                       "l2": f"flushed before every step ({args.flush_mb} MiB write)",
                       "parallelism": f"{world} GPU(s), shard-parallel",
                       "engine": ("tensor cores (tcgen05 %s), %d words per stage, %d SNPs j per tile%s"
                                  % ("block-scaled FP4" if engine_fp4 else "int8", tune["stage_words"],
                                     tune["pair_tile"], ", overlapped scoring" if tune.get("overlap") else ""))
                       if engine_tc else "integer (LOP3+POPC)",
                       "autotune_rates": {"int": tune["rate_int"], "tc_int8_4": tune["rate_tc4"],
                                          "tc_int8_8": tune["rate_tc8"], "tc_fp4_8_j32": tune["rate_fp4_8"],
                                          "tc_fp4_8_j64": tune["rate_fp4_8_pair"],
                                          "tc_fp4_16_j32": tune["rate_fp4_16_single"],
                                          "tc_fp4_16_j64": tune["rate_fp4_16"],
                                          "tc_fp4_4_j64_overlap": tune["rate_fp4_4_overlap"],
                                          "tc_fp4_8_j64_overlap": tune["rate_fp4_8_overlap"]}},
            "roofline": roof,
            "clocks": clocks,
            "gpu_launches": launches,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "scan_latency_ms": {"p50": float(np.percentile(kernel_ms, 50)), "p99": float(np.percentile(kernel_ms, 99)),
                                "what": "device time of one step's search kernel"},
            "best_in_last_step": {"score": bests[-1][0], "ijk": list(bests[-1][1])},
            "forms": forms,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _clock_ctx():
    import torch
    pci = None
    try:
        pci = torch.cuda.get_device_properties(0).pci_bus_id
    except Exception:
        pass
    return ClockSampler(pci)


def batched_form(steps=3, warmup=1):
    """Batched workload: 96 datasets (SNPs log-uniform 128..1536, samples log-uniform
    1000..12000, case fraction 0.3..0.7) in one graph-captured tensor-core launch sequence,
    against the same datasets scanned one by one (one epik2_scan each) and against the plain
    form's rate on plain-large."""
    import numpy as np
    import epik2
    from epik2 import workloads as W
    specs = W.batched_specs()
    ctx = epik2.Context(0)
    ids = []
    ts_total = 0.0
    for sp in specs:
        g, p = W.generate(sp)
        ids.append(ctx.load(g, p))
        ts_total += epik2.n_triplets(sp["n_snps"]) * sp["n_samples"]
    for _ in range(max(1, warmup)):
        ctx.scan_batch(ids)
        for d in ids:
            ctx.scan(d)
    sampler = _clock_ctx()
    sampler.start()
    batch_ms, batch_wall, obo_ms, obo_wall = [], [], [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        best_b = ctx.scan_batch(ids)
        batch_wall.append((time.perf_counter() - t0) * 1e3)
        batch_ms.append(ctx.stats()["last_scan_kernel_ms"])
        t0 = time.perf_counter()
        k_ms = 0.0
        best_o = []
        for d in ids:
            best_o.append(ctx.scan(d))
            k_ms += ctx.stats()["last_scan_kernel_ms"]
        obo_wall.append((time.perf_counter() - t0) * 1e3)
        obo_ms.append(k_ms)
    clocks = sampler.stop()
    same = all(a.ijk == b.ijk and a.score == b.score for a, b in zip(best_b, best_o))
    ctx.close()
    v_b = ts_total / (np.median(batch_ms) / 1e3)
    v_o = ts_total / (np.median(obo_wall) / 1e3)
    return {"value": v_b, "unit": UNIT, "ms_per_step": float(np.median(batch_ms)),
            "wall_ms_per_step": float(np.median(batch_wall)), "steps": steps,
            "triplet_samples_per_step": ts_total, "datasets": len(specs),
            "one_by_one": {"value": v_o, "ms_per_step": float(np.median(obo_wall)),
                           "kernel_ms_per_step": float(np.median(obo_ms)),
                           "what": "96 separate epik2_scan calls, wall time (host setup, launches, syncs)"},
            "speedup_vs_one_by_one": v_b / v_o, "results_identical_to_one_by_one": same, "clocks": clocks}


def precision_form(steps=3, warmup=1):
    """Precision workload (2048 SNPs x 8192 samples, three planted triplets): plain FP32 search
    vs search + per-warp top-32 + FP64 rescore on the GPU; the FP64 top-32 (set and order) is
    compared with the FP64 oracle's, recorded in tests/golden/precision_top32.json."""
    import numpy as np
    import epik2
    from epik2 import workloads as W
    cfg = W.PRECISION
    g, p = W.generate(cfg)
    ctx = epik2.Context(0)
    did = ctx.load(g, p)
    ts = epik2.n_triplets(cfg["n_snps"]) * cfg["n_samples"]
    for _ in range(max(1, warmup)):
        ctx.scan(did)
        ctx.scan_topk(did, 32, rescore_fp64=1)
    plain_ms, prec_ms = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        b = ctx.scan(did)
        plain_ms.append((time.perf_counter() - t0) * 1e3)
        t0 = time.perf_counter()
        top = ctx.scan_topk(did, 32, rescore_fp64=1)
        prec_ms.append((time.perf_counter() - t0) * 1e3)
    ctx.close()
    err = [abs(t.score - t.score_fp64) / t.score_fp64 for t in top]
    out = {"value": ts / (np.median(prec_ms) / 1e3), "unit": UNIT, "ms_per_step": float(np.median(prec_ms)),
           "workload": cfg["name"], "top_k": 32,
           "plain": {"value": ts / (np.median(plain_ms) / 1e3), "ms_per_step": float(np.median(plain_ms))},
           "k2_rel_error_fp32_vs_fp64": {"max": max(err), "median": float(np.median(err)), "tolerance": 1e-5},
           "top1": {"ijk": list(top[0].ijk), "score_fp32": top[0].score, "score_fp64": top[0].score_fp64,
                    "same_as_plain": top[0].ijk == b.ijk}}
    try:
        fx = json.load(open(os.path.join(ROOT, "tests", "golden", "precision_top32.json")))
        ref = [x["ijk"] for x in fx["top"]]
        got = [list(t.ijk) for t in top]
        out["vs_fp64_oracle"] = {"top1_equal": got[0] == ref[0], "top32_set_equal": sorted(got) == sorted(ref),
                                 "top32_order_equal": got == ref,
                                 "fp64_scores_bit_equal": all(t.score_fp64 == float.fromhex(x["s64"])
                                                              for t, x in zip(top, fx["top"]))}
    except (OSError, KeyError, ValueError):
        out["vs_fp64_oracle"] = None
    return out


def replicates_form(n_a=64, n_b=8):
    """Permutation replicates of the serving workload's resident matrices (A 1024 SNPs x 8192
    samples, B 3072 x 4096): the replicate form (all-sample counts shared across replicates,
    epik2_scan_replicates) against the same replicates searched one by one with the plain
    kernel (set_pheno + scan each, same CTA-pair FP4 configuration); results must be equal."""
    import numpy as np
    import epik2
    from epik2 import workloads as W
    out = {}
    rng = np.random.default_rng(1006)
    with epik2.Context(0) as ctx:
        for m, n in zip(W.SERVING["resident"], (n_a, n_b)):
            if n <= 0:
                continue
            g, p = W.generate(m)
            reps = np.stack([rng.permutation(p) for _ in range(n)])
            did = ctx.load(g, p)
            ts = epik2.n_triplets(m["n_snps"]) * m["n_samples"] * n
            ctx.scan_replicates(did, reps)  # warm-up: first launches, the replicates' allocation
            t0 = time.perf_counter()
            got = ctx.scan_replicates(did, reps)
            wall_r = time.perf_counter() - t0
            st = ctx.stats()
            kms_r = st["last_scan_kernel_ms"]
            parts = {"alloc_ms": st["last_load_ms"], "encode_ms": st["last_prepare_ms"],
                     "kernel_ms": kms_r, "call_wall_ms": st["last_scan_wall_ms"]}
            kms_p, plain = 0.0, []
            t0 = time.perf_counter()
            for r in reps:
                ctx.set_pheno(did, r)
                plain.append(ctx.scan(did, engine=epik2.ENGINE_TC_FP4, stage_words=16, pair_tile=64, overlap=1))
                kms_p += ctx.stats()["last_scan_kernel_ms"]
            wall_p = time.perf_counter() - t0
            ctx.unload(did)
            out[m["name"]] = {
                "replicates": n, "triplet_samples": ts,
                "replicate_form": {"value": ts / (kms_r / 1e3), "wall_value": ts / wall_r, "kernel_ms": kms_r,
                                   "breakdown": parts},
                "one_by_one_plain": {"value": ts / (kms_p / 1e3), "wall_value": ts / wall_p, "kernel_ms": kms_p},
                "speedup_kernel": kms_p / kms_r, "speedup_wall": wall_p / wall_r,
                "results_identical": all(a.ijk == b.ijk and a.score == b.score for a, b in zip(got, plain))}
    return out


def serving_form(seconds=15.0, drain=15.0, check_requests=6):
    """Serving workload: resident matrices A (1024 SNPs x 8192 samples) and B (3072 x 4096);
    Poisson arrivals; each request 16..1000 phenotype-permutation replicates of a random
    resident matrix, 10% a fresh 256..768-SNP x 4096-sample matrix.  Reports the offered and
    sustained load, completed/refused requests, p50/p99 latency, the FP32-vs-FP64 K2 error of
    every result, and a check of the first result of a few completed requests against a plain
    run of the same phenotype.  A second run offers half the measured capacity with
    16-replicate requests on A (latency at a sustainable rate)."""
    import numpy as np
    import epik2
    from epik2 import workloads as W
    spec = W.SERVING
    rng = np.random.default_rng(spec["seed"])
    gens = [W.generate(m) for m in spec["resident"]]
    pools = [np.stack([rng.permutation(p) for _ in range(256)]) for _, p in gens]

    def serve(rate, duration, req_maker, srv_opts):
        srv = epik2.Server(0, **srv_opts)
        mids = [srv.add_matrix(g, p) for g, p in gens]
        t_start = time.perf_counter()
        next_t = t_start
        pending, offered, refused, work_offered = [], 0, 0, 0.0
        while time.perf_counter() - t_start < duration:
            now = time.perf_counter()
            if now < next_t:
                time.sleep(min(next_t - now, 0.01))
                continue
            next_t += rng.exponential(1.0 / rate)
            offered += 1
            kind, payload, work, what = req_maker(mids)
            work_offered += work
            try:
                rid = srv.submit_replicates(*payload) if kind == "rep" else srv.submit_scan(*payload)
                pending.append((rid, what))
            except epik2.Epik2Error:
                refused += 1
        t_stop = time.perf_counter()
        lat, done, errs = [], [], []
        deadline = t_stop + drain
        while pending and time.perf_counter() < deadline:
            still = []
            for rid, what in pending:
                r = srv.poll(rid)
                if r is None:
                    still.append((rid, what))
                elif r[0] == epik2.OK:
                    lat.append(r[2])
                    done.append((what, r[1][0]))
                    errs += [abs(b.score - b.score_fp64) / b.score_fp64 for b in r[1]]
            pending = still
            time.sleep(0.01)
        st = srv.stats()
        wall = time.perf_counter() - t_start
        srv.close()
        return {"arrival_rate_per_s": rate, "duration_s": duration, "offered_requests": offered,
                "refused_requests": refused, "completed_requests": len(lat), "unfinished_requests": len(pending),
                "offered_triplet_samples_per_s": work_offered / duration,
                "sustained_triplet_samples_per_s": st["triplet_samples"] / wall,
                "latency_s": {"p50": float(np.percentile(lat, 50)) if lat else None,
                              "p99": float(np.percentile(lat, 99)) if lat else None},
                "k2_rel_error_fp32_vs_fp64": {"max": max(errs) if errs else None,
                                              "median": float(np.median(errs)) if errs else None,
                                              "results": len(errs)},
                "scans_done": st["scans_done"], "launches": st["launches"], "max_scans_per_launch": st["max_active"],
                "busy_fraction": st["busy_seconds"] / wall,
                "kernel_fraction_of_busy": st["kernel_seconds"] / max(st["busy_seconds"], 1e-9),
                "replicate_form_scans": st["replicate_scans"]}, done

    def full_request(mids):
        if rng.random() < spec["upload_frac"]:
            m = int(rng.integers(spec["upload_snps"][0], spec["upload_snps"][1] + 1))
            g, p = epik2.generate_hwe(int(rng.integers(1 << 30)), 4096, m, 2048)
            return "scan", (g, p), epik2.n_triplets(m) * 4096, ("fresh", g, p)
        a = int(rng.integers(len(mids)))
        n = int(rng.integers(spec["replicates"][0], spec["replicates"][1] + 1))
        start = int(rng.integers(256))
        ph = np.take(pools[a], np.arange(start, start + n) % 256, axis=0)
        m = spec["resident"][a]
        return "rep", (mids[a], ph), n * epik2.n_triplets(m["n_snps"]) * m["n_samples"], ("rep", a, start)

    srv_opts = dict(rescore_fp64=1, max_queued=20000)
    full, done_full = serve(spec["rate_per_s"], seconds, full_request, srv_opts)
    cap = full["sustained_triplet_samples_per_s"] / max(full["busy_fraction"], 1e-9)
    light_work = 16 * epik2.n_triplets(spec["resident"][0]["n_snps"]) * spec["resident"][0]["n_samples"]
    light_rate = max(0.05, 0.5 * cap / light_work)

    def light_request(mids):
        start = int(rng.integers(256))
        ph = np.take(pools[0], np.arange(start, start + 16) % 256, axis=0)
        return "rep", (mids[0], ph), light_work, ("rep", 0, start)

    light, done_light = serve(light_rate, seconds, light_request, srv_opts)
    # each checked request's first result against a plain run of its phenotype
    checked, matched = 0, 0
    with epik2.Context(0) as ctx:
        dids = [ctx.load(g, p) for g, p in gens]
        for what, best in (done_full[:check_requests] + done_light[:2]):
            if what[0] == "rep":
                ctx.set_pheno(dids[what[1]], pools[what[1]][what[2] % 256])
                ref = ctx.scan(dids[what[1]])
            else:
                ref = ctx.scan_u8(what[1], what[2])
            checked += 1
            matched += int(ref.ijk == best.ijk and ref.score == best.score)
    return {"offered_load_as_configured": full, "half_capacity_16_replicates_on_A": light,
            "capacity_triplet_samples_per_s": cap,
            "per_request_plain_match": {"checked": checked, "matched": matched,
                                        "what": "first result of each checked request vs epik2_scan of that "
                                                "phenotype (bit-exact FP32 score and triplet)"}}


def run_batched(args):
    r = batched_form(args.steps, args.warmup)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (96 seeded Hardy-Weinberg datasets)",
            "config": {"workload": "batched 96 datasets", "form": "batched",
                       "triplet_samples_per_step": r["triplet_samples_per_step"],
                       "step": "one batched launch over all 96 datasets"}, "batched": r}
    print(json.dumps(line))
    return 0


def run_precision(args):
    r = precision_form(args.steps, args.warmup)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 counts, f32 K2, f64 rescore",
            "data": "synthetic (seeded Hardy-Weinberg, MAF 0.01..0.5, planted triplets at 0.6/0.7/0.8)",
            "config": {"workload": r["workload"], "form": "precision", "top_k": 32}, "precision": r}
    print(json.dumps(line))
    return 0


def run_serving(args):
    r = serving_form(args.serve_seconds, args.serve_drain)
    light = r["half_capacity_16_replicates_on_A"]
    line = {"metric": "p50/p99 scan latency; triplet*samples/s", "value": light["latency_s"]["p50"], "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "steps": None, "warmup": None, "vs_baseline": None,
            "dtype": "u32 counts, f32 K2, f64 rescore", "data": "synthetic (seeded Hardy-Weinberg)",
            "config": {"workload": "serving: resident A 1024x8192, B 3072x4096", "form": "serving"}, "serving": r}
    print(json.dumps(line))
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
    ap.add_argument("--form", default="plain", choices=["plain", "batched", "precision", "serving", "replicates"])
    ap.add_argument("--replicates", default="64,8",
                    help="replicates form: replicates of serving matrices A and B (0 leaves a matrix out)")
    ap.add_argument("--engine", default="auto", choices=["auto", "int", "tc", "fp4"],
                    help="plain form: search engine (default: the autotuner's choice)")
    ap.add_argument("--stage-words", type=int, default=0, help="plain form: tensor-core stage depth (0 = tuned)")
    ap.add_argument("--pair-tile", type=int, default=0, help="plain form: SNPs j per tensor-core tile (0 = tuned)")
    ap.add_argument("--overlap", type=int, default=0, help="plain form: overlapped kernel 0 = tuned, 1 = off, 2 = on")
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-drain", type=float, default=30.0)
    ap.add_argument("--no-forms", action="store_true",
                    help="plain form: leave out the bounded batched/precision/serving runs after the timed steps")
    args = ap.parse_args()
    rank, world, local_rank = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.form == "batched":
        return run_batched(args)
    if args.form == "precision":
        return run_precision(args)
    if args.form == "serving":
        return run_serving(args)
    if args.form == "replicates":
        n_a, n_b = (int(x) for x in args.replicates.split(","))
        print(json.dumps({"form": "replicates", "data": "synthetic", "replicates": replicates_form(n_a, n_b)}))
        return 0
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
