#!/usr/bin/env python
"""Radix-join benchmark on B200.

Default workload (the large in-HBM radix join): R = 2^30 tuples (int64 key,
int64 payload) with keys a seeded permutation of 1..2^30, S = 2^30 tuples with
foreign keys drawn from R's keys (Zipf exponent --zipf, 0 = uniform),
payload = key, two radix passes of 9 + 9 bits, bucket-chaining shared-memory
join.  One step = one whole join (prefix sums, both partition passes, join,
result reduction) through the library's engine.  value = (|R| + |S|) / step
time in G tuples/s, inputs resident in HBM (34 GB, larger than L2, so no L2
flush is needed between steps).  e2e = the same join through the C ABI's
host-buffer entry point, with the four input columns copied from pinned host
memory and the result copied back inside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's CPU radix join (its own compiled CPU
partitioner for pass 1, the oracle restatement for pass 2 and the join) on all
host cores over a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "fast-interconnects_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

METRIC = "radix join G tuples/s"
UNIT = "G tuples/s"
# Algorithmic bytes per tuple of a P-pass radix join: key read for the
# histogram, P scatter round trips, one join read: K + P*2T + T.
KEY_B, TUPLE_B = 8, 16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--log2n", type=int, default=30, help="|R| = |S| = 2^log2n")
    ap.add_argument("--zipf", type=float, default=0.0)
    ap.add_argument("--bits", default="9,9")
    ap.add_argument("--scheme", default="chaining", choices=["chaining", "perfect"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-log2n", type=int, default=27,
                    help="CPU baseline sample: |R| = |S| = 2^cpu_log2n")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--workload", default="join",
                    choices=["join", "partition", "ooc", "serve", "dataset", "nopart",
                             "hybrid", "exchange", "refkernels", "sharded"],
                    help="partition: the partition-only sweep; ooc: the "
                         "out-of-core join from pinned host memory; serve: the "
                         "join server against back-to-back plain calls; dataset: "
                         "a named data set of the reference (--data-set); "
                         "refkernels: the reference's own GPU kernels beside "
                         "this repository's on the same inputs")
    ap.add_argument("--data-set", default="blanas",
                    choices=["blanas", "blanas4mb", "kim", "lutz2gv32g", "lutz32gv32g",
                             "custom"],
                    help="dataset workload: Blanas 16M x 256M int64, Kim 128e6 x "
                         "128e6 int32 (the papers' key sizes), ...; custom: |R| = |S| "
                         "= 2^log2n with --zipf and --bits (e.g. the 16M x 16M int32 "
                         "one-pass join: --log2n 24 --bits 10 --tuple-bytes 8)")
    ap.add_argument("--tuple-bytes", type=int, default=0,
                    help="dataset workload: 8 (int32) or 16 (int64); 0 = the "
                         "data set's own")
    ap.add_argument("--selectivity", type=int, default=100,
                    help="dataset workload: join selectivity in percent")
    ap.add_argument("--hybrid-log2n", type=int, default=28,
                    help="hybrid join: |R| = |S| = 2^hybrid_log2n int64 tuples in "
                         "host memory")
    ap.add_argument("--ht-scheme", default="linearprobing",
                    choices=["linearprobing", "perfect"],
                    help="nopart workload: hash table of the no-partitioning join")
    ap.add_argument("--ht-dim", default="0,256",
                    help="nopart workload: grid,block of build and probe (grid 0 "
                         "= 8 CTAs per SM)")
    ap.add_argument("--probe-grouping", default="on", choices=["on", "off"],
                    help="nopart workload: probe tuples grouped by table region "
                         "before probing (the library's default) or probed in "
                         "input order")
    ap.add_argument("--build-grouping", default="on", choices=["on", "off"],
                    help="nopart workload: build tuples grouped by table region "
                         "before inserting (the library's default) or inserted "
                         "in input order")
    ap.add_argument("--exchange-log2n", type=int, default=29,
                    help="exchange workload: int64 tuples one sender partitions "
                         "and sends")
    ap.add_argument("--exchange", default="peer", choices=["peer", "nccl"],
                    help="sharded workload: fused peer-store exchange or the "
                         "library partition + NCCL all-to-all")
    ap.add_argument("--emulate-ranks", type=int, default=1,
                    help="sharded workload on one GPU: ranks emulated in one process")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1 GPUs: N independent replicas of the join "
                         "instead of the sharded join")
    ap.add_argument("--exchange-ranks", type=int, default=8,
                    help="exchange workload: receivers (power of two), emulated "
                         "by local receive columns on this GPU")
    ap.add_argument("--ooc-log2n", type=int, default=31,
                    help="out-of-core join: |R| = |S| = 2^ooc_log2n int64 tuples")
    ap.add_argument("--ooc-block", type=int, default=0,
                    help="out-of-core join: tuples per streamed block (0 = default)")
    ap.add_argument("--serve-requests", type=int, default=10000)
    ap.add_argument("--serve-max-build", type=int, default=1 << 28,
                    help="largest |R| of the served stream (log-uniform from 64K)")
    ap.add_argument("--serve-load", type=float, default=0.8,
                    help="arrival rate relative to the plain path's measured "
                         "capacity")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-repeats", type=int, default=1,
                    help="serve workload: runs of each arm on the same stream")
    ap.add_argument("--serve-workers", type=int, default=2,
                    help="engines of the server that run large joins at once")
    ap.add_argument("--sweep", default="6,8,10,12,14,16,18",
                    help="radix bits of the partition sweep")
    ap.add_argument("--part-log2n", type=int, default=29,
                    help="partition sweep: 2^part_log2n int64 tuples")
    return ap.parse_args()


def workload_name(a):
    n = 1 << a.log2n
    bits = "+".join(a.bits.split(","))
    skew = "uniform" if a.zipf == 0 else "zipf%.1f" % a.zipf
    return "radix_join_%dMx%dM_int64_%sbits_%s_%s" % (n >> 20, n >> 20, bits,
                                                     skew, a.scheme)


def load_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """DRAM traffic per launch of the dominant kernels from the committed ncu
    summary (profiles/traffic.json: measured on a 64M x 64M case and scaled
    to a 1024M x 1024M launch), if present."""
    path = os.path.join(REPO, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        if torch.cuda.is_available():
            torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gen_relations(fi, torch, n, zipf, seed):
    rk = torch.empty(n, dtype=torch.int64, device="cuda")
    sk = torch.empty(n, dtype=torch.int64, device="cuda")
    fi.gen_primary_keys(rk, seed, base=1)
    fi.gen_zipf_foreign_keys(sk, n, zipf, seed + 1, seed, base=1)
    return rk, sk


def cpu_baseline(a, fi, torch):
    """The reference CPU radix join on a bounded sample, all host cores."""
    import numpy as np
    import oracle as O
    n = 1 << a.cpu_log2n
    b1, b2 = [int(x) for x in a.bits.split(",")]
    if torch.cuda.is_available():
        rk, sk = gen_relations(fi, torch, n, a.zipf, a.seed)
        r = rk.cpu().numpy()
        s = sk.cpu().numpy()
        del rk, sk
    else:
        r = O.primary_keys(n, a.seed, np.int64)
        s = O.zipf_foreign_keys(n, n, a.zipf, a.seed + 1, a.seed, np.int64)
    threads = os.cpu_count() or 1
    rp, sp = r.copy(), s.copy()  # payload = key, separate columns
    times = []
    res = None
    for _ in range(2):
        t0 = time.perf_counter()
        res = O.cpu_radix_join(r, rp, s, sp, b1, b2, threads, use_reference=True)
        times.append(time.perf_counter() - t0)
    sm, cnt, phases, kind = res
    assert cnt == n, "CPU baseline lost matches"
    best = min(times)
    return {"value": 2 * n / best / 1e9, "unit": UNIT, "cores": threads,
            "kind": kind,
            "sample": "R=S=2^%d int64 tuples (same generator and seeds), %s+%s bits, "
                      "pass 1 = reference cpu_chunked_prefix_sum + "
                      "cpu_chunked_radix_partition_swwc (one chunk per thread), "
                      "pass 2 + bucket-chaining join = oracle restatement; best of 2"
                      % (a.cpu_log2n, b1, b2),
            "seconds": best}


def run_reference(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np
    import oracle as O
    try:
        import torch
        import fi_sqlops as fi
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    n = 1 << a.cpu_log2n
    b1, b2 = [int(x) for x in a.bits.split(",")]
    if have_gpu:
        torch.cuda.set_device(0)
        rk, sk = gen_relations(fi, torch, n, a.zipf, a.seed)
        r, s = rk.cpu().numpy(), sk.cpu().numpy()
        del rk, sk
        torch.cuda.empty_cache()
    else:
        r = O.primary_keys(n, a.seed, np.int64)
        s = O.zipf_foreign_keys(n, n, a.zipf, a.seed + 1, a.seed, np.int64)
    threads = os.cpu_count() or 1
    rp, sp = r.copy(), s.copy()  # payload = key, separate columns
    kind = None
    for _ in range(a.warmup):
        O.cpu_radix_join(r, rp, s, sp, b1, b2, threads, use_reference=True)
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        sm, cnt, _, kind = O.cpu_radix_join(r, rp, s, sp, b1, b2, threads,
                                            use_reference=True)
        times.append(time.perf_counter() - t0)
    assert cnt == n
    t = sum(times) / len(times)
    value = 2 * n / t / 1e9
    sample = ("R=S=2^%d int64 (bounded sample of %s), %s+%s bits, %d host threads; "
              "pass 1 = reference CPU partitioner compiled from its sources, "
              "pass 2 + join = oracle restatement" % (a.cpu_log2n, workload_name(a),
                                                      b1, b2, threads))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded permutation PK, Zipf/uniform FK)",
            "config": {"workload": workload_name(a), "sample_tuples": 2 * n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                             "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


PHASES = [  # (name, event pairs, algorithmic bytes per tuple of the relation)
    ("pass1_histogram", [(0, 1), (4, 5)], KEY_B),
    ("pass1_scatter", [(1, 2), (5, 6)], 2 * TUPLE_B),
    ("pass2_histogram", [(2, 3), (6, 7)], TUPLE_B),
    ("pass2_scatter", [(3, 4), (7, 8)], 2 * TUPLE_B),
    ("join", [(8, 9)], TUPLE_B),
]


def run_ours(a):
    import torch
    import fi_sqlops as fi
    world, rank, local = dist_setup(a.gpus)
    n = 1 << a.log2n
    bits = [int(x) for x in a.bits.split(",")]
    passes = len(bits)
    rb = fi.RadixBits(*bits)
    scheme = fi.HashingScheme.BucketChaining if a.scheme == "chaining" else \
        fi.HashingScheme.Perfect
    seed = a.seed + 1000 * rank
    rk, sk = gen_relations(fi, torch, n, a.zipf, seed)
    # payload = key, in separate columns (separate memory, as in a table)
    rp, sp = rk.clone(), sk.clone()
    expected_sum = int(sk.sum().item())
    engine = fi.RadixJoinEngine(n, n, torch.int64, rb, scheme)
    stream = torch.cuda.current_stream()

    # warm-up (untimed), checked against the closed form: every S key is a
    # foreign key, so count = |S| and sum = sum(S.payload)
    verified = True
    for _ in range(max(a.warmup, 1)):
        s, c = engine.run(rk, rp, sk, sp)
        verified = verified and (c == n and s == expected_sum)
    engine.status()

    K = a.steps
    ev_sets = []
    for _ in range(K):
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(11)]
        for e in evs:
            e.record(stream)
        ev_sets.append(evs)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        start.record(stream)
        for k in range(K):
            engine.set_events(ev_sets[k])
            engine.run_async(rk, rp, sk, sp)
        end.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    engine.set_events(None)
    clocks = clk.summary()
    elapsed_ms = start.elapsed_time(end)
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    launches = engine.last_launches() * K
    r = engine.result.cpu()
    verified = verified and int(r[1]) == n and int(r[0]) == expected_sum
    ms_per_step = elapsed_ms / K
    value = world * 2 * n * K / (elapsed_ms / 1e3) / 1e9

    # per-phase device times from the events recorded on the launching stream
    peak, peak_kind = load_peaks()
    phases = {}
    for name, pairs, bpt in PHASES:
        if passes == 1 and name.startswith("pass2"):
            continue
        t = statistics.mean(sum(ev[b].elapsed_time(ev[e]) for b, e in pairs)
                            for ev in ev_sets)
        nbytes = 2 * n * bpt
        phases[name] = {"ms": t, "gb_per_s": nbytes / (t / 1e3) / 1e9,
                        "algorithmic_bytes": nbytes}
    dominant = max(phases, key=lambda k: phases[k]["ms"])
    d = phases[dominant]
    traffic = load_traffic().get(dominant)
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": d["gb_per_s"],
                "peak": peak, "unit": "GB/s", "frac": d["gb_per_s"] / peak,
                "peak_source": peak_kind,
                "traffic": traffic,
                "traffic_source": "ncu dram bytes per launch of a 64M x 64M capture, "
                                  "scaled x16 (profiles/traffic.json)",
                "launch_ms": d["ms"] / 2 if dominant != "join" else d["ms"],
                "algorithmic_bytes_per_launch":
                    d["algorithmic_bytes"] // (1 if dominant == "join" else 2)}
    pipe_bytes = 2 * n * (KEY_B + passes * 2 * TUPLE_B + TUPLE_B)
    pipeline = {"algorithmic_bytes_per_step": pipe_bytes,
                "achieved_gb_per_s": pipe_bytes / (ms_per_step / 1e3) / 1e9,
                "frac_of_peak": pipe_bytes / (ms_per_step / 1e3) / 1e9 / peak}

    # e2e through the host-buffer entry point
    e2e = None
    if not a.no_e2e and a.e2e_steps > 0:
        host = [torch.empty(n, dtype=torch.int64, pin_memory=True) for _ in range(4)]
        for h, d in zip(host, (rk, rp, sk, sp)):
            h.copy_(d)
        del rk, rp, sk, sp
        torch.cuda.empty_cache()
        engine.run_host(*host)  # warm-up (allocates device columns)
        t_e2e = []
        for _ in range(a.e2e_steps):
            barrier(world)
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            s, c = engine.run_host(*host)
            t1.record(stream)
            torch.cuda.synchronize()
            verified = verified and c == n and s == expected_sum
            t_e2e.append(t0.elapsed_time(t1))
        e2e_ms = max_over_ranks(statistics.mean(t_e2e), world)
        e2e = {"value": world * 2 * n / (e2e_ms / 1e3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * n * 8, "d2h_bytes_per_step": 16,
               "ms_per_step": e2e_ms,
               "path": "fi_radix_join_engine_run_host_int64 (pinned host columns; the first pass streamed block by block behind the copy)"}
        del host

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a, fi, torch)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": K, "warmup": a.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "int64",
                "data": "synthetic (seeded permutation PK 1..N, Zipf(s)/uniform FK, "
                        "payload = key)",
                "config": {"workload": workload_name(a), "build_tuples": n,
                           "probe_tuples": n, "radix_bits": bits,
                           "hashing_scheme": a.scheme, "zipf_s": a.zipf,
                           "l2_flush": "none: inputs (%d GB) larger than L2"
                                       % (4 * n * 8 // 10**9),
                           "parallelism": "replicas" if world > 1 else "single"},
                "roofline": roofline, "pipeline_roofline": pipeline,
                "phases": phases, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clocks,
                "verified": bool(verified),
                "workspace_gb": engine.workspace_bytes() / 1e9}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def verify_partitioned(torch, keys, pays, rel, chunks, bits, pad):
    """Size-independent check of one partitioned relation against its input:
    the offsets equal the chunked prefix sum of the keys, every stored key
    lies in its region's partition, and per (chunk, partition) region the
    count and the wrapping sums of keys and payloads equal the input's."""
    n = keys.numel()
    F = 1 << bits
    mask = F - 1
    clen = ((n + chunks - 1) // chunks) & ~(128 // 8 - 1)
    idx = torch.arange(n, device="cuda", dtype=torch.int64)
    chunk = torch.clamp(idx // max(clen, 1), max=chunks - 1)
    del idx
    region_in = chunk * F + (keys & mask)
    del chunk
    counts = torch.bincount(region_in, minlength=chunks * F)
    lens = counts.view(chunks, F)
    excl = torch.cumsum(lens, dim=1) - lens
    pidx = torch.arange(F, device="cuda", dtype=torch.int64)
    cidx = torch.arange(chunks, device="cuda", dtype=torch.int64).view(-1, 1)
    exp_off = excl + (clen + pad * F) * cidx + (pidx + 1) * pad
    ok = bool(torch.equal(rel.offsets.view(chunks, F), exp_off))
    ksum = torch.zeros(chunks * F, dtype=torch.int64, device="cuda")
    psum = torch.zeros_like(ksum)
    ksum.index_add_(0, region_in, keys)
    psum.index_add_(0, region_in, pays)
    del region_in
    off = rel.offsets.view(-1)
    slot_region = torch.repeat_interleave(
        torch.arange(chunks * F, device="cuda", dtype=torch.int64), counts)
    slot = torch.repeat_interleave(off - torch.cumsum(counts, 0) + counts, counts) + \
        torch.arange(n, device="cuda", dtype=torch.int64)
    t = rel.relation.view(-1, 2)
    gk, gp = t[slot, 0], t[slot, 1]
    del slot
    ok = ok and bool(((gk & mask) == (slot_region % F)).all())
    gks = torch.zeros_like(ksum)
    gps = torch.zeros_like(psum)
    gks.index_add_(0, slot_region, gk)
    gps.index_add_(0, slot_region, gp)
    return ok and bool(torch.equal(gks, ksum)) and bool(torch.equal(gps, psum))


def run_partition_sweep(a):
    """Partition-only sweep: 2^part_log2n (int64 key, int64 payload) tuples,
    keys and payloads uniform 64-bit from a seed; one step = Chunked prefix
    sum + partition over SM-count chunks.  GB/s counts 40 B per tuple (key
    read + tuple read + tuple write)."""
    import torch
    import fi_sqlops as fi
    world, rank, local = dist_setup(a.gpus)
    n = 1 << a.part_log2n
    seed = a.seed + 1000 * rank
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    pays = torch.empty(n, dtype=torch.int64, device="cuda")
    fi.gen_uniform_u64_keys(keys, seed)
    fi.gen_uniform_u64_keys(pays, seed + 1)
    chunks = torch.cuda.get_device_properties(0).multi_processor_count
    peak, peak_kind = load_peaks()
    stream = torch.cuda.current_stream()
    pad = fi.padding_len(torch.int64)
    sweep = []
    K = a.steps
    with ClockSampler(local) as clk:
        for bits in [int(b) for b in a.sweep.split(",")]:
            # the reference's first-pass choice; the library uses the tile
            # scatter up to 11 bits and the two-level scatter above
            p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                                       fi.GpuRadixPartitionAlgorithm.HSSWWCv4,
                                       fi.RadixBits(bits), chunks, 1024)
            o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, chunks, bits,
                                    torch.int64)
            rel = fi.PartitionedRelation(n, fi.GpuHistogramAlgorithm.Chunked, bits,
                                         chunks, torch.int64)
            for _ in range(max(a.warmup, 1)):
                p.prefix_sum(fi.RadixPass.First, keys, o)
                p.partition(fi.RadixPass.First, keys, pays, o, rel)
            p.status()
            evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)]
                   for _ in range(K)]
            barrier(world)
            torch.cuda.synchronize()
            for k in range(K):
                evs[k][0].record(stream)
                p.prefix_sum(fi.RadixPass.First, keys, o)
                evs[k][1].record(stream)
                p.partition(fi.RadixPass.First, keys, pays, o, rel)
                evs[k][2].record(stream)
            torch.cuda.synchronize()
            barrier(world)
            p.status()
            hist_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
            part_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
            step_ms = max_over_ranks(hist_ms + part_ms, world)
            ok = verify_partitioned(torch, keys, pays, rel, chunks, bits, pad)
            gbs = world * n * 40 / (step_ms / 1e3) / 1e9
            sweep.append({"radix_bits": bits,
                          "scatter": "tile" if bits <= 11 else "two-level",
                          "ms_per_step": step_ms, "prefix_sum_ms": hist_ms,
                          "partition_ms": part_ms, "gb_per_s": gbs,
                          "frac": gbs / world / peak,
                          "prefix_sum_gb_per_s": n * 8 / (hist_ms / 1e3) / 1e9,
                          "verified": ok})
            del p, o, rel
            torch.cuda.empty_cache()
    clocks = clk.summary()
    if rank == 0:
        line = {"metric": "radix partition GB/s",
                "value": min(r["gb_per_s"] for r in sweep), "unit": "GB/s",
                "value_is": "the slowest radix-bit setting of the sweep",
                "n_gpus": world, "steps": K, "warmup": a.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "int64",
                "data": "synthetic (uniform 64-bit keys and payloads from a seed)",
                "config": {"workload": "radix_partition_%dM_int64_uniform_u64"
                                       % (n >> 20), "tuples": n, "chunks": chunks,
                           "histogram": "Chunked",
                           "l2_flush": "none: inputs (%d GB) larger than L2"
                                       % (n * 16 // 10**9)},
                "peak": peak, "peak_source": peak_kind, "sweep": sweep,
                "clocks": clocks, "verified": all(r["verified"] for r in sweep)}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def sharded_relations(fi, torch, D, n, world, rank, seed):
    """Rank `rank`'s shards: R = n primary keys, a seeded permutation spread
    over the ranks (distributed.shard_primary_keys: all ranks' shards make a
    permutation of 1..world*n); S = n foreign keys uniform over 1..world*n
    with a seed per rank; payload = key."""
    rk = torch.empty(n, dtype=torch.int64, device="cuda")
    sk = torch.empty(n, dtype=torch.int64, device="cuda")
    fi.gen_primary_keys(rk, seed, base=1)
    D.shard_primary_keys(rk, world, rank)
    fi.gen_uniform_foreign_keys(sk, world * n, seed + 1 + rank, base=1)
    return rk, sk


def run_sharded(a):
    """The join of R and S sharded over the ranks (the default for N > 1):
    each rank holds 2^log2n tuples of R and of S (weak scaling), sends every
    tuple to the rank named by the key bits above the local join's with the
    fused partition + peer-store kernel (distributed.PeerExchange, CUDA IPC
    receive columns; --exchange nccl: library partition + NCCL all-to-all),
    joins what it received with one reused engine, and an all-reduce adds
    the ranks' {sum, count}.  value = all ranks' tuples / the step's device
    time, max over ranks.  Checked against the closed form (every S key is a
    foreign key: count = world * n, sum = sum of all S payloads).

    With one GPU and --emulate-ranks W > 1 the W ranks are emulated in one
    process: every emulated sender's fused scatter writes into the W local
    receive columns, one after another, then the W local joins run; the
    value is all tuples / the whole time on the one GPU."""
    import torch
    import torch.distributed as dist
    import fi_sqlops as fi
    import distributed as D
    world, rank, local = dist_setup(a.gpus)
    n = 1 << a.log2n
    bits = tuple(int(b) for b in a.bits.split(","))
    scheme = (fi.HashingScheme.Perfect if a.scheme == "perfect"
              else fi.HashingScheme.BucketChaining)
    stream = torch.cuda.current_stream()
    emulate = a.emulate_ranks if world == 1 else 1
    own_group = False
    if world == 1 and emulate == 1:
        # one rank: the exchange's collectives still need a process group
        import datetime
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port,
                                rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=600))
        own_group = True
    W = max(world, emulate)
    shift = sum(bits)
    g = D.exchange_bits(W)
    mask = (1 << 64) - 1
    K = a.steps

    if emulate > 1:
        m = n // emulate
        shards = [sharded_relations(fi, torch, D, m, emulate, r, a.seed) for r in range(emulate)]
        expected = (sum(int(sk.sum().item()) for _, sk in shards) & mask, emulate * m)
        mats = []
        for rel in (0, 1):
            mats.append(torch.stack([fi.exchange_histogram(sh[rel], shift, g)
                                     for sh in shards]).cpu())
        recv = [m_.sum(0).tolist() for m_ in mats]
        cols = [[torch.empty((2, max(c, 1)), dtype=torch.int64, device="cuda")
                 for c in recv[rel]] for rel in (0, 1)]
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        engine = D.EngineJoin(max(recv[0]), max(recv[1]), torch.int64, bits, scheme)

        def step():
            for rel in (0, 1):
                for s_, sh in enumerate(shards):
                    base, _ = D.region_bases(mats[rel], s_)
                    dests = [(cols[rel][d][0].data_ptr(), cols[rel][d][1].data_ptr(),
                              base[d], recv[rel][d]) for d in range(W)]
                    fi.exchange_scatter(sh[rel], sh[rel], shift, g, dests, status=status)
            tot_s, tot_c = 0, 0
            for d in range(W):
                nr, ns = recv[0][d], recv[1][d]
                if nr and ns:
                    sm_, c_ = engine(cols[0][d][0][:nr], cols[0][d][1][:nr],
                                     cols[1][d][0][:ns], cols[1][d][1][:ns], bits, scheme)
                    tot_s, tot_c = (tot_s + sm_) & mask, tot_c + c_
            return tot_s, tot_c
        ex_ms = None
    else:
        rk, sk = sharded_relations(fi, torch, D, n, world, rank, a.seed)
        part = torch.tensor([int(sk.sum().item())], dtype=torch.int64, device="cuda")
        if world > 1:
            dist.all_reduce(part)
        expected = (int(part.item()) & mask, world * n)
        caps = [max(D.region_bases(D.all_gather_counts(
            fi.exchange_histogram(k, shift, g)), rank)[1]) for k in (rk, sk)]
        peers = None
        if a.exchange == "peer":
            peers = (D.PeerExchange(caps[0], torch.int64), D.PeerExchange(caps[1], torch.int64))
        engine = D.EngineJoin(caps[0], caps[1], torch.int64, bits, scheme)
        ev_x = []

        def step():
            # exchange_join's steps, with events around the two shuffles
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if peers is not None:
                rk2, rp2 = peers[0].shuffle(rk, rk, shift)
                sk2, sp2 = peers[1].shuffle(sk, sk, shift)
            else:
                rk2, rp2 = D.shuffle(rk, rk, shift)
                sk2, sp2 = D.shuffle(sk, sk, shift)
            e1.record(stream)
            ev_x.append((e0, e1))
            s_, c_ = engine(rk2, rp2, sk2, sp2, bits, scheme)
            tt = torch.tensor([s_, c_], dtype=torch.int64, device="cuda")
            if world > 1:
                dist.all_reduce(tt)
            return int(tt[0].item()) & mask, int(tt[1].item())

    verified = True
    for _ in range(max(a.warmup, 1)):
        verified = verified and step() == expected
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if emulate == 1:
        ev_x.clear()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(K):
            verified = step() == expected and verified
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms_per_step = max_over_ranks(ev0.elapsed_time(ev1) / K, world)
    value = 2 * W * (n if emulate == 1 else n // emulate) / (ms_per_step / 1e3) / 1e9
    clocks = clk.summary()
    nvlink = None
    if emulate == 1:
        ex_ms = max_over_ranks(statistics.mean(a_.elapsed_time(b_) for a_, b_ in ev_x), world)
        sent = 2 * n * 16 * (W - 1) / W  # tuples leaving this rank, both relations
        nvlink = {"exchange_ms": ex_ms, "bytes_sent_per_rank": int(sent),
                  "achieved_gb_per_s": sent / (ex_ms / 1e3) / 1e9 if W > 1 else None,
                  "peak_gb_per_s": 770.0, "peak_source": "measured peer copy per direction"}

    e2e = None
    if emulate == 1 and not a.no_e2e and a.e2e_steps > 0:
        # the public API with host columns: H2D copies of this rank's four
        # columns, exchange_join, result back to the host
        host = [torch.empty(n, dtype=torch.int64, pin_memory=True) for _ in range(4)]
        for h, d in zip(host, (rk, rk, sk, sk)):
            h.copy_(d)
        rp_d, sp_d = torch.empty_like(rk), torch.empty_like(sk)
        t_e2e = []
        for _ in range(a.e2e_steps):
            barrier(world)
            torch.cuda.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for dst, h in zip((rk, rp_d, sk, sp_d), host):
                dst.copy_(h, non_blocking=True)
            res = D.exchange_join(rk, rp_d, sk, sp_d, bits=bits, scheme=scheme,
                                  exchange=a.exchange, peers=peers, local_join=engine)
            t1.record(stream)
            torch.cuda.synchronize()
            verified = verified and ((res[0] & mask), res[1]) == expected
            t_e2e.append(t0.elapsed_time(t1))
        e2e_ms = max_over_ranks(statistics.mean(t_e2e), world)
        e2e = {"value": 2 * world * n / (e2e_ms / 1e3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * n * 8 * world, "d2h_bytes_per_step": 16 * world,
               "ms_per_step": e2e_ms,
               "path": "distributed.exchange_join over pinned host columns copied in per step"}
        del host
    if emulate == 1 and peers is not None:
        for p_ in peers:
            p_.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": K, "warmup": a.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "int64",
                "data": "synthetic (seeded permutation PK spread over the ranks, "
                        "uniform FK over all ranks' keys, payload = key)",
                "config": {"workload": "sharded_radix_join_%dx(%dMx%dM)_int64_%sbits_%s"
                                       % (W, (n // emulate) >> 20, (n // emulate) >> 20,
                                          "+".join(map(str, bits)), a.scheme),
                           "tuples_per_rank_per_relation": n // emulate,
                           "ranks": W, "emulated_ranks": emulate > 1,
                           "exchange": "emulated local receive columns" if emulate > 1
                                       else a.exchange,
                           "exchange_bits": g, "radix_bits": list(bits),
                           "l2_flush": "none: inputs larger than L2",
                           "parallelism": "sharded%d" % W},
                "nvlink": nvlink, "e2e": e2e, "clocks": clocks,
                "verified": bool(verified)}
        print(json.dumps(line), flush=True)
    if world > 1 or own_group:
        dist.barrier()
        dist.destroy_process_group()


def run_refkernels(a):
    """The reference's own GPU kernels (baseline/refgpu: compiled for sm_100a
    from its sources, launched with its argument structs, grids and shared
    memory) beside this repository's on the same B200 and the same inputs.

    Partition (config 2 shape): 2^part_log2n int64 tuples, uniform 64-bit
    keys, SM-count chunks; per radix-bit setting the Chunked prefix sum and
    the NC and LASWWC scatters of the reference against this repository's
    prefix sum and scatter.  Every output is verified: offsets identical,
    and each scattered relation checked region by region against its input.
    The reference's SSWWC variants spin on buffer slots without a bound and
    are not run.

    Join: R = S = 2^24 int32 at 10 bits (config 1) and 2^28 int64 at 16 bits
    (the final partitions of the config-3 join: ~4096 tuples each), keys a
    seeded permutation of 1..N, uniform foreign keys, payload = key;
    assign_tasks + the reference's shared-memory join (grid = SMs, 1024
    threads) against this repository's join on the same partitioned
    relations, both checked against the closed form (sum of S payloads)."""
    import types
    import torch
    import fi_sqlops as fi
    sys.path.insert(0, os.path.join(REPO, "baseline", "refgpu"))
    import refgpu
    world, rank, local = dist_setup(a.gpus)
    if rank != 0:
        return
    if not refgpu.available():
        print(json.dumps({"workload": "reference_gpu_kernels",
                          "unavailable": "baseline/refgpu/_build/libref_gpu.so not built"}))
        return
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    stream = torch.cuda.current_stream()
    K, W = a.steps, max(a.warmup, 1)
    peak, peak_kind = load_peaks()

    def timed(fn):
        for _ in range(W):
            fn()
        evs = [(torch.cuda.Event(enable_timing=True),
                torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        torch.cuda.synchronize()
        for e0, e1 in evs:
            e0.record(stream)
            fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return statistics.mean(e0.elapsed_time(e1) for e0, e1 in evs)

    n = 1 << a.part_log2n
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    pays = torch.empty(n, dtype=torch.int64, device="cuda")
    fi.gen_uniform_u64_keys(keys, a.seed)
    fi.gen_uniform_u64_keys(pays, a.seed + 1)
    pad = fi.padding_len(torch.int64)
    prows, jrows = [], []
    with ClockSampler(local) as clk:
        for bits in [int(b) for b in a.sweep.split(",") if int(b) <= 14]:
            F = 1 << bits
            row = {"radix_bits": bits}
            ref_off = torch.empty(sms * F, dtype=torch.int64, device="cuda")
            row["ref_prefix_sum_ms"] = timed(
                lambda: refgpu.chunked_prefix_sum(keys, sms, bits, out=ref_off))
            p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                                       fi.GpuRadixPartitionAlgorithm.HSSWWCv4,
                                       fi.RadixBits(bits), sms, 1024)
            o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, sms, bits,
                                    torch.int64)
            rel = fi.PartitionedRelation(n, fi.GpuHistogramAlgorithm.Chunked, bits, sms,
                                         torch.int64)
            row["our_prefix_sum_ms"] = timed(
                lambda: p.prefix_sum(fi.RadixPass.First, keys, o))
            row["offsets_identical"] = bool(torch.equal(o.offsets.view(-1), ref_off))

            def ours_part():
                p.prefix_sum(fi.RadixPass.First, keys, o)
                p.partition(fi.RadixPass.First, keys, pays, o, rel)
            both = timed(ours_part)
            row["our_partition_ms"] = both - row["our_prefix_sum_ms"]
            p.status()
            row["our_verified"] = verify_partitioned(torch, keys, pays, rel, sms, bits, pad)
            del p, o, rel
            torch.cuda.empty_cache()
            ref_rel = torch.empty((n + sms * F * pad, 2), dtype=torch.int64, device="cuda")
            view = types.SimpleNamespace(offsets=ref_off, relation=ref_rel)
            for name, variant in (("nc", refgpu.NC), ("laswwc", refgpu.LASWWC)):
                try:
                    part = refgpu.Partition(variant, keys, pays, sms, bits, ref_off,
                                            ref_rel)
                except refgpu.RefGpuError as e:
                    row["ref_%s" % name] = "refused: %s" % e
                    continue
                row["ref_%s_partition_ms" % name] = timed(part.launch)
                row["ref_%s_verified" % name] = verify_partitioned(
                    torch, keys, pays, view, sms, bits, pad)
            del ref_rel, view
            torch.cuda.empty_cache()
            row["ref_best_ms"] = row["ref_prefix_sum_ms"] + min(
                v for k, v in row.items()
                if k.startswith("ref_") and k.endswith("_partition_ms"))
            row["our_ms"] = row["our_prefix_sum_ms"] + row["our_partition_ms"]
            row["speedup"] = row["ref_best_ms"] / row["our_ms"]
            row["our_gb_per_s"] = n * 40 / (row["our_ms"] / 1e3) / 1e9
            row["ref_best_gb_per_s"] = n * 40 / (row["ref_best_ms"] / 1e3) / 1e9
            prows.append(row)
        del keys, pays
        torch.cuda.empty_cache()
        for label, dt, log2n, bits in (("config1_16Mx16M_int32_10bits", torch.int32, 24, 10),
                                       ("final_partitions_256Mx256M_int64_16bits",
                                        torch.int64, 28, 16)):
            m = 1 << log2n
            rk = torch.empty(m, dtype=dt, device="cuda")
            sk = torch.empty(m, dtype=dt, device="cuda")
            fi.gen_primary_keys(rk, a.seed + 7, base=1)
            fi.gen_uniform_foreign_keys(sk, m, a.seed + 8, base=1)
            exp = int(sk.to(torch.int64).sum().item()) & ((1 << 64) - 1)
            rels = []
            for k in (rk, sk):
                pp = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Contiguous,
                                            fi.GpuRadixPartitionAlgorithm.SSWWCv2,
                                            fi.RadixBits(bits), sms, 1024)
                oo = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Contiguous, sms, bits, dt)
                rr = fi.PartitionedRelation(m, fi.GpuHistogramAlgorithm.Contiguous, bits,
                                            sms, dt)
                pp.prefix_sum(fi.RadixPass.First, k, oo)
                pp.partition(fi.RadixPass.First, k, k, oo, rr)
                pp.status()
                rels.append(rr)
            b, pr = rels
            for sname, rscheme, fscheme in (("perfect", refgpu.PERFECT, fi.HashingScheme.Perfect),
                                            ("chaining", refgpu.CHAINING,
                                             fi.HashingScheme.BucketChaining)):
                jr = {"workload": label, "scheme": sname, "tuples": 2 * m}
                try:
                    j = refgpu.Join(rscheme, b.relation, b.offsets, b.padded_len(),
                                    pr.relation, pr.offsets, pr.padded_len(), bits,
                                    bits, sms, 1024)
                    j.launch()
                    jr["ref_verified"] = j.sum() == exp
                    jr["ref_join_ms"] = timed(j.launch)
                except refgpu.RefGpuError as e:
                    jr["ref"] = "refused: %s" % e
                res = torch.zeros(sms * 1024, dtype=torch.int64, device="cuda")
                tasks = torch.zeros(sms + 1, dtype=torch.int32, device="cuda")
                jo = fi.CudaRadixJoin(fi.RadixPass.First, fi.RadixBits(bits), fscheme,
                                      sms, 1024)
                jo.join(b, pr, res, tasks)
                jo.status()
                jr["our_verified"] = (int(res.sum().item()) & ((1 << 64) - 1)) == exp
                jr["our_join_ms"] = timed(lambda: jo.join(b, pr, res, tasks))
                if "ref_join_ms" in jr:
                    jr["speedup"] = jr["ref_join_ms"] / jr["our_join_ms"]
                jrows.append(jr)
            del rels, b, pr, rk, sk
            torch.cuda.empty_cache()
    line = {"metric": "reference GPU kernels vs this repository's (ms per launch)",
            "workload": "reference_gpu_kernels", "n_gpus": 1, "steps": K,
            "warmup": W, "dtype": "int64 / int32",
            "data": "synthetic (uniform 64-bit keys; seeded permutation PK, uniform FK)",
            "config": {"workload": "reference_gpu_kernels",
                       "partition_tuples": n, "chunks": sms,
                       "reference_grid_block": [sms, 1024]},
            "peak": peak, "peak_source": peak_kind,
            "partition": prows, "join": jrows, "clocks": clk.summary(),
            "verified": all(r.get("offsets_identical") and r.get("our_verified")
                            and all(v for k, v in r.items() if k.endswith("_verified"))
                            for r in prows)
            and all(all(v for k, v in r.items() if k.endswith("_verified"))
                    for r in jrows)}
    print(json.dumps(line), flush=True)


def h2d_probe(torch, nbytes=1 << 30, reps=5):
    """Pinned host-to-device copy bandwidth (GB/s): the host-link roofline."""
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d.copy_(h, non_blocking=True)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(reps):
        d.copy_(h, non_blocking=True)
    t1.record()
    torch.cuda.synchronize()
    gbs = nbytes * reps / (t0.elapsed_time(t1) / 1e3) / 1e9
    del h, d
    return gbs


def run_ooc(a):
    """Out-of-core join: R = S = 2^ooc_log2n (int64 key, int64 payload) in
    pinned host memory (fewer if the host cannot hold them), R keys a
    permutation of 1..N, S uniform foreign keys, payload = key in its own
    column.  One step = one whole join with the first pass streamed over the
    host link.  Reports tuples/s and host-link GB/s (16 B per tuple read
    once over the link) against the measured pinned host-to-device copy."""
    import psutil
    import torch
    import fi_sqlops as fi
    world, rank, local = dist_setup(a.gpus)
    log2n = a.ooc_log2n
    avail = psutil.virtual_memory().available
    while log2n > 20 and 4 * 8 * (1 << log2n) * 1.25 > avail:
        log2n -= 1
    n = 1 << log2n
    seed = a.seed + 1000 * rank
    host = []
    for gen in ("pk", "fk"):
        d = torch.empty(n, dtype=torch.int64, device="cuda")
        if gen == "pk":
            fi.gen_primary_keys(d, seed, base=1)
        else:
            fi.gen_uniform_foreign_keys(d, n, seed + 1, base=1)
            expected_sum = int(d.sum().item())
        for _ in range(2):  # key column, then payload = key
            h = torch.empty(n, dtype=torch.int64, pin_memory=True)
            h.copy_(d)
            host.append(h)
        del d
    torch.cuda.empty_cache()
    link = h2d_probe(torch)
    engine = fi.RadixJoinEngine(n, n, torch.int64, fi.RadixBits(9, 9),
                                fi.HashingScheme.BucketChaining)
    verified = True
    for _ in range(max(a.warmup, 1)):
        s, c = engine.run_streamed(*host, block_tuples=a.ooc_block)
        verified = verified and (c == n and s == expected_sum)
    K = a.steps
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(11)] for _ in range(K)]
    wall = []
    with ClockSampler(local) as clk:
        for k in range(K):
            engine.set_events(evs[k])
            barrier(world)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s, c = engine.run_streamed(*host, block_tuples=a.ooc_block)
            wall.append(time.perf_counter() - t0)
            verified = verified and (c == n and s == expected_sum)
    engine.set_events(None)
    engine.status()
    clocks = clk.summary()
    dev_ms = max_over_ranks(statistics.mean(e[0].elapsed_time(e[10]) for e in evs),
                            world)
    stream_ms = statistics.mean(e[1].elapsed_time(e[2]) + e[5].elapsed_time(e[6])
                                for e in evs)
    link_bytes = 2 * n * 16
    if rank == 0:
        line = {"metric": "out-of-core radix join G tuples/s",
                "value": world * 2 * n / (dev_ms / 1e3) / 1e9, "unit": "G tuples/s",
                "n_gpus": world, "steps": K, "warmup": a.warmup,
                "ms_per_step": dev_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int64",
                "data": "synthetic (seeded permutation PK 1..N, uniform FK, "
                        "payload = key) in pinned host memory",
                "config": {"workload": "ooc_radix_join_%dMx%dM_int64_9+9bits_uniform"
                                       % (n >> 20, n >> 20),
                           "tuples_per_relation": n, "requested_log2n": a.ooc_log2n,
                           "block_tuples": a.ooc_block or (1 << 26),
                           "host_bytes": 4 * 8 * n,
                           "l2_flush": "none: inputs in host memory"},
                "host_link": {"bytes_per_step": link_bytes,
                              "achieved_gb_per_s": link_bytes / (dev_ms / 1e3) / 1e9,
                              "peak_gb_per_s": link,
                              "peak_source": "pinned cudaMemcpyAsync H2D, 1 GiB x 5",
                              "frac": link_bytes / (dev_ms / 1e3) / 1e9 / link,
                              "streamed_pass1_ms": stream_ms},
                "wall_ms_per_step": 1e3 * statistics.mean(wall),
                "gpu_launches": engine.last_launches() * K,
                "clocks": clocks, "verified": bool(verified),
                "workspace_gb": engine.workspace_bytes() / 1e9}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def serve_requests(a):
    """The served-join stream: |R| log-uniform in [64K, max], |S| = k |R|
    with k in {1,2,4,8,16}, int32 or int64 tuples, S uniform or Zipf(1.0),
    all from a seed.  Arrivals are set by serve_arrivals."""
    import numpy as np
    rng = np.random.default_rng(a.seed)
    reqs = []
    lo, hi = np.log(64 << 10), np.log(a.serve_max_build)
    for i in range(a.serve_requests):
        rn = int(np.exp(rng.uniform(lo, hi)))
        k = int(rng.choice([1, 2, 4, 8, 16]))
        tb = int(rng.choice([8, 16]))
        z = float(rng.choice([0.0, 1.0]))
        reqs.append({"tb": tb, "rn": rn, "sn": k * rn, "seed": a.seed + 7 * i, "zipf": z})
    return reqs


def serve_arrivals(a, reqs, capacity_s):
    """Seeded Poisson arrivals at a.serve_load times the plain path's
    measured capacity (requests / sum of its service times)."""
    import numpy as np
    rng = np.random.default_rng(a.seed + 1)
    rate = a.serve_load * len(reqs) / capacity_s
    t = 0.0
    for r in reqs:
        t += rng.exponential(1.0 / rate)
        r["arrival"] = t
    return rate


def pctl(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs), q))


def run_plain_calls(fi, torch, reqs, max_build, slice_, t_start=None):
    """Back-to-back plain calls: one request after the other on one reused
    engine per tuple type (build once, probe slices), generating its
    relations with the same kernels.  Returns per-request (result, service
    seconds, completion time).  With t_start, request i starts no earlier
    than t_start + its arrival (a live run of the arrival stream)."""
    engines = {tb: fi.RadixJoinEngine(max_build, slice_,
                                      torch.int64 if tb == 16 else torch.int32,
                                      fi.RadixBits(12, 10),
                                      fi.HashingScheme.BucketChaining)
               for tb in (8, 16)}
    out = []
    for r in reqs:
        dt = torch.int64 if r["tb"] == 16 else torch.int32
        torch.cuda.synchronize()
        if t_start is not None:
            delay = t_start + r["arrival"] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
        t0 = time.perf_counter()
        rk = torch.empty(r["rn"], dtype=dt, device="cuda")
        sk = torch.empty(r["sn"], dtype=dt, device="cuda")
        fi.gen_primary_keys(rk, r["seed"])
        if r["zipf"] > 0:
            fi.gen_zipf_foreign_keys(sk, r["rn"], r["zipf"], r["seed"] + 1, r["seed"])
        else:
            fi.gen_uniform_foreign_keys(sk, r["rn"], r["seed"] + 1)
        e = engines[r["tb"]]
        p = fi.autotune_plan(r["tb"], r["rn"], r["sn"], 1 if r["zipf"] > 0 else 0,
                             small_tuples=1)
        e.set_plan(fi.RadixBits(*p["bits"]), p["scheme"], p["join_block"], p["scatter"])
        e.build(rk, rk)
        s_tot, c_tot = 0, 0
        for o in range(0, r["sn"], slice_):
            s, c = e.probe(sk[o:o + slice_], sk[o:o + slice_])
            s_tot, c_tot = (s_tot + s) & ((1 << 64) - 1), c_tot + c
        t1 = time.perf_counter()
        out.append(((s_tot, c_tot), t1 - t0, t1))
        del rk, sk
    e = None
    engines.clear()
    return out


def run_serve(a):
    """Served and batched joins against back-to-back plain calls on the same
    request stream, both live: a first plain pass measures the service times
    (the arrival rate is set from that capacity); then, --serve-repeats
    times each, the plain arm runs the requests one after the other in
    arrival order, each starting no earlier than its arrival, and the served
    arm hands each request to the join server at its arrival time from a
    submitter thread.  Latency = completion - arrival; throughput = all
    tuples / (last completion - first arrival)."""
    import threading
    import torch
    import fi_sqlops as fi
    world, rank, local = dist_setup(a.gpus)
    reqs = serve_requests(a)
    slice_ = a.serve_max_build
    tuples = sum(r["rn"] + r["sn"] for r in reqs)
    mask = (1 << 64) - 1
    # warm-up of both paths on a few requests (untimed)
    warm = reqs[:max(a.warmup, 1)]
    for r in warm:
        r["arrival"] = 0.0
    run_plain_calls(fi, torch, warm, a.serve_max_build, slice_)
    torch.cuda.empty_cache()
    # capacity from measured service times, then the arrival timeline
    first = run_plain_calls(fi, torch, reqs, a.serve_max_build, slice_)
    torch.cuda.empty_cache()
    rate = serve_arrivals(a, reqs, sum(p[1] for p in first))
    expected = [p[0] for p in first]
    verified = all(c == r["sn"] for (_, c), r in zip(expected, reqs))

    def plain_arm():
        t_start = time.perf_counter() + 0.05
        res = run_plain_calls(fi, torch, reqs, a.serve_max_build, slice_, t_start)
        torch.cuda.empty_cache()
        lat = [p[2] - (t_start + r["arrival"]) for p, r in zip(res, reqs)]
        span = res[-1][2] - (t_start + reqs[0]["arrival"])
        ok = all(p[0] == e for p, e in zip(res, expected))
        return {"g_tuples_per_s": tuples / span / 1e9, "makespan_s": span,
                "busy_g_tuples_per_s": tuples / sum(p[1] for p in res) / 1e9,
                "p50_ms": 1e3 * pctl(lat, 50), "p99_ms": 1e3 * pctl(lat, 99),
                "p999_ms": 1e3 * pctl(lat, 99.9)}, lat, ok

    def served_arm():
        srv = fi.JoinServer(hbm_budget_bytes=int(a.serve_budget_gb * 1e9),
                            workers=a.serve_workers, max_build=a.serve_max_build,
                            probe_slice=slice_)
        for t in [srv.submit(tuple_bytes=r["tb"], build_len=r["rn"], probe_len=r["sn"],
                             seed=r["seed"], zipf_s=r["zipf"]) for r in warm]:
            srv.wait(t)
        tickets = [None] * len(reqs)
        lag = [0.0] * len(reqs)

        def submitter(t_start):
            for i, r in enumerate(reqs):
                delay = t_start + r["arrival"] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                lag[i] = time.perf_counter() - (t_start + r["arrival"])
                tickets[i] = srv.submit(tuple_bytes=r["tb"], build_len=r["rn"],
                                        probe_len=r["sn"], seed=r["seed"],
                                        zipf_s=r["zipf"])

        t_start = time.perf_counter() + 0.05
        th = threading.Thread(target=submitter, args=(t_start,))
        th.start()
        resp = []
        for i in range(len(reqs)):
            while tickets[i] is None:
                time.sleep(50e-6)
            resp.append(srv.wait(tickets[i]))
        t_end = time.perf_counter()
        th.join()
        stats = srv.stats()
        srv.close()
        lat = [g["latency_us"] / 1e6 + lag[i] for i, g in enumerate(resp)]
        span = t_end - (t_start + reqs[0]["arrival"])
        ok = all(g["status"] == 0 and ((g["sum"] & mask), g["count"]) == e
                 for g, e in zip(resp, expected))
        small = [i for i, g in enumerate(resp) if g["batched"]]
        out = {"g_tuples_per_s": tuples / span / 1e9, "makespan_s": span,
               "p50_ms": 1e3 * pctl(lat, 50), "p99_ms": 1e3 * pctl(lat, 99),
               "p999_ms": 1e3 * pctl(lat, 99.9),
               "small_p99_ms": 1e3 * pctl([lat[i] for i in small], 99) if small else None,
               "batched_requests": len(small), "batches": stats["batches"],
               "engine_runs": stats["engine_runs"],
               "engine_busy_s": stats["engine_busy_us"] / 1e6,
               "batch_busy_s": stats["batch_busy_us"] / 1e6,
               "scheduler_enqueue_s": stats["enqueue_us"] / 1e6,
               "peak_reserved_gb": stats["peak_reserved_bytes"] / 1e9,
               "fixed_gb": stats["fixed_bytes"] / 1e9}
        return out, small, ok

    served_runs, plain_runs = [], []
    with ClockSampler(local) as clk:
        for _ in range(max(a.serve_repeats, 1)):
            sv, small, ok_s = served_arm()
            pl, plat, ok_p = plain_arm()
            pl["small_p99_ms"] = 1e3 * pctl([plat[i] for i in small], 99) if small else None
            served_runs.append(sv)
            plain_runs.append(pl)
            verified = verified and ok_s and ok_p
    clocks = clk.summary()

    def spread(runs, key):
        xs = [r[key] for r in runs]
        return {"mean": sum(xs) / len(xs), "min": min(xs), "max": max(xs)}

    served, plain = served_runs[-1], plain_runs[-1]
    if rank == 0:
        line = {"metric": "served radix join G tuples/s",
                "value": spread(served_runs, "g_tuples_per_s")["mean"],
                "unit": "G tuples/s",
                "n_gpus": world, "steps": len(reqs), "warmup": len(warm),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "int32+int64",
                "data": "synthetic (seeded Poisson stream; PK permutations, "
                        "uniform/Zipf FK, payload = key)",
                "config": {"workload": "served_joins_%d_requests" % len(reqs),
                           "requests": len(reqs), "tuples": tuples,
                           "max_build": a.serve_max_build,
                           "arrival_rate_per_s": rate, "offered_load": a.serve_load,
                           "hbm_budget_gb": a.serve_budget_gb,
                           "server_workers": a.serve_workers,
                           "repeats": len(served_runs),
                           "l2_flush": "none: relations of most requests exceed L2"},
                "served": served, "plain": plain,
                "repeats": {"served_g_tuples_per_s": spread(served_runs, "g_tuples_per_s"),
                            "plain_g_tuples_per_s": spread(plain_runs, "g_tuples_per_s"),
                            "served_p99_ms": spread(served_runs, "p99_ms"),
                            "plain_p99_ms": spread(plain_runs, "p99_ms"),
                            "served_runs": served_runs, "plain_runs": plain_runs},
                "clocks": clocks, "verified": bool(verified)}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


DATASETS = {  # name -> (fi.Dataset member, tuple bytes of the paper)
    "blanas": ("Blanas", 16), "blanas4mb": ("Blanas4MB", 16), "kim": ("Kim", 8),
    "lutz2gv32g": ("Lutz2Gv32G", 16), "lutz32gv32g": ("Lutz32Gv32G", 16),
    "custom": ("Custom", 16)}


def gen_custom(fi, torch, a, dt, seed):
    """The reference's Custom data set (radix-join/src/main.rs:727-757):
    |R| = |S| = 2^log2n, primary keys with the join selectivity, foreign keys
    uniform or Zipf(--zipf) over them; payload = key."""
    n = 1 << a.log2n
    rk = torch.empty(n, dtype=dt, device="cuda")
    sk = torch.empty(n, dtype=dt, device="cuda")
    fi.gen_primary_keys(rk, seed)
    fi.null_keys(rk, a.selectivity, seed + 7)
    fi.gen_zipf_foreign_keys(sk, n, a.zipf, seed + 1, seed)
    return rk, rk.clone(), sk, sk.clone()


def run_dataset(a):
    """Join of one of the reference's named data sets (seeded primary keys
    with the join selectivity applied, uniform foreign keys, payload = key)
    on the autotuner's plan; checked against the match count and payload sum
    recomputed from the selectivity draw of each foreign key."""
    import torch
    import fi_sqlops as fi
    world, rank, local = dist_setup(a.gpus)
    name, paper_tb = DATASETS[a.data_set]
    tb = a.tuple_bytes or paper_tb
    dt = torch.int32 if tb == 8 else torch.int64
    seed = a.seed + 1000 * rank
    if name == "Custom":
        rk, rp, sk, sp = gen_custom(fi, torch, a, dt, seed)
    else:
        rk, rp, sk, sp = fi.gen_dataset(getattr(fi.Dataset, name), dt,
                                        selectivity=a.selectivity, seed=seed)
    nb, npr = rk.numel(), sk.numel()
    kept = fi.null_keys(sk.clone(), a.selectivity, seed + 7) != -1
    exp_c = int(kept.sum().item())
    exp_s = int(sp.to(torch.int64)[kept].sum().item())
    del kept
    plan = fi.autotune_plan(tb, nb, npr, small_tuples=1)
    bits = plan["bits"] if plan["bits"] and plan["bits"][0] > 0 else (1,)
    if name == "Custom":  # the given bits, default join shape and scatter
        bits = tuple(int(x) for x in a.bits.split(","))
        plan = dict(plan, join_block=0, scatter=0)
    engine = fi.RadixJoinEngine(nb, npr, dt, fi.RadixBits(*bits),
                                fi.HashingScheme.BucketChaining)
    engine.set_plan(fi.RadixBits(*bits), fi.HashingScheme.BucketChaining,
                    plan["join_block"], plan["scatter"])
    stream = torch.cuda.current_stream()
    verified = True
    for _ in range(max(a.warmup, 1)):
        s, c = engine.run(rk, rp, sk, sp)
        verified = verified and (s, c) == (exp_s, exp_c)
    engine.status()
    K = a.steps
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(K):
            engine.run_async(rk, rp, sk, sp)
        end.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    r = engine.result.cpu()
    verified = verified and (int(r[0]), int(r[1])) == (exp_s, exp_c)
    ms = max_over_ranks(start.elapsed_time(end), world) / K
    value = world * (nb + npr) / (ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    kb = tb // 2
    pipe_bytes = (nb + npr) * (kb + len(bits) * 2 * tb + tb)
    e2e = None
    if not a.no_e2e and a.e2e_steps > 0:
        host = [torch.empty(x.numel(), dtype=dt, pin_memory=True) for x in (rk, rp, sk, sp)]
        for h, d in zip(host, (rk, rp, sk, sp)):
            h.copy_(d)
        del rk, rp, sk, sp
        torch.cuda.empty_cache()
        engine.run_host(*host)
        t_e2e = []
        for _ in range(a.e2e_steps):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            s, c = engine.run_host(*host)
            t1.record(stream)
            torch.cuda.synchronize()
            verified = verified and (s, c) == (exp_s, exp_c)
            t_e2e.append(t0.elapsed_time(t1))
        e2e_ms = max_over_ranks(statistics.mean(t_e2e), world)
        e2e = {"value": world * (nb + npr) / (e2e_ms / 1e3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 2 * (nb + npr) * kb, "d2h_bytes_per_step": 16,
               "ms_per_step": e2e_ms,
               "path": "fi_radix_join_engine_run_host_%s (pinned host columns)"
                       % ("int32" if tb == 8 else "int64")}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": K, "warmup": a.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "int32" if tb == 8 else "int64",
                "data": "synthetic %s data set (seeded permutation PK with %d%% "
                        "selectivity, uniform FK, payload = key)" % (name, a.selectivity),
                "config": {"workload": "radix_join_%s_%s_sel%d" % (
                               a.data_set if name != "Custom" else "%dMx%dM_%sbits_zipf%.1f" % (
                                   nb >> 20, npr >> 20, "+".join(str(b) for b in bits), a.zipf),
                               "int32" if tb == 8 else "int64", a.selectivity),
                           "build_tuples": nb, "probe_tuples": npr,
                           "radix_bits": list(bits), "hashing_scheme": "chaining",
                           "join_block": plan["join_block"],
                           "l2_flush": "none: inputs larger than L2" if (nb + npr) * tb > 2**27
                                       else "none: inputs smaller than L2",
                           "parallelism": "replicas" if world > 1 else "single"},
                "pipeline_roofline": {"algorithmic_bytes_per_step": pipe_bytes,
                                      "achieved_gb_per_s": pipe_bytes / (ms / 1e3) / 1e9,
                                      "frac_of_peak": pipe_bytes / (ms / 1e3) / 1e9 / peak,
                                      "peak": peak, "peak_source": peak_kind},
                "e2e": e2e, "gpu_launches": engine.last_launches() * K,
                "clocks": clk.summary(), "matches": exp_c,
                "verified": bool(verified)}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_nopart(a):
    """No-partitioning hash join (CudaHashJoin build + probe_sum over a
    device hash table) on a named data set, Blanas by default: the
    comparison point for small build sides.  A step re-initialises the table
    (the reference allocates a fresh one per join), builds and probes.  The
    table holds 2^floor(log2(2|R|)) entries for linear probing (the
    reference's load factor 2) and |R|+1 for perfect hashing (keys 1..|R|)."""
    import torch
    import fi_sqlops as fi
    world, rank, local = dist_setup(a.gpus)
    name, paper_tb = DATASETS[a.data_set]
    tb = a.tuple_bytes or paper_tb
    dt = torch.int32 if tb == 8 else torch.int64
    seed = a.seed + 1000 * rank
    rk, rp, sk, sp = fi.gen_dataset(getattr(fi.Dataset, name), dt,
                                    selectivity=a.selectivity, seed=seed)
    nb, npr = rk.numel(), sk.numel()
    kept = fi.null_keys(sk.clone(), a.selectivity, seed + 7) != -1
    exp_s = int(sp.to(torch.int64)[kept].sum().item())
    del kept
    perfect = a.ht_scheme == "perfect"
    scheme = fi.HashingScheme.Perfect if perfect else fi.HashingScheme.LinearProbing
    # the kernels mask with 2^floor(log2(size)) (as the reference's do), so
    # the table is a power of two at most half full
    size = nb + 1 if perfect else 1 << (2 * nb - 1).bit_length()
    g, blk = [int(x) for x in a.ht_dim.split(",")]
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    grid = g or sms * (2048 // blk)
    ht = fi.HashTable(size, dt)
    hj = fi.CudaHashJoin(scheme, ht, (grid, blk), (grid, blk),
                         is_selective=a.selectivity < 100)
    hj.set_probe_grouping(a.probe_grouping == "on")
    hj.set_build_grouping(a.build_grouping == "on")
    res = torch.zeros(grid * blk, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    init = getattr(fi.lib(), "fi_hash_table_init_" + ("int32" if tb == 8 else "int64"))

    def step(evs=None):
        if evs: evs[0].record(stream)
        fi._check(init(fi._ptr(ht.mem), fi.C.c_uint64(ht.mem.shape[0]), fi._stream(None)))
        hj.build(rk, rp)
        if evs: evs[1].record(stream)
        hj.probe_sum(sk, sp, res)
        if evs: evs[2].record(stream)

    verified = True
    for _ in range(max(a.warmup, 1)):
        res.zero_()
        step()
        verified = verified and int(res.sum().item()) == exp_s
    K = a.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    res.zero_()
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        for k in range(K):
            step(ev[k])
        torch.cuda.synchronize()
        barrier(world)
    tot = int(res.sum().item())
    verified = verified and tot == (exp_s * K + (1 << 63)) % (1 << 64) - (1 << 63)
    build_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    probe_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    ms = max_over_ranks(build_ms + probe_ms, world)
    value = world * (nb + npr) / (ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    # algorithmic bytes: table init (one entry per slot), build (read a tuple,
    # write an entry), probe (read a tuple, read an entry)
    build_bytes = size * tb + nb * 2 * tb
    probe_bytes = npr * 2 * tb
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        cpu = nopart_cpu_baseline(rk, rp, sk, sp, size, perfect)
    if rank == 0:
        line = {"metric": "no-partitioning join G tuples/s", "value": value,
                "unit": UNIT, "n_gpus": world, "steps": K, "warmup": a.warmup,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int32" if tb == 8 else "int64",
                "data": "synthetic %s data set (seeded permutation PK, uniform FK, "
                        "payload = key)" % name,
                "config": {"workload": "nopart_join_%s_%s_%s" % (
                               a.data_set, "int32" if tb == 8 else "int64", a.ht_scheme),
                           "build_tuples": nb, "probe_tuples": npr,
                           "hash_table_entries": size, "grid": grid, "block": blk,
                           "probe_grouping": a.probe_grouping,
                           "build_grouping": a.build_grouping,
                           "l2_flush": "none: probe input larger than L2"},
                "phases": {"init_build": {"ms": build_ms,
                                          "gb_per_s": build_bytes / (build_ms / 1e3) / 1e9},
                           "probe": {"ms": probe_ms,
                                     "gb_per_s": probe_bytes / (probe_ms / 1e3) / 1e9}},
                "roofline": {"bound": "hbm", "kernel": "probe",
                             "achieved": probe_bytes / (probe_ms / 1e3) / 1e9,
                             "peak": peak, "unit": "GB/s",
                             "frac": probe_bytes / (probe_ms / 1e3) / 1e9 / peak,
                             "peak_source": peak_kind, "traffic": None},
                # the same probe against the DRAM-sector bound: each table
                # access moves at least one 32-byte sector, plus the probe
                # tuple streamed; and as random sectors per second
                "sector_roofline": {
                    "bytes_per_probe": 32 + 2 * tb,
                    "achieved_gb_per_s": npr * (32 + 2 * tb) / (probe_ms / 1e3) / 1e9,
                    "frac": npr * (32 + 2 * tb) / (probe_ms / 1e3) / 1e9 / peak,
                    "probes_per_s": npr / (probe_ms / 1e3)},
                "cpu_baseline": cpu,
                "clocks": clk.summary(), "verified": bool(verified)}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def nopart_cpu_baseline(rk, rp, sk, sp, size, perfect):
    """The reference's own CPU no-partitioning join (cpu_ht_build_* +
    cpu_ht_probe_aggregate_*, compiled from its sources; single-threaded
    as the reference's kernels are) on the whole build side and the first
    eighth of the probe side, with the same table size."""
    import oracle as O
    npr = max(1, sk.numel() // 8)
    r, p = rk.cpu().numpy(), rp.cpu().numpy()
    s, q = sk[:npr].cpu().numpy(), sp[:npr].cpu().numpy()
    kind = "reference" if O.ref_available() else "port"
    if perfect:  # the perfect kernels index the table with the key unchecked:
        # null build keys need the selective build, probe keys lie in 1..|R|
        sel = bool((r == -1).any())
        f = O.ref_ht_perfect_sum if kind == "reference" else O.ht_perfect_sum
        fn = lambda *x: f(*x, selective=sel)
    else:
        fn = O.ref_ht_linearprobing_sum if kind == "reference" else O.ht_linearprobing_sum
    t0 = time.perf_counter()
    fn(r, p, s, q, size)
    sec = time.perf_counter() - t0
    return {"value": (len(r) + npr) / sec / 1e9, "unit": UNIT, "cores": 1,
            "kind": kind,
            "sample": "build all %d tuples, probe the first %d (1/8) of the same "
                      "data, %d-entry %s table; one run" % (
                          len(r), npr, size, "perfect" if perfect else "linear-probing"),
            "seconds": sec}


def run_exchange(a):
    """The fused radix exchange kernel (partition + send into the receivers'
    columns) on one GPU: one sender's 2^exchange_log2n int64 tuples go to
    --exchange-ranks receivers whose receive columns are local buffers (on
    several GPUs they are peer pointers and all but 1/W of the stores cross
    NVLink).  A step = the destination histogram + the fused scatter.
    Algorithmic bytes: key read (histogram) + tuple read + tuple write = 40
    B/tuple; the scatter kernel alone 32 B/tuple."""
    import torch
    import fi_sqlops as fi
    import distributed as D
    world, rank, local = dist_setup(a.gpus)
    n = 1 << a.exchange_log2n
    W = a.exchange_ranks
    g = D.exchange_bits(W)
    shift = 18  # above 9+9 local join bits
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    pays = torch.empty(n, dtype=torch.int64, device="cuda")
    fi.gen_uniform_foreign_keys(keys, 1 << 40, a.seed + rank)
    pays.copy_(keys)
    counts = fi.exchange_histogram(keys, shift, g)
    cnt = counts.cpu().tolist()
    cols = [(torch.empty(max(c, 1), dtype=torch.int64, device="cuda"),
             torch.empty(max(c, 1), dtype=torch.int64, device="cuda")) for c in cnt]
    dests = [(k.data_ptr(), p.data_ptr(), 0, c) for (k, p), c in zip(cols, cnt)]
    cursors = torch.empty(W, dtype=torch.int64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def step(evs=None):
        if evs: evs[0].record(stream)
        fi.exchange_histogram(keys, shift, g, counts)
        if evs: evs[1].record(stream)
        fi.exchange_scatter(keys, pays, shift, g, dests, cursors, status)
        if evs: evs[2].record(stream)

    for _ in range(max(a.warmup, 3)):
        step()
    K = a.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        for k in range(K):
            step(ev[k])
        torch.cuda.synchronize()
        barrier(world)
    # every receiver holds its tuples: counts, and key sums per destination
    d_of = (keys >> shift) & (W - 1)
    exp_sum = torch.zeros(W, dtype=torch.int64, device="cuda").index_add_(0, d_of, keys)
    verified = int(status.item()) == 0 and cursors.cpu().tolist() == cnt
    for d, (k, p) in enumerate(cols):
        c = cnt[d]
        verified = verified and int(k[:c].sum().item()) == int(exp_sum[d].item()) \
            and bool(torch.equal(k[:c], p[:c]))
    hist_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    scat_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    ms = max_over_ranks(hist_ms + scat_ms, world)
    peak, peak_kind = load_peaks()
    step_bytes, scat_bytes = n * 40, n * 32
    nvlink_gbs = 770.0
    if rank == 0:
        line = {"metric": "radix exchange G tuples/s", "value": world * n / (ms / 1e3) / 1e9,
                "unit": UNIT, "n_gpus": world, "steps": K, "warmup": max(a.warmup, 3),
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int64",
                "data": "synthetic (seeded uniform keys in [1, 2^40], payload = key)",
                "config": {"workload": "radix_exchange_%dM_int64_%d_receivers_local" % (
                               n >> 20, W),
                           "tuples": n, "receivers": W, "exchange_bits": [shift, shift + g],
                           "l2_flush": "none: inputs (%.1f GB) larger than L2" % (n * 16 / 1e9)},
                "phases": {"histogram": {"ms": hist_ms,
                                         "gb_per_s": n * 8 / (hist_ms / 1e3) / 1e9},
                           "scatter": {"ms": scat_ms,
                                       "gb_per_s": scat_bytes / (scat_ms / 1e3) / 1e9}},
                "roofline": {"bound": "hbm", "kernel": "exchange_scatter",
                             "achieved": scat_bytes / (scat_ms / 1e3) / 1e9, "peak": peak,
                             "unit": "GB/s",
                             "frac": scat_bytes / (scat_ms / 1e3) / 1e9 / peak,
                             "peak_source": peak_kind, "traffic": None},
                "pipeline_roofline": {"algorithmic_bytes_per_step": step_bytes,
                                      "achieved_gb_per_s": step_bytes / (ms / 1e3) / 1e9,
                                      "frac_of_peak": step_bytes / (ms / 1e3) / 1e9 / peak},
                "nvlink_bound_ms_on_%d_gpus" % W: n * 16 * (W - 1) / W / (nvlink_gbs * 1e9) * 1e3,
                "gpu_launches": 2 * K,
                "clocks": clk.summary(), "verified": bool(verified)}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_hybrid(a):
    """Hybrid join (the reference's cpu_partitioned_radix_join): host
    columns, first pass on all host threads, second pass and join on the GPU.
    Wall-clock time per join (the CPU pass dominates); G tuples/s."""
    import torch
    import fi_sqlops as fi
    world, rank, local = dist_setup(a.gpus)
    n = 1 << a.hybrid_log2n
    seed = a.seed + 1000 * rank
    host = []
    for gen in ("pk", "fk"):
        d = torch.empty(n, dtype=torch.int64, device="cuda")
        if gen == "pk":
            fi.gen_primary_keys(d, seed, base=1)
        else:
            fi.gen_uniform_foreign_keys(d, n, seed + 1, base=1)
            expected_sum = int(d.sum().item())
        for _ in range(2):
            h = torch.empty(n, dtype=torch.int64, pin_memory=True)
            h.copy_(d)
            host.append(h)
        del d
    torch.cuda.empty_cache()
    threads = os.cpu_count() or 1
    engine = fi.RadixJoinEngine(n, n, torch.int64, fi.RadixBits(9, 9),
                                fi.HashingScheme.BucketChaining)
    verified = True
    for _ in range(max(a.warmup, 1)):
        s, c = engine.run_hybrid(*host, threads=threads)
        verified = verified and (c == n and s == expected_sum)
    wall = []
    with ClockSampler(local) as clk:
        for _ in range(a.steps):
            barrier(world)
            t0 = time.perf_counter()
            s, c = engine.run_hybrid(*host, threads=threads)
            wall.append(time.perf_counter() - t0)
            verified = verified and (c == n and s == expected_sum)
    ms = max_over_ranks(statistics.mean(wall) * 1e3, world)
    if rank == 0:
        line = {"metric": "hybrid radix join G tuples/s",
                "value": world * 2 * n / (ms / 1e3) / 1e9, "unit": UNIT,
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int64",
                "data": "synthetic (seeded permutation PK, uniform FK, payload = key) "
                        "in pinned host memory",
                "config": {"workload": "hybrid_radix_join_%dMx%dM_int64_9+9bits"
                                       % (n >> 20, n >> 20),
                           "host_threads": threads, "timing": "wall clock per join",
                           "parallelism": "replicas" if world > 1 else "single"},
                "clocks": clk.summary(), "verified": bool(verified)}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "partition":
        run_partition_sweep(a)
    elif a.workload == "ooc":
        run_ooc(a)
    elif a.workload == "serve":
        run_serve(a)
    elif a.workload == "dataset":
        run_dataset(a)
    elif a.workload == "nopart":
        run_nopart(a)
    elif a.workload == "hybrid":
        run_hybrid(a)
    elif a.workload == "exchange":
        run_exchange(a)
    elif a.workload == "refkernels":
        run_refkernels(a)
    elif a.workload == "sharded" or (int(os.environ.get("WORLD_SIZE", "1")) > 1
                                     and not a.replicas):
        run_sharded(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
