"""Benchmark of the bulk hash-container hot path on B200.

Headline workload (one step = one bulk Find of 2^27 keys):
    StaticMap<int64_t,int64_t>, requested capacity 2^28 slots (268,728,155 after
    the prime rule, 4.3 GB of 16-byte pairs), DoubleHashing<xxhash_32>, bucket 5,
    sentinels -1; filled by InsertAndFind (first-wins) to load factor 0.5 with
    uniform unique int64 keys plus 10% duplicate keys in the insert stream;
    queried with 2^27 keys at a 50% hit rate.  Other hit rates, a Zipf(1.1)
    stream, load factor 0.8 and Insert are reported under "extra".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line.  --impl reference times the reference algorithm's CPU
restatement (the reference has no CPU implementation of its own) on the host
cores, same metric and workload, on a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "ops-collections_b200"))

REQ_CAPACITY = 1 << 28
N_QUERIES = 1 << 27
LOAD_FACTOR = 0.5
DUP_FRACTION = 0.10
SEED = 2026
METRIC = "StaticMap Find/Insert Gkeys/s @LF0.5 (% HBM roofline); batched keys/s; p50/p99 lat"
UNIT = "Gkeys/s"
WORKLOAD = ("StaticMap<int64,int64> single table, capacity 2^28 requested (268,728,155 slots, 4.3 GB), "
            "DoubleHashing<xxhash_32> bucket 5, filled by InsertAndFind to LF 0.5 (10% duplicate inserts); "
            "bulk Find of 2^27 int64 queries at 50% hits")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# seeded synthetic inputs (generated on the device; the same arithmetic on the
# host for the CPU arm)
# ---------------------------------------------------------------------------

M64 = (1 << 64) - 1


def _to_i64(u: int) -> int:
    return u - (1 << 64) if u >= (1 << 63) else u


def mix64_torch(x):
    """SplitMix64 finalizer, a bijection on 64-bit words, over int64 tensors."""
    import torch

    def srl(v, k):  # logical shift right on int64
        return (v >> k) & ((1 << (64 - k)) - 1)

    x = x + _to_i64(0x9E3779B97F4A7C15)
    x = (x ^ srl(x, 30)) * _to_i64(0xBF58476D1CE4E5B9)
    x = (x ^ srl(x, 27)) * _to_i64(0x94D049BB133111EB)
    return x ^ srl(x, 31)


def mix64_np(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return x.view(np.int64)


def counters(lo, n, backend):
    if backend == "torch":
        import torch
        return torch.arange(lo, lo + n, dtype=torch.int64, device="cuda")
    return np.arange(lo, lo + n, dtype=np.int64)


KEY_STREAM, MISS_STREAM, VALUE_STREAM = 0, 1 << 40, 2 << 40


def workload_sizes(capacity: int, lf: float):
    unique = int(math.floor(lf * capacity))
    dups = int(round(unique * DUP_FRACTION / (1.0 - DUP_FRACTION)))
    return unique, dups


def make_insert_stream(unique, dups, backend):
    """Unique keys (bijective mix of a counter: distinct, uniform, never -1 in practice)
    followed by duplicates of earlier keys, shuffled; values are another mixed stream."""
    if backend == "torch":
        import torch
        g = torch.Generator(device="cuda").manual_seed(SEED)
        keys = mix64_torch(counters(KEY_STREAM, unique, "torch"))
        dup_idx = torch.randint(0, unique, (dups,), generator=g, device="cuda")
        stream = torch.cat([keys, keys[dup_idx]])
        perm = torch.randperm(stream.numel(), generator=g, device="cuda")
        stream = stream[perm]
        vals = mix64_torch(counters(VALUE_STREAM, stream.numel(), "torch"))
        assert not bool((keys == -1).any())
        return keys, stream, vals
    rng = np.random.default_rng(SEED)
    keys = mix64_np(counters(KEY_STREAM, unique, "np"))
    dup_idx = rng.integers(0, unique, size=dups)
    stream = np.concatenate([keys, keys[dup_idx]])
    rng.shuffle(stream)
    vals = mix64_np(counters(VALUE_STREAM, len(stream), "np"))
    return keys, stream, vals


def make_queries(keys, n, hit_rate, backend, zipf_s=None):
    """n queries: hit_rate of them drawn from the inserted keys, the rest from a
    disjoint stream; shuffled.  With zipf_s, all are hits with Zipf-ranked popularity."""
    if backend == "torch":
        import torch
        g = torch.Generator(device="cuda").manual_seed(SEED + 1)
        u = keys.numel()
        if zipf_s is not None:
            r = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
            a = 1.0 - zipf_s
            rank = torch.floor((1.0 + r * (float(u) ** a - 1.0)) ** (1.0 / a)).to(torch.int64) - 1
            rank = rank.clamp_(0, u - 1)
            idx = (rank * 2654435761 + 12345) % u  # seeded permutation: rank -> key
            return keys[idx]
        nh = int(round(n * hit_rate))
        hits = keys[torch.randint(0, u, (nh,), generator=g, device="cuda")]
        miss = mix64_torch(counters(MISS_STREAM, n - nh, "torch"))
        q = torch.cat([hits, miss])
        return q[torch.randperm(n, generator=g, device="cuda")]
    rng = np.random.default_rng(SEED + 1)
    u = len(keys)
    nh = int(round(n * hit_rate))
    hits = keys[rng.integers(0, u, size=nh)]
    miss = mix64_np(counters(MISS_STREAM, n - nh, "np"))
    q = np.concatenate([hits, miss])
    rng.shuffle(q)
    return q


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def parse_shape(s: str):
    """'LxK', 'LxKs', 'LxKw', 'LxKd' or 'bulk': L lanes per key, K keys in flight
    per lane group; s = segmented windows, w = keys staged per warp, d = per-warp
    staging with deferred continuations, bulk = one bulk copy per bucket window."""
    if s == "bulk":
        return 1, 1, False, True, False, False
    warp = s.endswith("w")
    seg = s.endswith("s")
    defer = s.endswith("d")
    lanes, items = (int(x) for x in s.rstrip("swd").split("x"))
    return lanes, items, seg, False, warp, defer


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per Find launch from the committed ncu summary, if present."""
    p = os.path.join(REPO, "profiles", "find_map88_lf05_ncu.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_full_launch:"):
            return float(line.split(":")[1])
    return None


def dist_setup(gpus):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The largest of every rank's x (the job's time is its slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def run_gpu(args):
    import torch
    import b2co
    rank, world, local = dist_setup(args.gpus)
    stream = torch.cuda.current_stream()
    peak, peak_kind = peaks()

    t = b2co.StaticMap(REQ_CAPACITY, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64, bucket_size=5,
                       probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)
    cap = t.Capacity()
    unique, dups = workload_sizes(cap, LOAD_FACTOR)
    keys, stream_keys, vals = make_insert_stream(unique, dups, "torch")
    pairs = b2co.pack_pairs(stream_keys, vals)
    found = torch.empty(stream_keys.numel(), dtype=torch.int64, device="cuda")
    inserted = torch.empty(stream_keys.numel(), dtype=torch.uint8, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # scratch for the largest fill this run times (LF 0.8), so no timed region allocates
    t.ReserveInsertAndFind(sum(workload_sizes(cap, 0.8)))
    torch.cuda.synchronize()
    e0.record(stream)
    t.InsertAndFindAsync(pairs, found, inserted, mode=b2co.IAF_FIRST_WINS)
    e1.record(stream)
    torch.cuda.synchronize()
    fill_ms = e0.elapsed_time(e1)
    n_inserted = int(inserted.sum().item())
    assert n_inserted == unique, (n_inserted, unique)
    # the fill's inputs and outputs, kept on the host for the full-size parity check after timing
    fill_host = None
    if rank == 0 and not args.no_host:
        fill_host = (stream_keys.cpu().numpy(), vals.cpu().numpy(), found.cpu().numpy(), inserted.cpu().numpy())
    del found, inserted, pairs
    log(f"[bench] capacity {cap}, unique {unique}, stream {stream_keys.numel()}, fill {fill_ms:.1f} ms")
    del stream_keys, vals

    q = make_queries(keys, N_QUERIES, 0.5, "torch")
    out = torch.empty(N_QUERIES, dtype=torch.int64, device="cuda")
    if args.l2_fetch:
        import b2co
        b2co.set_l2_fetch_granularity(args.l2_fetch)
    if args.sweep:
        sweep = {}
        shapes = args.sweep_shapes.split(",") if args.sweep_shapes else [
            "4x2d", "2x2d", "4x1d", "8x2d", "2x2w", "4x2w", "2x2", "4x2", "2x2s"]
        for shape in shapes:
            t.set_find_shape(*parse_shape(shape))
            for _ in range(3):
                t.FindAsync(q, out)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(10):
                t.FindAsync(q, out)
            e1.record(stream)
            torch.cuda.synchronize()
            sweep[shape] = round(N_QUERIES * 10 / e0.elapsed_time(e1) / 1e6, 3)
            log(f"[sweep] shape {shape}: {sweep[shape]} Gkeys/s")
        t.set_find_shape(0, 0)
    if args.shape:
        t.set_find_shape(*parse_shape(args.shape))

    for _ in range(args.warmup):
        t.FindAsync(q, out)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            t.FindAsync(q, out)
        e1.record(stream)
        torch.cuda.synchronize()
    local_ms = e0.elapsed_time(e1)
    barrier(world)
    total_ms = max_over_ranks(local_ms, world)
    ms_per_step = total_ms / args.steps
    value = world * N_QUERIES * args.steps / (total_ms / 1e3) / 1e9

    # exact probe-window count of the timed queries and parity on a sample, by
    # the CPU oracle over a host copy of the very same table
    extra = {}
    if args.sweep:
        extra["find_shape_sweep_gkeys"] = sweep
    windows_mean, cpu = None, None
    if rank == 0 and not args.no_host:
        windows_mean, cpu, parity = host_side_checks(t, q, out, args, fill_host)
        extra["parity_full_size"] = parity
        del fill_host
    bytes_per_query = 8 + 8 + 80 * (windows_mean if windows_mean else 1.0)
    achieved = N_QUERIES * bytes_per_query / (ms_per_step / 1e3) / 1e9
    traffic = profiled_traffic()
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "peak_source": peak_kind, "bytes_per_query": round(bytes_per_query, 3),
                "windows_per_query": windows_mean,
                "one_window_bound_gbs": round(N_QUERIES * 96 / (ms_per_step / 1e3) / 1e9, 1)}
    roofline.update(window_gather_ceiling(t, stream, value, windows_mean))

    e2e = None if args.no_e2e else measure_e2e(t, q, out, stream, world, args)

    if not args.quick:
        extra.update(extra_measurements(t, keys, q, out, stream, args))

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "capacity": cap, "unique_keys": unique, "insert_stream": unique + dups,
                       "queries": N_QUERIES, "hit_rate": 0.5, "bucket_size": 5, "probing": "DoubleHashing<xxhash_32>",
                       "l2": "inputs larger than L2 (4.3 GB table + 1 GB keys)", "parallelism": f"replicas x{world}",
                       "find_shape": args.shape or "default (4x2d: 4 lanes per window, 2 windows in flight, "
                                     "per-warp key staging, deferred continuations)"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps,
            "clocks": clk.summary(), "fill_ms": round(fill_ms, 2), "extra": extra,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def measure_e2e(t, q, out, stream, world, args):
    """Find through the C ABI with pinned HOST buffers: copy-in and copy-out
    of every step are inside the timed region."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hq = q.cpu().pin_memory()
    ho = torch.empty(N_QUERIES, dtype=torch.int64).pin_memory()
    t.FindHost(hq.numpy(), ho.numpy())
    torch.cuda.synchronize()
    e2e_steps = max(3, min(args.steps, 10))
    e0.record(stream)
    for _ in range(e2e_steps):
        t.FindHost(hq.numpy(), ho.numpy())
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world) / e2e_steps
    assert torch.equal(ho, out.cpu()), "host-buffer Find differs from device Find"
    floor_ms = pcie_floor_ms(hq, ho, q, out)
    return {"value": round(world * N_QUERIES / (e2e_ms / 1e3) / 1e9, 4), "unit": UNIT,
            "h2d_bytes_per_step": N_QUERIES * 8, "d2h_bytes_per_step": N_QUERIES * 8,
            "ms_per_step": round(e2e_ms, 3), "gpu_launches_per_step": host_find_chunks(N_QUERIES),
            "pcie_floor_ms": round(floor_ms, 3), "frac_of_pcie_floor": round(floor_ms / e2e_ms, 4)}


def host_find_chunks(n, full=1 << 22):
    """Chunks (one Find launch each) of the host-buffer Find of n keys: batches
    of 16 Mi keys or more ramp up with 1 and 2 Mi chunks and down with 2 and 1 Mi."""
    q, h, off, count = full // 4, full // 2, 0, 0
    while off < n:
        left = n - off
        if n < 4 * full:
            m = min(left, full)
        elif off == 0:
            m = q
        elif off == q:
            m = h
        elif left <= q:
            m = left
        elif left <= q + h:
            m = left - q
        elif left <= q + h + full:
            m = left - q - h
        else:
            m = full
        off, count = off + m, count + 1
    return count


def pcie_floor_ms(hq, ho, q, out):
    """Time of the step's bare copies alone: the keys in and the results out at
    once on two streams, the same pinned buffers and byte counts as one e2e step.
    No lookup can finish a step faster; measured after the timed e2e region."""
    import torch
    dq, dout = torch.empty_like(q), torch.empty_like(out)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def both():
        cur = torch.cuda.current_stream()
        s1.wait_stream(cur)
        s2.wait_stream(cur)
        with torch.cuda.stream(s1):
            dq.copy_(hq, non_blocking=True)
        with torch.cuda.stream(s2):
            ho.copy_(dout, non_blocking=True)
        cur.wait_stream(s1)
        cur.wait_stream(s2)

    both()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        both()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 5


def window_gather_ceiling(t, stream, find_gkeys, windows_mean):
    """The random bucket-window read rate of this GPU over the very same table:
    bare reads of whole windows (80 bytes for 16-byte slots, 40 for 8-byte) at
    random bucket starts, none of a lookup's other work (key stream, hashing,
    outputs, second windows).  Random windows move whole DRAM fill units, so
    this rate, not the copy peak, is what Find can approach; timed after (never
    inside) the Find region."""
    import torch
    n = 1 << 27
    for i in range(3):
        t.window_gather(n, seed=11 + i, stream=stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(10):
        t.window_gather(n, seed=101 + i, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    gwin = n * 10 / (e0.elapsed_time(e1) / 1e3) / 1e9
    out = {"window_gather_ceiling_gwin": round(gwin, 3)}
    if windows_mean:
        out["find_windows_vs_ceiling"] = round(find_gkeys * windows_mean / gwin, 4)
    return out


def host_side_checks(t, q, out, args, fill_host):
    """Exact parity of the timed workload at full size, the probe windows per
    query (exact, oracle over the device table's bytes) and the CPU baseline
    on the host cores.  Parity: the oracle refills the table sequentially from
    the same insert stream (the first-wins golden) and must give every found
    value and inserted flag of the device fill and the same stored pair set;
    the last timed Find's 2^27 outputs must equal the oracle's Find on its own
    table.  All of it runs after the timed region."""
    import oracle
    import torch
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    d = oracle.Table(np.int64, np.int64, t.Capacity(), 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, -1, -1)
    d.load_slots(t.dump_slots())
    o = oracle.Table(np.int64, np.int64, t.Capacity(), 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, -1, -1)
    s_keys, s_vals, dev_found, dev_ins = fill_host
    exp_found, exp_ins = o.insert_and_find(s_keys, s_vals)
    t1 = time.perf_counter()
    same, n_o, n_d, mism = o.same_pairs(d, threads)
    qh = q.cpu().numpy()
    exp = o.find_parallel(qh, threads)
    parity = {"fill_inputs": int(len(s_keys)),
              "fill_found_and_flags_identical": bool(np.array_equal(exp_found, dev_found)
                                                     and np.array_equal(exp_ins, dev_ins)),
              "stored_pairs_identical": bool(same), "stored_pairs": int(n_d),
              "find_queries": int(len(qh)), "find_identical": bool(np.array_equal(exp, out.cpu().numpy())),
              "oracle_fill_s": round(t1 - t0, 1)}
    log(f"[bench] full-size parity {parity} in {time.perf_counter() - t0:.1f} s")
    del o, exp_found, exp_ins, exp
    sample = 1 << 22
    _, win = d.find(qh[:sample])
    windows_mean = float(win.mean())
    o = d
    cpu = None
    if not args.no_cpu:
        threads = os.cpu_count() or 1
        qa = q.cpu().numpy()
        done, t0 = 0, time.perf_counter()
        chunk = 1 << 22
        while done < len(qa) and time.perf_counter() - t0 < args.cpu_seconds:
            o.find_parallel(qa[done:done + chunk], threads)
            done += chunk
        el = time.perf_counter() - t0
        st_n = 1 << 21  # single thread: the sequential oracle Find on a 2 Mi-query slice
        t1 = time.perf_counter()
        o.find(qa[:st_n])
        st_el = time.perf_counter() - t1
        cpu = {"value": round(done / el / 1e9, 5), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{done} of the 2^27 timed queries (50% hits) over a host copy of the same LF0.5 table, "
                         f"oracle Find on {threads} OpenMP threads, {el:.1f} s",
               "single_thread_value": round(st_n / st_el / 1e9, 5), "cpu_model": cpu_model()}
    return windows_mean, cpu, parity


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def extra_measurements(t, keys, q50, out, stream, args):
    """Secondary numbers: other hit rates, Zipf, contains, insert, LF 0.8."""
    import torch
    import b2co
    res = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    for hr in (0.0, 1.0):
        qq = make_queries(keys, N_QUERIES, hr, "torch")
        ms = timed(lambda: t.FindAsync(qq, out))
        res[f"find_hit{int(hr * 100)}_gkeys"] = round(N_QUERIES / ms / 1e6, 3)
        del qq
    qz = make_queries(keys, N_QUERIES, 1.0, "torch", zipf_s=1.1)
    ms = timed(lambda: t.FindAsync(qz, out))
    res["find_zipf1.1_gkeys"] = round(N_QUERIES / ms / 1e6, 3)
    del qz
    c = torch.empty(N_QUERIES, dtype=torch.uint8, device="cuda")
    ms = timed(lambda: t.ContainsAsync(q50, c))
    res["contains_hit50_gkeys"] = round(N_QUERIES / ms / 1e6, 3)
    del c
    # Insert: unique pairs into a cleared table (clear not timed)
    cap = t.Capacity()
    unique, _ = workload_sizes(cap, LOAD_FACTOR)
    pairs = b2co.pack_pairs(keys, mix64_torch(counters(VALUE_STREAM, unique, "torch")))
    tot = 0.0
    for _ in range(3):
        t.Clear()
        torch.cuda.synchronize()
        e0.record(stream)
        t.InsertAsync(pairs)
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    res["insert_lf05_gkeys"] = round(unique / (tot / 3) / 1e6, 3)
    # LF 0.8: refill, Find at 50% hits
    u8, d8 = workload_sizes(cap, 0.8)
    t.Clear()
    k8, s8, v8 = make_insert_stream(u8, d8, "torch")
    p8 = b2co.pack_pairs(s8, v8)
    f8 = torch.empty(s8.numel(), dtype=torch.int64, device="cuda")
    i8 = torch.empty(s8.numel(), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    e0.record(stream)
    t.InsertAndFindAsync(p8, f8, i8, mode=b2co.IAF_FIRST_WINS)
    e1.record(stream)
    torch.cuda.synchronize()
    res["insert_and_find_fill_lf08_gkeys"] = round(s8.numel() / e0.elapsed_time(e1) / 1e6, 3)
    del p8, f8, i8, s8, v8
    q8 = make_queries(k8, N_QUERIES, 0.5, "torch")
    ms = timed(lambda: t.FindAsync(q8, out))
    res["find_lf08_hit50_gkeys"] = round(N_QUERIES / ms / 1e6, 3)
    del q8
    res.update(small_map_measurements(stream))
    res.update(dynamic_map_measurements(stream))
    res.update(bloom_hll_measurements(stream))
    res.update(batched_measurements(stream))
    res.update(multi_measurements(stream))
    res.update(roaring_measurements(stream))
    res.update(served_measurements(stream))
    return res


def fill_measurements(stream, reps=3):
    """The headline table's fill on its own: StaticMap<int64,int64>, 2^28 slots
    requested, first-wins InsertAndFind of the benchmark's insert streams to
    load factor 0.5 and 0.8 (10% duplicate keys), `reps` times each into a
    cleared table (clears not timed, scratch reserved beforehand, so no timed
    region allocates); every run's inserted count is checked."""
    import b2co
    import torch
    t = b2co.StaticMap(REQ_CAPACITY, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64, bucket_size=5,
                       probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)
    cap = t.Capacity()
    t.ReserveInsertAndFind(sum(workload_sizes(cap, 0.8)))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = {}
    for lf in (0.5, 0.8):
        unique, dups = workload_sizes(cap, lf)
        _, stream_keys, vals = make_insert_stream(unique, dups, "torch")
        pairs = b2co.pack_pairs(stream_keys, vals)
        del vals
        found = torch.empty(stream_keys.numel(), dtype=torch.int64, device="cuda")
        ins = torch.empty(stream_keys.numel(), dtype=torch.uint8, device="cuda")
        runs = []
        for _ in range(reps):
            t.ClearAsync(stream=stream)
            torch.cuda.synchronize()
            e0.record(stream)
            t.InsertAndFindAsync(pairs, found, ins, stream=stream, mode=b2co.IAF_FIRST_WINS)
            e1.record(stream)
            torch.cuda.synchronize()
            assert int(ins.sum().item()) == unique
            runs.append(e0.elapsed_time(e1))
        key = f"lf{int(lf * 10):02d}"
        res[f"fill_{key}_ms"] = [round(x, 3) for x in runs]
        res[f"fill_{key}_gkeys"] = round(stream_keys.numel() / min(runs) / 1e6, 3)
        res[f"fill_{key}_spread"] = round(max(runs) / min(runs) - 1.0, 4)
        del pairs, found, ins, stream_keys
    return res


INSERT_SHAPES = [(1, 1), (2, 1), (2, 2), (4, 1), (4, 2), (4, 4), (8, 2), (8, 4)]


def insert_measurements(stream, capacity_log2=28, reps=3, shapes=None):
    """The write side of the headline table on its own: StaticMap<int64,int64>,
    DoubleHashing<xxhash_32>, bucket 5, requested capacity 2^capacity_log2; a
    cleared table filled to LF 0.5 by Insert (unique keys), by InsertAndFind in
    race and in first-wins mode, then every pair upserted again by
    InsertOrAssign (all duplicates: payload overwrites).  Clears are not timed;
    each figure is the best of `reps`.  The insert stream of first-wins is
    checked: every key inserted once, every found payload its own."""
    import b2co
    import torch
    t = b2co.StaticMap(1 << capacity_log2, -1, -1, key_dtype=torch.int64, value_dtype=torch.int64, bucket_size=5,
                       probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)
    unique, _ = workload_sizes(t.Capacity(), LOAD_FACTOR)
    keys = mix64_torch(counters(KEY_STREAM, unique, "torch"))
    vals = mix64_torch(counters(VALUE_STREAM, unique, "torch"))
    pairs = b2co.pack_pairs(keys, vals)
    found = torch.empty(unique, dtype=torch.int64, device="cuda")
    ins = torch.empty(unique, dtype=torch.uint8, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t.ReserveInsertAndFind(unique)

    def best(fn, clear=True):
        out = []
        for _ in range(reps):
            if clear:
                t.ClearAsync(stream=stream)
            torch.cuda.synchronize()
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return min(out)

    res = {"insert_capacity": t.Capacity(), "insert_pairs": unique}
    ms = best(lambda: t.InsertAsync(pairs, stream=stream))
    res["insert_gkeys"] = round(unique / ms / 1e6, 3)
    ms = best(lambda: t.InsertAndFindAsync(pairs, found, ins, stream=stream, mode=b2co.IAF_RACE))
    res["insert_and_find_race_gkeys"] = round(unique / ms / 1e6, 3)
    ms = best(lambda: t.InsertAndFindAsync(pairs, found, ins, stream=stream, mode=b2co.IAF_FIRST_WINS))
    res["insert_and_find_first_wins_gkeys"] = round(unique / ms / 1e6, 3)
    res["first_wins_exact"] = bool(int(ins.sum().item()) == unique) and bool(torch.equal(found, vals))
    ms = best(lambda: t.InsertOrAssignAsync(pairs, stream=stream), clear=False)
    res["insert_or_assign_dup_gkeys"] = round(unique / ms / 1e6, 3)
    if shapes:  # Insert with every write-kernel shape (lanes per window x keys per lane group)
        sweep = {}
        for lanes, items in shapes:
            t.set_write_shape(lanes, items)
            sweep[f"{lanes}x{items}"] = round(unique / best(lambda: t.InsertAsync(pairs, stream=stream)) / 1e6, 3)
        t.set_write_shape(0, 0)
        res["insert_shape_sweep_gkeys"] = sweep
    del t
    return res


def dynamic_map_measurements(stream, log2n=26, batch_log2=22):
    """DynamicMap<int64,int64> (the reference's defaults: LinearProbing<murmurhash3_32>,
    bucket 5): created for 2^20 slots, then 2^log2n unique pairs inserted in
    batches of 2^batch_log2 -- the map adds a submap of twice the capacity
    whenever the load would pass 0.6, so the timed inserts include every growth
    step -- and Find / Contains of 2^log2n queries at 50% hits over all the
    submaps.  Hits must return their own values, misses the empty value."""
    import b2co
    import torch
    n, bs = 1 << log2n, 1 << batch_log2
    keys = mix64_torch(counters(11 << 40, n, "torch")) >> 1
    vals = mix64_torch(counters(12 << 40, n, "torch")) >> 1
    g = torch.Generator(device="cuda").manual_seed(SEED + 31)
    hit = torch.rand(n, generator=g, device="cuda") < 0.5
    pick = torch.randint(0, n, (n,), generator=g, device="cuda")
    q = torch.where(hit, keys[pick], mix64_torch(counters(13 << 40, n, "torch")) >> 1)
    exp = torch.where(hit, vals[pick], torch.full_like(vals, -1))
    pairs = b2co.pack_pairs(keys, vals)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m = b2co.DynamicMap(1 << 20, -1, -1, -2, key_dtype=torch.int64, value_dtype=torch.int64)
    torch.cuda.synchronize()
    e0.record(stream)
    inserted = 0
    for off in range(0, n, bs):
        inserted += m.Insert(pairs[off:off + bs], stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    insert_ms = e0.elapsed_time(e1)
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    m.Find(q, out, stream=stream)
    torch.cuda.synchronize()
    e0.record(stream)
    m.Find(q, out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    find_ms = e0.elapsed_time(e1)
    exact = bool(torch.equal(out, exp))
    flags = torch.empty(n, dtype=torch.uint8, device="cuda")
    e0.record(stream)
    m.Contains(q, flags, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    contains_ms = e0.elapsed_time(e1)
    exact = exact and bool(torch.equal(flags.bool(), hit))
    res = {"dmap_pairs": n, "dmap_inserted": inserted, "dmap_submaps": m.NumSubmaps(), "dmap_capacity": m.Capacity(),
           "dmap_insert_with_growth_gkeys": round(n / insert_ms / 1e6, 3),
           "dmap_find_gkeys": round(n / find_ms / 1e6, 3), "dmap_contains_gkeys": round(n / contains_ms / 1e6, 3),
           "dmap_results_exact": exact}
    del m
    return res


def small_map_measurements(stream, reps=200):
    """The small single-table workload: StaticMap<int32,int32>, DoubleHashing<xxhash_32>,
    bucket 5, requested capacity 2,097,152 (2,621,735 slots, 21 MB: it stays in the
    126 MB L2), 1,000,000 unique keys uniform in [0, 2^31-2] (seed 1), value 2*key+1,
    1,000,000 queries at 50% hits (misses drawn from the same range and rejected
    against the inserted set), shuffled.  L2-resident, so GB/s of algorithmic bytes
    (4 key + 4 value + 40 per bucket window) is reported, not an HBM fraction.  Each
    launch is short, so `reps` back-to-back launches are timed."""
    import b2co
    import torch
    rng = np.random.default_rng(1)
    n = 1_000_000
    draw = np.unique(rng.integers(0, 2**31 - 1, size=int(n * 1.05), dtype=np.int64))
    rng.shuffle(draw)
    keys = draw[:n].astype(np.int32)
    vals = (2 * keys.astype(np.int64) + 1).astype(np.int32)
    cand = rng.integers(0, 2**31 - 1, size=n, dtype=np.int64).astype(np.int32)
    miss = cand[~np.isin(cand, keys)][: n // 2]
    q = np.concatenate([keys[rng.integers(0, n, size=n // 2)], miss])
    rng.shuffle(q)
    exp = np.where(np.isin(q, keys), (2 * q.astype(np.int64) + 1).astype(np.int32), np.int32(-1))
    t = b2co.StaticMap(2_097_152, -1, -1, key_dtype=torch.int32, value_dtype=torch.int32, bucket_size=5,
                       probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)
    dk, dv, dq = (torch.from_numpy(a).cuda() for a in (keys, vals, q))
    pairs = b2co.pack_pairs(dk, dv)
    out = torch.empty(len(q), dtype=torch.int32, device="cuda")
    flags = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    insert_ms = 0.0
    for i in range(reps // 10 + 3):
        ev[0].record(stream)
        t.ClearAsync(stream=stream)
        ev[1].record(stream)
        t.InsertAsync(pairs, stream=stream)
        ev[2].record(stream)
        torch.cuda.synchronize()
        if i >= 3:
            insert_ms += ev[1].elapsed_time(ev[2])
    insert_ms /= reps // 10

    def timed(fn):
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(reps):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / reps

    find_ms = timed(lambda: t.FindAsync(dq, out, stream=stream))
    ok = bool(np.array_equal(out.cpu().numpy(), exp))
    contains_ms = timed(lambda: t.ContainsAsync(dq, flags, stream=stream))
    ok = ok and bool(np.array_equal(flags.cpu().numpy(), (exp != -1).astype(np.uint8)))
    res = {"small_map_capacity": t.Capacity(), "small_map_insert_gkeys": round(n / insert_ms / 1e6, 3),
           "small_map_find_gkeys": round(len(q) / find_ms / 1e6, 3),
           "small_map_find_gbs_1window": round(len(q) * 48 / find_ms / 1e6, 1),
           "small_map_contains_gkeys": round(len(q) / contains_ms / 1e6, 3),
           "small_map_find_us_per_launch": round(find_ms * 1e3, 2), "small_map_results_exact": ok}
    del t
    return res


def mix32_torch(x):
    """MurmurHash3 fmix32 over int64 tensors holding uint32 values: a bijection on 32 bits."""
    m = 0xFFFFFFFF
    x = x & m
    x = x ^ (x >> 16)
    x = (x * 0x85EBCA6B) & m
    x = x ^ (x >> 13)
    x = (x * 0xC2B2AE35) & m
    return x ^ (x >> 16)


BATCHED_TABLES = 4096


def batched_workload():
    """The batched workload's inputs, on the device: 4,096 StaticMap<int32,int32>
    tables with log-normal key counts (median 32,768, sigma(log2) = 2.0, clipped
    to [1,024; 4,194,304]); per table its own distinct keys, then 2x its key
    count of queries at 50% hits.  Returns the per-table sizes and offsets
    (numpy) and the concatenated keys, values, packed pairs, queries and the
    hit mask (tensors)."""
    import torch
    import b2co
    rng = np.random.default_rng(SEED + 11)
    count = BATCHED_TABLES
    sizes = np.clip(np.round(np.exp2(rng.normal(15.0, 2.0, size=count))), 1024, 4194304).astype(np.int64)
    total = int(sizes.sum())
    ins_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    q_off = 2 * ins_off
    # keys of table t: fmix32 of a per-table counter range (distinct within the
    # table, uniform), skipping the -1 sentinel; misses from the next range
    t_of = torch.repeat_interleave(torch.arange(count, device="cuda"), torch.from_numpy(sizes).cuda())
    j = torch.arange(total, device="cuda") - torch.from_numpy(ins_off[:-1]).cuda()[t_of]
    salt = (t_of * 0x9E3779B1) & 0xFFFFFFFF
    k32 = mix32_torch(j ^ salt)
    k32 = torch.where(k32 == 0xFFFFFFFF, mix32_torch((j + (1 << 31)) ^ salt), k32)
    keys = k32.to(torch.int32)  # two's-complement wrap of the uint32 value
    vals = (k32 >> 1).to(torch.int32)  # never the -1 sentinel
    pairs = b2co.pack_pairs(keys, vals)
    vals_keep = vals
    del t_of, j, salt, k32
    g = torch.Generator(device="cuda").manual_seed(SEED + 12)
    qt = torch.repeat_interleave(torch.arange(count, device="cuda"), 2 * torch.from_numpy(sizes).cuda())
    qj = torch.arange(2 * total, device="cuda") - torch.from_numpy(q_off[:-1]).cuda()[qt]
    n_t = torch.from_numpy(sizes).cuda()[qt]
    base = torch.from_numpy(ins_off[:-1]).cuda()[qt]
    hit = qj < n_t
    rnd = torch.randint(0, 1 << 40, (2 * total,), generator=g, device="cuda")
    hit_keys = keys[base + rnd % n_t]
    qsalt = (qt * 0x9E3779B1) & 0xFFFFFFFF
    miss = mix32_torch((qj + (1 << 30)) ^ qsalt).to(torch.int64).to(torch.int32)  # j >= 2^30 never used above
    q = torch.where(hit, hit_keys, miss)
    del qt, qj, n_t, base, rnd, hit_keys, qsalt, miss
    return {"count": count, "sizes": sizes, "total": total, "ins_off": ins_off, "q_off": q_off, "keys": keys,
            "vals": vals_keep, "pairs": pairs, "queries": q, "hit": hit}


def batched_measurements(stream):
    """Batched tables: 4,096 StaticMap<int32,int32> (DoubleHashing<xxhash_32>, bucket 5)
    at load factor 0.5 with log-normal key counts (median 32,768, sigma(log2) = 2.0,
    clipped to [1,024; 4,194,304]); each table inserts its own keys, then finds 2x its
    key count at 50% hits.  One persistent group launch (and its CUDA-graph replay,
    lane count from the autotuner) against one plain launch per table."""
    import torch
    import b2co
    w = batched_workload()
    count, sizes, total, ins_off, q_off = w["count"], w["sizes"], w["total"], w["ins_off"], w["q_off"]
    pairs, q, hit = w["pairs"], w["queries"], w["hit"]
    del w
    d_ins_off = torch.from_numpy(ins_off).cuda()
    d_q_off = torch.from_numpy(q_off).cuda()
    out = torch.empty(2 * total, dtype=torch.int32, device="cuda")
    ref = torch.empty(2 * total, dtype=torch.int32, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    grp = b2co.TableGroup(2 * sizes, -1, -1, key_dtype=torch.int32, value_dtype=torch.int32)
    torch.cuda.synchronize()
    e0.record(stream)
    failed = grp.Insert(pairs, d_ins_off, sync=False)
    e1.record(stream)
    torch.cuda.synchronize()
    res = {"batched_tables": count, "batched_total_keys": total, "batched_total_queries": 2 * total,
           "batched_group_insert_gkeys": round(total / e0.elapsed_time(e1) / 1e6, 3)}
    per = b2co.TableGroup(2 * sizes, -1, -1, key_dtype=torch.int32, value_dtype=torch.int32)
    torch.cuda.synchronize()
    e0.record(stream)
    per.InsertPerTable(pairs, ins_off.astype(np.uint64))
    e1.record(stream)
    torch.cuda.synchronize()
    res["batched_per_table_insert_gkeys"] = round(total / e0.elapsed_time(e1) / 1e6, 3)
    b2co.tune_cache_clear()
    shape, _ = grp.Autotune(q, d_q_off, ref)
    res["batched_autotuned_shape"] = {"lanes": shape[0], "keys_per_tile": shape[1], "block": shape[2]}
    res["batched_autotune_reused_from_cache"] = grp.Autotune(q, d_q_off, ref)[1]
    ms = timed(lambda: grp.Find(q, d_q_off, out))
    res["batched_group_find_gkeys"] = round(2 * total / ms / 1e6, 3)
    ms = timed(lambda: grp.Find(q, d_q_off, out, graph=True))
    res["batched_graph_find_gkeys"] = round(2 * total / ms / 1e6, 3)
    res["batched_graph_equals_group"] = bool(torch.equal(out, ref))
    out2 = torch.empty_like(out)
    ms = timed(lambda: per.FindPerTable(q, q_off.astype(np.uint64), out2), reps=2)
    res["batched_per_table_find_gkeys"] = round(2 * total / ms / 1e6, 3)
    # the 4,096 per-table launches captured once in a CUDA graph and replayed:
    # what a graph buys when the work is many small launches
    graph = torch.cuda.CUDAGraph()
    out2.zero_()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        per.FindPerTable(q, q_off.astype(np.uint64), out2)
    ms = timed(lambda: graph.replay(), reps=2)
    res["batched_per_table_graph_find_gkeys"] = round(2 * total / ms / 1e6, 3)
    res["batched_per_table_graph_equals_group"] = bool(torch.equal(out2, ref))
    del graph
    res["batched_per_table_equals_group"] = bool(torch.equal(out2, ref))
    res["batched_hits_found"] = bool(((ref != -1) == hit).all().item())
    del out2, per
    # the random-window ceiling for these 8-byte slots: bare 40-byte window reads
    # over one table with as many slots as the whole group (after the timed regions)
    flat = b2co.StaticMap(grp.total_slots(), -1, -1, key_dtype=torch.int32, value_dtype=torch.int32)
    ceil = window_gather_ceiling(flat, stream, res["batched_group_find_gkeys"], None)
    res["batched_window_gather_ceiling_gwin"] = ceil["window_gather_ceiling_gwin"]
    # every query reads at least one window, so this is a lower bound of the share of the ceiling used
    res["batched_find_queries_vs_ceiling"] = round(res["batched_group_find_gkeys"] / ceil["window_gather_ceiling_gwin"], 4)
    del flat
    return res


def bloom_hll_measurements(stream, bloom=True, hll_log2=30):
    """The BloomFilter / HyperLogLog workload: a 2^30-bit filter (2^22 blocks of 256 bits)
    with 2^28 uniform uint64 adds and 2^28 queries (half absent); an int64 HyperLogLog of
    64 KiB (p = 16) with 2^hll_log2 (default 2^30) adds drawn from 10^7 distinct keys, and
    a merge of 16 sub-sketches.  Size-independent checks: no false negatives, merge ==
    one-shot.  `bloom=False` runs the HyperLogLog part alone (profiling)."""
    import torch
    import b2co
    peak, _ = peaks()
    res = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_once(fn):
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    g = torch.Generator(device="cuda").manual_seed(SEED + 7)
    if bloom:
        res.update(bloom_part(f_time=time_once, g=g, peak=peak))
    n_hll = 1 << hll_log2
    keys = hll_keys(g, n_hll)
    h = b2co.HyperLogLog(16)
    h.AddAsync(keys[: 1 << 20])
    h.Clear()
    ms = time_once(lambda: h.AddAsync(keys))
    res["hll_adds"] = n_hll
    res["hll_add_gkeys"] = round(n_hll / ms / 1e6, 3)
    res["hll_add_hbm_frac"] = round(n_hll * 8 / (ms / 1e3) / 1e9 / peak, 4)
    est = h.Estimate()
    res["hll_estimate"] = est
    res["hll_estimate_rel_err_vs_1e7"] = round(abs(est - 10_000_000) / 10_000_000, 5)
    parts = [b2co.HyperLogLog(16) for _ in range(16)]
    for i, p in enumerate(parts):
        p.AddAsync(keys[i * (n_hll >> 4):(i + 1) * (n_hll >> 4)])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for p in parts[1:]:
        parts[0].Merge(p)
    res["hll_merge16_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
    res["hll_merge_equals_one_shot"] = bool(np.array_equal(parts[0].registers(), h.registers()))
    return res


def bloom_workload(g):
    """A filter of 2^22 blocks (2^30 bits), 2^28 uniform 64-bit adds, and 2^28
    queries: half drawn from the adds, half from a disjoint stream, in that
    order.  Returns (num_blocks, adds, queries) on the device."""
    import torch
    nb, n = 1 << 22, 1 << 28
    adds = mix64_torch(counters(3 << 40, n, "torch"))
    absent = mix64_torch(counters(4 << 40, n // 2, "torch"))
    q = torch.cat([adds[torch.randint(0, n, (n // 2,), generator=g, device="cuda")], absent])
    return nb, adds, q


def hll_keys(g, n):
    """n int64 HyperLogLog inputs drawn uniformly with replacement from 10^7
    distinct uniform keys, on the device."""
    import torch
    distinct = mix64_torch(counters(5 << 40, 10_000_000, "torch"))
    return distinct[torch.randint(0, distinct.numel(), (n,), generator=g, device="cuda")]


def bloom_part(f_time, g, peak):
    import torch
    import b2co
    res = {}
    time_once = f_time
    nb, adds, q = bloom_workload(g)
    n = adds.numel()
    f = b2co.BloomFilter(nb, key_dtype=torch.int64)
    f.AddAsync(adds)  # warm-up: the same batch, so the timed Add runs the path (and scratch) it will use
    f.Clear()
    ms = time_once(lambda: f.AddAsync(adds))
    res["bloom_add_gkeys"] = round(n / ms / 1e6, 3)
    # per-key block model: the key plus its 32-byte block read and written
    res["bloom_add_hbm_frac"] = round(n * 72 / (ms / 1e3) / 1e9 / peak, 4)
    # least traffic of any Add: every key read once, the filter read and written once
    res["bloom_add_hbm_frac_keys_filter"] = round((n * 8 + 2 * nb * 32) / (ms / 1e3) / 1e9 / peak, 4)
    # the same Add through the other paths; same bits
    default_words = f.words()
    for name, mode in (("bulk", b2co.BLOOM_ADD_BULK), ("atomic", b2co.BLOOM_ADD_ATOMIC)):
        f.set_add_mode(mode)
        f.Clear()
        f.AddAsync(adds)
        f.Clear()
        ms = time_once(lambda: f.AddAsync(adds))
        res[f"bloom_add_{name}_gkeys"] = round(n / ms / 1e6, 3)
        res[f"bloom_add_{name}_equals_default"] = bool(np.array_equal(f.words(), default_words))
    del default_words
    f.set_add_mode(b2co.BLOOM_ADD_AUTO)
    out = torch.empty(q.numel(), dtype=torch.uint8, device="cuda")
    f.ContainsAsync(q, out)
    ms = time_once(lambda: f.ContainsAsync(q, out))
    res["bloom_contains_gkeys"] = round(q.numel() / ms / 1e6, 3)
    res["bloom_contains_hbm_frac"] = round(q.numel() * 41 / (ms / 1e3) / 1e9 / peak, 4)
    res["bloom_no_false_negatives"] = bool(out[: n // 2].all().item())
    res["bloom_false_positive_rate"] = round(float(out[n // 2:].float().mean().item()), 6)
    del adds, q, out, f
    return res


# ---------------------------------------------------------------------------
# reference arm: the reference algorithm's CPU restatement on the host cores
# ---------------------------------------------------------------------------

def multi_measurements(stream, log2n=26):
    """StaticMultimap<int64,int64> and StaticMultiset<int64>: 2^log2n entries
    over 2^(log2n-2) distinct keys (uniform, about 4 per key); Insert, the lazy
    grouped-index build of the multimap (first query after the insert), Find
    and Count on 2^log2n queries at 50% hits, Retrieve on 2^(log2n-2) queries,
    and the multiset's CountEach.  Device time by CUDA events on the stream
    (the calls are synchronous, so host time is inside)."""
    import torch
    import b2co
    n = 1 << log2n
    lo = -(1 << 63)
    g = torch.Generator(device="cuda").manual_seed(SEED + 21)
    distinct = mix64_torch(counters(7 << 40, n >> 2, "torch")) >> 1  # halved: never the int64 sentinel
    keys = distinct[torch.randint(0, n >> 2, (n,), generator=g, device="cuda")]
    vals = mix64_torch(counters(8 << 40, n, "torch")) >> 1
    q = torch.where(torch.rand(n, generator=g, device="cuda") < 0.5, distinct[torch.randint(0, n >> 2, (n,),
                    generator=g, device="cuda")], mix64_torch(counters(9 << 40, n, "torch")) >> 1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        torch.cuda.synchronize()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    res = {"multi_entries": n, "multi_distinct_keys": n >> 2}
    mm = b2co.StaticMultimap(n, lo, lo, key_dtype=torch.int64, value_dtype=torch.int64)
    pairs = b2co.pack_pairs(keys, vals)
    ms, failed = timed(lambda: mm.Insert(pairs))
    assert failed == 0
    res["multimap_insert_gpairs"] = round(n / ms / 1e6, 3)
    ms, _ = timed(lambda: mm.Count(q[:1]))  # builds the grouped index
    res["multimap_index_build_ms"] = round(ms, 2)
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    mm.Find(q, out)
    ms, _ = timed(lambda: mm.Find(q, out))
    res["multimap_find_gkeys"] = round(n / ms / 1e6, 3)
    ms, total = timed(lambda: mm.Count(q))
    res["multimap_count_gkeys"] = round(n / ms / 1e6, 3)
    qr = q[: n >> 2]
    cnt = mm.Count(qr)
    ko = torch.empty(cnt, dtype=torch.int64, device="cuda")
    vo = torch.empty(cnt, dtype=torch.int64, device="cuda")
    ms, w = timed(lambda: mm.Retrieve(qr, ko, vo, cnt))
    assert w == cnt
    res["multimap_retrieve_gkeys"] = round((n >> 2) / ms / 1e6, 3)
    res["multimap_retrieve_gpairs_out"] = round(cnt / ms / 1e6, 3)
    kk, vv = ko.cpu().numpy(), vo.cpu().numpy()
    del mm, pairs, ko, vo, out
    st = b2co.StaticMultiset(n, lo, key_dtype=torch.int64)
    ms, failed = timed(lambda: st.Insert(keys))
    assert failed == 0
    res["multiset_insert_gkeys"] = round(n / ms / 1e6, 3)
    ce = torch.empty(n, dtype=torch.int64, device="cuda")
    st.CountEach(q, ce)
    ms, _ = timed(lambda: st.CountEach(q, ce))
    res["multiset_count_each_gkeys"] = round(n / ms / 1e6, 3)
    res["multiset_count_matches_multimap"] = bool(int(ce.sum().item()) == total)
    # size-independent checks of the multimap's Retrieve: each query's run has the
    # multiset's multiplicity of its key and its values ascend within the run
    per_query = ce[: n >> 2].cpu().numpy()
    starts = np.zeros(len(vv), dtype=bool)
    starts[np.cumsum(per_query)[:-1][per_query[1:] > 0]] = True
    starts[0] = True
    inner = ~starts[1:]
    res["multimap_runs_ascending"] = bool(int(per_query.sum()) == len(vv) and (vv[1:][inner] >= vv[:-1][inner]).all()
                                          and (kk[1:][inner] == kk[:-1][inner]).all())
    del st, ce
    torch.cuda.empty_cache()
    return res


def roaring_serialize32(values: np.ndarray) -> bytes:
    """Portable Roaring serialization (cookie 12346: arrays and bitsets, with
    offsets) of a set of uint32 values -- the bench's own input builder."""
    import struct
    vals = np.unique(values.astype(np.uint32))
    hi = (vals >> 16).astype(np.uint32)
    keys, starts = np.unique(hi, return_index=True)
    bounds = np.append(starts, len(vals))
    bodies = []
    for i in range(len(keys)):
        lo = (vals[bounds[i]:bounds[i + 1]] & 0xFFFF).astype(np.uint16)
        if len(lo) <= 4096:
            bodies.append((len(lo), lo.astype("<u2").tobytes()))
        else:
            bits = np.zeros(65536, dtype=np.uint8)
            bits[lo] = 1
            bodies.append((len(lo), np.packbits(bits, bitorder="little").tobytes()))
    n = len(keys)
    head = bytearray(struct.pack("<II", 12346, n))
    head += np.stack([keys.astype(np.uint16), np.array([c - 1 for c, _ in bodies], np.uint16)], 1).astype("<u2").tobytes()
    pos = len(head) + 4 * n
    offs = np.cumsum([pos] + [len(b) for _, b in bodies[:-1]]).astype("<u4") if n else np.zeros(0, "<u4")
    return bytes(head) + offs.tobytes() + b"".join(b for _, b in bodies)


def roaring_measurements(stream, log2q=27):
    """RoaringBitmap<uint32_t> Contains on 2^log2q queries at 50% hits against
    (a) a sparse bitmap: 2^24 uniform keys over the whole 32-bit range (65,536
    array containers of ~256) and (b) a dense one: 2^26 even keys in 2,048
    bitset containers.  Device time by CUDA events on the stream."""
    import torch
    import b2co
    res = {}
    rng = np.random.default_rng(SEED + 31)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nq = 1 << log2q
    for name, vals in [("sparse", rng.integers(0, 2**32, size=1 << 24, dtype=np.uint64)),
                       ("dense", np.arange(1 << 26, dtype=np.uint64) * 2)]:
        data = roaring_serialize32(vals)
        bm = b2co.RoaringBitmap(data, 4)
        u = np.unique(vals.astype(np.uint32))
        hits = u[rng.integers(0, len(u), size=nq // 2)]
        q = np.concatenate([hits, rng.integers(0, 2**32, size=nq - nq // 2, dtype=np.uint64).astype(np.uint32)])
        rng.shuffle(q)
        qd = torch.from_numpy(q.view(np.int32)).cuda()
        out = torch.empty(nq, dtype=torch.uint8, device="cuda")
        bm.ContainsAsync(qd, out)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(5):
            bm.ContainsAsync(qd, out)
        e1.record(stream)
        torch.cuda.synchronize()
        res[f"roaring_{name}_contains_gkeys"] = round(5 * nq / e0.elapsed_time(e1) / 1e6, 3)
        res[f"roaring_{name}_bitmap_bytes"] = bm.SizeBytes()
        res[f"roaring_{name}_hits_found"] = bool(int(out.sum().item()) >= nq // 2)  # every planted hit at least
        del bm, qd, out
    return res


SERVED_RATES = (1000, 2000, 5000, 10000, 20000, 50000, 200000)  # the last one is past saturation
SERVED_STREAM, SERVED_MISS, SERVED_NEW, SERVED_VALUES = 3 << 40, 4 << 40, 5 << 40, 6 << 40


def served_measurements(stream, rates=SERVED_RATES, seconds=0.5, pool=384, inflight=8):
    """Served tables: 8 resident StaticMap<int64,int64> (DoubleHashing<xxhash_32>,
    bucket 5) of 10M..200M pairs (geometric spacing) at load factor 0.6, 15 GB in
    all, behind one b2co Server (HBM budget 150 GB, `inflight` launch streams,
    at most 4 Mi keys per coalesced launch).  Requests arrive as a Poisson
    stream at each swept rate for `seconds`; sizes are log-normal (median
    31,623 keys, sigma 1.15) clipped to [1e3, 1e6]; 90% Find / 10%
    InsertOrAssign, tables uniform, keys at a 70% hit rate (misses from a
    disjoint stream; IOA non-hits are new keys).  Payloads come from a pool of
    `pool` pinned host requests reused round-robin; the schedule is submitted
    in chunks of 32 (submit_many), chunk c after chunk c - pool/32 completed
    (its buffers are reused).  Latency = done - scheduled arrival (queueing
    included); keys/s = all keys / (last done - first arrival)."""
    import torch
    import b2co
    rng = np.random.default_rng(SEED + 5)
    sizes = np.geomspace(10e6, 200e6, 8).astype(np.int64)
    tables = []
    t_build = time.time()
    for j, n in enumerate(sizes):
        m = b2co.StaticMap(int(n / 0.6), -1, -1, key_dtype=torch.int64, value_dtype=torch.int64, bucket_size=5,
                           probing=b2co.PROBE_DOUBLE, hash_kind=b2co.HASH_XXH32)
        k = mix64_torch(counters(SERVED_STREAM + (j << 32), int(n), "torch"))
        v = mix64_torch(counters(SERVED_VALUES + (j << 32), int(n), "torch"))
        p = b2co.pack_pairs(k, v)
        del k, v
        assert m.Insert(p) == 0
        del p
        tables.append(m)
    torch.cuda.synchronize()
    table_gb = sum(m.Capacity() * 16 for m in tables) / 1e9
    log(f"[served] 8 tables, {int(sizes.sum())} pairs, {table_gb:.1f} GB, built in {time.time() - t_build:.1f} s")

    # request pool: one pinned arena for inputs, one for outputs
    ops = np.where(rng.random(pool) < 0.1, b2co.OP_INSERT_OR_ASSIGN, b2co.OP_FIND)
    tabs = rng.integers(0, 8, size=pool)
    ns = np.clip(np.exp(rng.normal(math.log(31623), 1.15, size=pool)), 1e3, 1e6).astype(np.int64)
    in_words = np.where(ops == b2co.OP_FIND, ns, 2 * ns)
    in_arena = b2co.pinned((int(in_words.sum()),), np.int64)
    out_arena = b2co.pinned((int(ns.sum()),), np.int64)
    pool_desc = np.zeros(pool, dtype=b2co.REQUEST_DESC)
    io, oo, new_ctr = 0, 0, 0
    for i in range(pool):
        n, j = int(ns[i]), int(tabs[i])
        hit = rng.random(n) < 0.7
        other = SERVED_MISS if ops[i] == b2co.OP_FIND else SERVED_NEW
        idx = np.where(hit, SERVED_STREAM + (j << 32) + rng.integers(0, sizes[j], size=n),
                       other + new_ctr + np.arange(n))
        new_ctr += n
        keys = mix64_np(idx)
        inp = in_arena[io:io + in_words[i]]
        io += int(in_words[i])
        if ops[i] == b2co.OP_FIND:
            inp[:] = keys
            out_ptr = out_arena[oo:oo + n].ctypes.data
            oo += n
        else:
            pr = inp.reshape(n, 2)
            pr[:, 0] = keys
            pr[:, 1] = mix64_np(SERVED_VALUES + (7 << 32) + np.arange(n) + i * (1 << 20))
            out_ptr = 0
        pool_desc[i] = (tables[j]._h.value, int(ops[i]), 0, inp.ctypes.data, out_ptr, n, 0)

    srv = b2co.Server(max_inflight=inflight, hbm_budget_bytes=150 * 10**9, max_batch_keys=1 << 22)
    for m in tables:
        srv.register(m)
    chunk = 32  # requests per submit_many / wait_many call
    assert pool % chunk == 0
    ring = pool // chunk

    def run_rate(rate, count):
        count = -(-count // chunk) * chunk
        t0 = b2co.Server.now_ns() + 5_000_000
        arrivals = (t0 + np.cumsum(rng.exponential(1e9 / rate, size=count))).astype(np.uint64)
        ids, infos, late = [], [], 0
        s0 = srv.stats()
        for c in range(count // chunk):
            if c >= ring:
                infos.append(srv.wait_many(ids[c - ring]))
            d = pool_desc[(c % ring) * chunk:(c % ring + 1) * chunk].copy()
            d["arrival_ns"] = arrivals[c * chunk:(c + 1) * chunk]
            late += int(b2co.Server.now_ns() > int(d["arrival_ns"][0]))
            ids.append(srv.submit_many(d))
        infos += [srv.wait_many(x) for x in ids[max(0, len(ids) - ring):]]
        s1 = srv.stats()
        inf = np.concatenate(infos)
        assert (inf["status"] == 0).all()
        lat = (inf["done_ns"] - inf["arrival_ns"]).astype(np.float64) / 1e6
        queued = (inf["admit_ns"] - inf["arrival_ns"]).astype(np.float64) / 1e6
        service = lat - queued
        is_find = inf["op"] == b2co.OP_FIND
        keys = int(inf["n"].sum())
        span = float(inf["done_ns"].max() - inf["arrival_ns"].min()) / 1e9
        launches = s1["launches"] - s0["launches"]
        return {"offered_req_s": rate, "requests": count, "achieved_req_s": round(count / span, 1),
                "keys_per_s": round(keys / span, 1), "gkeys_s": round(keys / span / 1e9, 4),
                "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                "find_p99_ms": round(float(np.percentile(lat[is_find], 99)), 3),
                "p99_queue_ms": round(float(np.percentile(queued, 99)), 3),
                "p99_service_ms": round(float(np.percentile(service, 99)), 3),
                "max_ms": round(float(lat.max()), 3), "chunks_submitted_late": late,
                "launches": launches, "requests_per_launch": round(count / max(1, launches), 2),
                "host_us_per_launch": round((s1["total_launch_host_ns"] - s0["total_launch_host_ns"])
                                            / max(1, launches) / 1e3, 1),
                "copies": s1["copies"] - s0["copies"], "packed_launches": s1["packed_launches"] - s0["packed_launches"],
                "direct_launches": s1["direct_launches"] - s0["direct_launches"]}

    run_rate(rates[0], 128)  # warm-up: first launches of every table
    out, plain = [], []
    for rate in rates:
        r = run_rate(rate, max(200, int(rate * seconds)))
        log(f"[served] {rate} req/s: p50 {r['p50_ms']} ms, p99 {r['p99_ms']} ms, {r['gkeys_s']} Gkeys/s, "
            f"{r['requests_per_launch']} req/launch, {r['host_us_per_launch']} us host/launch")
        out.append(r)
    # the same server with lookup results written by the GPU into the pinned
    # result buffers, and with coalesced requests packed into one copy each way
    copied, packed = [], []
    for arm, lst in (("direct", copied), ("packed", packed)):
        srv.set_direct_results(arm == "direct")
        srv.set_packing(arm == "packed")
        for rate in rates:
            r = run_rate(rate, max(200, int(rate * seconds)))
            log(f"[served {arm}] {rate} req/s: p50 {r['p50_ms']} ms, p99 {r['p99_ms']} ms, {r['gkeys_s']} Gkeys/s")
            lst.append({k: r[k] for k in ("offered_req_s", "achieved_req_s", "gkeys_s", "p50_ms", "p99_ms",
                                          "copies", "launches", "packed_launches")})
    srv.set_packing(False)
    srv.set_direct_results(False)
    # the baseline on the same schedule: one plain launch per request, one
    # request per table at a time (copy in, Find / InsertOrAssign, copy out)
    srv.set_plain(True)
    for rate in rates:
        r = run_rate(rate, max(200, int(rate * seconds)))
        log(f"[served plain] {rate} req/s: p50 {r['p50_ms']} ms, p99 {r['p99_ms']} ms, {r['gkeys_s']} Gkeys/s")
        plain.append({k: r[k] for k in ("offered_req_s", "requests", "achieved_req_s", "gkeys_s", "p50_ms", "p99_ms",
                                        "launches")})
    srv.set_plain(False)
    st = srv.stats()
    srv.close()
    bus = copy_probe(in_arena, in_words, out_arena, ns)
    del tables
    torch.cuda.empty_cache()
    return {"served": {"tables": [int(x) for x in sizes], "table_gb": round(table_gb, 2), "load_factor": 0.6,
                       "inflight_streams": inflight, "max_batch_keys": 1 << 22, "hbm_budget_gb": 150,
                       "request_pool": pool, "mean_request_keys": round(float(np.mean(ns)), 1),
                       "seconds_per_rate": seconds, "host_buffers": "pinned",
                       "staging_grows": st["staging_grows"], "max_loop_gap_us": round(st["max_loop_gap_ns"] / 1e3, 1),
                       "sweep": out, "direct_results_sweep": copied, "packed_sweep": packed,
                       "plain_per_table_sweep": plain,
                       "server_over_plain_gkeys": [round(a["gkeys_s"] / b["gkeys_s"], 3) for a, b in zip(out, plain)],
                       "copy_probe": bus}}


def copy_probe(in_arena, in_words, out_arena, ns, streams=8, reps=3):
    """What the bus moves for the served request sizes with no lookups at all:
    every pool request's input copied in and a result of its size copied out,
    back to back on `streams` streams; host to device only, device to host
    only, and both at once (GB/s of payload each way, requests per second)."""
    import torch
    ss = [torch.cuda.Stream() for _ in range(streams)]
    hin, hout, io, oo = [], [], 0, 0
    for w, n in zip(in_words, ns):
        hin.append(torch.from_numpy(in_arena[io:io + int(w)]))
        hout.append(torch.from_numpy(out_arena[oo:oo + int(n)]))
        io, oo = io + int(w), oo + int(n)
    dev_in = torch.empty(int(in_words.max()), dtype=torch.int64, device="cuda")
    dev_out = torch.empty(int(ns.max()), dtype=torch.int64, device="cuda")
    res = {}
    for name, h2d, d2h in (("h2d_only", True, False), ("d2h_only", False, True), ("both", True, True)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            for i in range(len(hin)):
                with torch.cuda.stream(ss[i % streams]):
                    if h2d:
                        dev_in[:hin[i].numel()].copy_(hin[i], non_blocking=True)
                    if d2h:
                        hout[i].copy_(dev_out[:hout[i].numel()], non_blocking=True)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        moved = (float(in_words.sum()) if h2d else float(ns.sum())) * 8 * reps
        res[name] = {"requests_per_s": round(reps * len(hin) / el), "gbs_each_way": round(moved / el / 1e9, 2)}
    return res


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return  # rank 0 alone times the host-CPU reference
    import oracle
    threads = os.cpu_count() or 1
    cap = oracle.valid_capacity(REQ_CAPACITY, 5, oracle.PROBE_DOUBLE)
    unique, dups = workload_sizes(cap, LOAD_FACTOR)
    t0 = time.perf_counter()
    keys, stream_keys, vals = make_insert_stream(unique, dups, "np")
    o = oracle.Table(np.int64, np.int64, cap, 5, oracle.PROBE_DOUBLE, oracle.HASH_XXH32, -1, -1)
    o.insert(stream_keys, vals)  # sequential first-wins fill (same stored set as InsertAndFind)
    del stream_keys, vals
    log(f"[reference] host table built in {time.perf_counter() - t0:.1f} s")
    q = make_queries(keys, N_QUERIES, 0.5, "np")
    sample = 1 << 24
    for s in range(args.warmup):
        o.find_parallel(q[(s * sample) % N_QUERIES:][:sample], threads)
    times = []
    for s in range(args.steps):
        off = (s * sample) % N_QUERIES
        t0 = time.perf_counter()
        o.find_parallel(q[off:off + sample], threads)
        times.append(time.perf_counter() - t0)
    ms_per_step = 1e3 * float(np.mean(times))
    value = sample / (ms_per_step / 1e3) / 1e9
    desc = (f"oracle port of the reference Find (same hash, probing, capacity, bucket scan), {threads} OpenMP "
            f"threads, {sample} queries per step of the 2^27 50%-hit stream over the LF0.5 table")
    line = {
        "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": WORKLOAD, "capacity": cap, "unique_keys": unique, "queries_per_step": sample},
        "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": threads, "kind": "port", "sample": desc,
                         "cpu_model": cpu_model()},
        "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b2co", choices=["b2co", "reference"])
    ap.add_argument("--shape", default="", help="Find kernel shape LANESxITEMS, e.g. 8x1")
    ap.add_argument("--quick", action="store_true", help="skip the secondary measurements")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-host", action="store_true", help="skip the host-side oracle checks and CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end measurement")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--capacity-log2", type=int, default=28, help="requested capacity 2^k (profiling: smaller)")
    ap.add_argument("--queries-log2", type=int, default=27, help="queries per step 2^k (profiling: smaller)")
    ap.add_argument("--sweep", action="store_true", help="time every Find kernel shape and report each")
    ap.add_argument("--sweep-shapes", default="", help="comma-separated shapes for --sweep (default: a fixed list)")
    ap.add_argument("--l2-fetch", type=int, default=0, help="L2 fetch granularity hint in bytes (0 = leave default)")
    ap.add_argument("--only", default="",
                    choices=["", "served", "batched", "bloom_hll", "hll", "multi", "roaring", "small_map",
                             "insert", "dmap", "fill"],
                    help="run one secondary measurement alone and print its JSON (not the headline line)")
    ap.add_argument("--hll-log2", type=int, default=30, help="HyperLogLog adds 2^k with --only hll (profiling)")
    ap.add_argument("--batched-tables", type=int, default=4096, help="tables of the batched workload (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("warmup must be >= 3")
    global REQ_CAPACITY, N_QUERIES, BATCHED_TABLES
    REQ_CAPACITY, N_QUERIES = 1 << args.capacity_log2, 1 << args.queries_log2
    BATCHED_TABLES = args.batched_tables
    if args.only:
        import torch
        fn = {"served": served_measurements, "batched": batched_measurements, "bloom_hll": bloom_hll_measurements,
              "hll": lambda s: bloom_hll_measurements(s, bloom=False, hll_log2=args.hll_log2),
              "multi": multi_measurements, "roaring": roaring_measurements,
              "small_map": small_map_measurements, "dmap": dynamic_map_measurements, "fill": fill_measurements,
              "insert": lambda st: insert_measurements(st, capacity_log2=args.capacity_log2,
                                                       shapes=INSERT_SHAPES if args.sweep else None)}[args.only]
        print(json.dumps(fn(torch.cuda.current_stream())), flush=True)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
