"""Benchmark: LeCo-fix bulk decode GB/s and batched random access on B200.

Workload (one GPU): 200M sorted uint64 keys from a piecewise-linear trend
(segment lengths geometric, mean 50k; slopes log-uniform in [1, 2^20]) plus
round(N(0, 2^12)) noise, LeCo-fix linear codec with 4096-value blocks
(48,829 blocks).  A step is one bulk decode of the whole column (inputs and
outputs are larger than L2) followed by one batch of 2^24 uniform random
lookups.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  --impl reference times the reference's own CPU
codec (the compiled reference headers, oracle/_ref) on the host cores on the
same workload.  Under torchrun each rank decodes its own 200M-key column
(weak scaling, no data-path collective); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LeCo-fix decode GB/s and batched random-access Mlookups/s, p50/p99, 1 B200"
N_DEFAULT = 200_000_000
BS = 4096
RA_BATCH = 1 << 24
DECODE_KERNEL = "decode_staged_kernel"
RA_DRAM_BYTES = 8 + 8 + 32  # per lookup: index, value, one payload sector (directory L2-resident)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="leco", choices=["leco", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT, help="keys per GPU (default: 200M)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", default="decode",
                    choices=["decode", "batch", "serve", "varlen", "filter", "gather", "codecs", "encode"],
                    help="decode: the 200M-key LeCo-fix column (default); batch: 4096 mixed columns through "
                         "the persistent batch engine vs per-column launches")
    ap.add_argument("--ncols", type=int, default=4096)
    ap.add_argument("--fit", default="reference", choices=["reference", "exact"])
    ap.add_argument("--serve-cols", type=int, default=64)
    ap.add_argument("--serve-n", type=int, default=100_000_000)
    ap.add_argument("--requests", type=int, default=4000)
    ap.add_argument("--rate", type=float, default=50_000.0, help="offered requests per second (Poisson)")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name: str = "decode_staged_kernel_leco_u64_200M.txt"):
    """Per-launch DRAM bytes of a kernel at the bench's full size, from its
    committed ncu summary (line `traffic_bytes_per_launch_full_size:`)."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch_full_size:"):
            try:
                return int(float(line.split(":", 1)[1].strip().split()[0]))
            except ValueError:
                return None
    return None


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons through NVML every
    few milliseconds while the timed region runs."""

    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index: int, period_s: float = 0.002):
        self.idx, self.period = gpu_index, period_s
        self.sm, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._live = threading.Event()  # set once the first sample is taken

    def _run(self):
        import pynvml

        try:
            pynvml.nvmlInit()
        except Exception:
            self._live.set()
            return
        try:
            uuid = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            h = pynvml.nvmlDeviceGetHandleByIndex(self.idx if not uuid or "," in uuid or not uuid.isdigit() else 0)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            while not self._stop.is_set():
                self.sm.append(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                r = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                for name, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
                self._live.set()
                time.sleep(self.period)
        finally:
            self._live.set()
            pynvml.nvmlShutdown()

    def __enter__(self):
        # the timed region starts only once sampling runs (NVML's start-up can take
        # longer than a short timed region)
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        self._live.wait(timeout=5.0)
        return self

    def __exit__(self, *a):
        self._stop.set()
        self.t.join(timeout=5)

    def summary(self):
        return {"sm_mhz": float(np.median(self.sm)) if self.sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def decode_config(n: int, world: int) -> dict:
    """The decode workload's config; both arms (this library and --impl
    reference) print exactly this dict."""
    return {"workload": f"leco_fix u64 {n / 1e6:g}M piecewise-linear sorted keys, {BS}-value blocks, "
                        f"bulk decode + 2^{RA_BATCH.bit_length() - 1} uniform random lookups per step",
            "keys_per_gpu": n, "block_size": BS, "blocks": (n + BS - 1) // BS, "ra_batch": RA_BATCH,
            "l2": "inputs and outputs larger than L2 (no flush needed)", "parallelism": f"shard{world}",
            "generator_seed": 2}


def reference_lib():
    """The compiled reference headers (oracle/_ref), or None if not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return oracle.Reference() if os.path.exists(oracle.REF_SO) else None


def cpu_reference_baseline(R, x: np.ndarray, pay: np.ndarray, off: np.ndarray, threads: int, budget_s: float = 6.0):
    """Times the compiled reference (Leco_int<uint64_t>::decodeArray8 per block,
    randomdecodeArray8 per index) on the workload's whole column, as the
    reference's drivers run it (experiments/leco_int_fix_template.cpp:142-153
    bulk decode, :180-213 random access): (ii) `threads` host threads over
    disjoint block / index ranges, repeated for about `budget_s`; (i) one
    thread.  Every run is checked against the input."""
    n = len(x)
    padded = R.pad(pay)
    out = np.empty(n + 64, np.uint64)
    rng = np.random.default_rng(7)
    idx = rng.integers(0, n, 1 << 22).astype(np.uint64)
    rout = np.empty(len(idx), np.uint64)
    R.decode_column(0, padded, off, n, 8, BS, threads=threads, out=out, padded=True)  # warm the pages
    reps, t0 = 0, time.perf_counter()
    while True:
        R.decode_column(0, padded, off, n, 8, BS, threads=threads, out=out, padded=True)
        reps += 1
        el = time.perf_counter() - t0
        if el > budget_s or reps >= 1000:
            break
    assert np.array_equal(out[:n], x), "reference decode mismatch"
    gbs = reps * n * 8 / el / 1e9
    t0 = time.perf_counter()
    R.random_column(0, padded, off, 8, BS, idx, threads=threads, out=rout, padded=True)
    ra = len(idx) / (time.perf_counter() - t0) / 1e6
    assert np.array_equal(rout, x[idx.astype(np.int64)]), "reference random access mismatch"
    # (i) one thread, the reference drivers' own loop structure
    t1 = []
    for _ in range(2):
        t0 = time.perf_counter()
        R.decode_column(0, padded, off, n, 8, BS, threads=1, out=out, padded=True)
        t1.append(time.perf_counter() - t0)
    assert np.array_equal(out[:n], x), "reference decode mismatch"
    m1 = 1 << 20
    t0 = time.perf_counter()
    R.random_column(0, padded, off, 8, BS, idx[:m1], threads=1, out=rout, padded=True)
    ra1 = m1 / (time.perf_counter() - t0) / 1e6
    assert np.array_equal(rout[:m1], x[idx[:m1].astype(np.int64)])
    return {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": f"the whole {n / 1e6:g}M-key column, {reps} full decodes in {el:.1f}s on {threads} threads; "
                      f"{len(idx)} random lookups",
            "ra_mlookups_s": round(ra, 2),
            "single_thread": {"value": round(n * 8 / min(t1) / 1e9, 3), "unit": "GB/s", "cores": 1,
                              "ra_mlookups_s": round(ra1, 2),
                              "sample": f"the whole column decoded twice (best of 2) and {m1} random lookups on one "
                                        "thread, the reference drivers' per-block and per-index loops"}}


def run_reference(args, world, rank):
    """--impl reference: the reference's CPU codec (the unmodified headers,
    compiled into oracle/_ref) on the host cores, on the same column as this
    library's rank-0 arm: each step is one bulk decode of the whole column
    and one batch of 2^24 uniform random lookups, on all host threads."""
    if rank != 0:
        return
    from leco_b200 import workloads

    R = reference_lib()
    if R is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libleco_ref.so was not built"}))
        return
    threads = host_threads()
    n = args.n
    x = workloads.piecewise_linear_u64(n, seed=2).numpy().view(np.uint64)
    pay, off = R.encode_column(0, x, BS, threads=threads)
    padded = R.pad(pay)
    out = np.empty(n + 64, np.uint64)
    rng = np.random.default_rng(11)
    idx_sets = [rng.integers(0, n, RA_BATCH).astype(np.uint64) for _ in range(2)]
    rout = np.empty(RA_BATCH, np.uint64)
    dec, ra = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        R.decode_column(0, padded, off, n, 8, BS, threads=threads, out=out, padded=True)
        t1 = time.perf_counter()
        R.random_column(0, padded, off, 8, BS, idx_sets[i % 2], threads=threads, out=rout, padded=True)
        t2 = time.perf_counter()
        if i >= args.warmup:
            dec.append(t1 - t0)
            ra.append(t2 - t1)
    assert np.array_equal(out[:n], x), "reference decode mismatch"
    last = idx_sets[(args.warmup + args.steps - 1) % 2]
    assert np.array_equal(rout, x[last.astype(np.int64)]), "reference random access mismatch"
    dec_s, ra_s = float(np.mean(dec)), float(np.mean(ra))
    gbs = n * 8 / dec_s / 1e9
    base = cpu_reference_baseline(R, x, pay, off, threads, budget_s=3.0)
    cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
           "sample": f"the whole {n / 1e6:g}M-key column per step ({args.steps} timed steps, {threads} threads)",
           "single_thread": base["single_thread"]}
    out_line = {"metric": METRIC, "value": round(gbs, 3), "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round((dec_s + ra_s) * 1e3, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": decode_config(n, world),
                "decode_ms": round(dec_s * 1e3, 3), "ra_mlookups_s": round(RA_BATCH / ra_s / 1e6, 2),
                "compressed_ratio": round(len(pay) / (n * 8), 5),
                "cpu_baseline": cpu,
                "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out_line), flush=True)


def run_batch(args, world, rank, local):
    """4096 columns, lengths log-uniform in [1K, 4M], 50 % u32 / 50 % u64, four
    data families, codec LeCo-fix / Delta-fix / FOR per column, block size from
    the committed autotune table.  Times one encode+decode pass three ways on
    the same columns: one leco_encode + leco_decode call per column, the
    persistent batch kernels, and the batch pass replayed as a CUDA graph."""
    import math

    import torch

    import leco_b200 as lc
    from leco_b200 import autotune, workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cols, raw, shapes, launch = [], 0, {}, {}
    for x, codec, _ in workloads.batch_columns(args.ncols, seed=3 + rank):
        s, n = x.dtype.itemsize, len(x)
        bs, g, u = autotune.pick(codec, s, n, autotune.classify(x))
        shapes[bs] = shapes.get(bs, 0) + 1
        launch[f"{g}x{u}"] = launch.get(f"{g}x{u}", 0) + 1
        cols.append((torch.from_numpy(x.view(np.int64 if s == 8 else np.int32)).to(dev), codec, bs, g, u))
        raw += n * s
    fit = lc.FIT_EXACT if args.fit == "exact" else lc.FIT_REFERENCE
    b = lc.Batch(cols, fit_mode=fit)
    stream = torch.cuda.current_stream()

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def verify():
        lc.check()
        for spec, c in zip(cols, b.cols):
            assert torch.equal(c.out, spec[0]), "batch decode mismatch"

    per_col = lambda: (b.encode_per_column(), b.decode_per_column())
    batch = lambda: (b.encode(), b.decode())
    graph = lambda: b.run_graph(3)
    for fn in (per_col, batch, graph):
        for _ in range(max(1, args.warmup)):
            fn()
    torch.cuda.synchronize()
    verify()
    k = max(3, args.steps // 5)
    t_col = timed(per_col, k)
    verify()
    t_batch = timed(batch, k)
    verify()
    with ClockSampler(local) as clk:
        t_graph = timed(graph, k)
    verify()
    t_dec_col = timed(b.decode_per_column, k)
    t_dec_batch = timed(b.decode, k)
    comp = sum(c.nbytes for c in b.cols)
    if rank == 0:
        line = {"metric": "batched persistent encode+decode pass vs per-column launches (speed-up)",
                "value": round(t_col / t_graph, 3), "unit": "x", "n_gpus": world, "steps": k, "warmup": args.warmup,
                "ms_per_step": round(t_graph, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u32+u64", "data": "synthetic",
                "config": {"workload": f"{args.ncols} columns, lengths log-uniform 1K-4M, 50% u32/50% u64, "
                                       "families linear/step/walk/uniform, codecs LeCo/Delta/FOR, autotuned block "
                                       "size, threads per block and unroll depth",
                           "raw_bytes": raw, "blocks": b.total_blocks, "fit": args.fit,
                           "block_sizes": {str(k_): v for k_, v in sorted(shapes.items())},
                           "threads_x_unroll": dict(sorted(launch.items()))},
                "ms_per_pass": {"per_column_launches": round(t_col, 3), "persistent": round(t_batch, 3),
                                "persistent_graph": round(t_graph, 3)},
                "decode_ms": {"per_column_launches": round(t_dec_col, 3), "persistent": round(t_dec_batch, 3)},
                "pass_gbs_graph": round(2 * raw / (t_graph / 1e3) / 1e9, 1),
                "compressed_ratio": round(comp / raw, 5), "gpu_launches_per_pass": 3 + (1 if b.fit_mode == 0 else 0),
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    b.close()


def run_serve(args, world, rank, local):
    """64 resident LeCo-fix columns of 100M u64 keys (the 200M-key generator,
    one seed per column), a Poisson request stream: 80 % point lookups of
    log-uniform 1..65536 random indices, 20 % range scans of log-uniform
    16..1M values.  The same trace is served twice: by the continuous-batching
    server and by plain per-request launches (one request per launch, one at
    a time).  Latency = submit -> results in the client's pinned buffer."""
    import math
    import threading

    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    raws, cols = [], []
    for c in range(args.serve_cols):
        x = workloads.piecewise_linear_u64(args.serve_n, seed=100 + c + 1000 * rank, device=dev, noise_on="device")
        cols.append(lc.encode(x, lc.LINEAR, BS, lc.FIT_EXACT).compact())
        raws.append(x)
    torch.cuda.synchronize()
    comp = sum(c.nbytes for c in cols)
    rng = np.random.default_rng(17 + rank)
    reqs, n_look, n_scan = [], 0, 0
    for i in range(args.requests):
        ci = int(rng.integers(args.serve_cols))
        if rng.random() < 0.8:
            m = int(math.exp(rng.uniform(0, math.log(65536))))
            idx = torch.from_numpy(rng.integers(0, args.serve_n, m).astype(np.int64)).pin_memory()
            reqs.append((ci, idx, 0, m))
            n_look += m
        else:
            m = int(math.exp(rng.uniform(math.log(16), math.log(1_000_000))))
            reqs.append((ci, None, int(rng.integers(0, args.serve_n - m)), m))
            n_scan += m
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, args.requests))
    outs = [torch.empty(r[3], dtype=torch.int64).pin_memory() for r in reqs]

    def serve(**opt):
        srv = lc.Server(cols, **opt)
        # warm-up: a few requests through the same server
        for r, o in list(zip(reqs, outs))[:16]:
            srv.wait(srv.submit(r[0], o, idx=r[1], first=r[2], count=r[3]))
        srv.reset_stats()
        ids = []
        t0 = time.perf_counter()
        for (ci, idx, first, m), o, ta in zip(reqs, outs, arrivals):
            while time.perf_counter() - t0 < ta:
                pass
            ids.append(srv.submit(ci, o, idx=idx, first=first, count=m))
        srv.drain()
        span = time.perf_counter() - t0
        st = srv.stats()
        for i in ids:
            srv.wait(i)
        srv.close()
        lc.check()
        # verify a sample of the results against the stored keys
        for j in range(0, len(reqs), max(1, len(reqs) // 64)):
            ci, idx, first, m = reqs[j]
            exp = raws[ci][idx.to(dev)] if idx is not None else raws[ci][first:first + m]
            assert torch.equal(outs[j].to(dev), exp), "served result mismatch"
        return st, span

    with ClockSampler(local) as clk:
        st_b, span_b = serve(slots=4, max_requests_per_batch=1024)
    st_p, span_p = serve(slots=1, max_requests_per_batch=1)
    if rank == 0:
        arm = lambda st, span: {"lookups_per_s": round(st["lookups"] / span, 1), "scanned_values_per_s": round(st["scanned_values"] / span, 1),
                                "p50_us": round(st["p50_us"], 1), "p99_us": round(st["p99_us"], 1), "mean_us": round(st["mean_us"], 1),
                                "makespan_s": round(span, 4), "batches": st["batches"], "max_requests_in_batch": st["max_requests_in_batch"]}
        line = {"metric": "served random access: lookups/s and p50/p99 latency (continuous batching)",
                "value": round(st_b["lookups"] / span_b / 1e6, 3), "unit": "Mlookups/s", "n_gpus": world,
                "steps": args.requests, "warmup": 16, "ms_per_step": round(1e3 * span_b / args.requests, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": {"workload": f"{args.serve_cols} resident LeCo-fix columns x {args.serve_n} u64, Poisson "
                                       f"{args.rate:.0f} req/s, 80% lookups logU[1,65536], 20% scans logU[16,1M]",
                           "requests": args.requests, "lookups": n_look, "scanned_values": n_scan,
                           "compressed_bytes_resident": comp},
                "continuous_batching": arm(st_b, span_b), "per_request_launches": arm(st_p, span_p),
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)


def run_varlen(args, world, rank, local):
    """500M u64 keys from the regime-switching generator (linear, quadratic and
    flat regimes of geometric length, noise 2^8): variable-length segments from
    the host partitioner (coarse blocks of 2000 values, merge penalty 12 bits,
    as the reference's benchmark script runs its u64 variable-length codec) and
    the degree-2 polynomial codec with 8192-value blocks.  Times GPU encode,
    bulk decode, 2^24 random lookups and the compressed-domain sum."""
    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n if args.n != N_DEFAULT else 500_000_000
    x = workloads.regime_switching_u64(n, seed=5 + rank, device=dev)
    xh = x.cpu().numpy().view(np.uint64)
    stream = torch.cuda.current_stream()

    def ev_time(fn, reps=max(3, args.steps // 4)):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    t0 = time.perf_counter()
    starts = lc.varlen_partition(xh, n // 2000, 12)
    t_part = time.perf_counter() - t0
    pws = torch.empty(int(lc.lib().leco_varlen_partition_workspace_bytes(n, n // 2000)), dtype=torch.uint8, device=dev)
    dstarts = lc.varlen_partition_device(x, n // 2000, 12, ws=pws)
    assert np.array_equal(dstarts.cpu().numpy().view(np.uint64), starts), "GPU partition differs from the host's"
    t_part_dev = ev_time(lambda: lc.varlen_partition_device(x, n // 2000, 12, ws=pws), reps=3)
    del dstarts, pws
    vc = lc.varlen_encode(x, starts, lc.FIT_REFERENCE)
    out = torch.empty_like(x)
    idx = torch.randint(0, n, (RA_BATCH,), device=dev)
    ra = torch.empty(RA_BATCH, dtype=torch.int64, device=dev)
    res = {}
    clk = ClockSampler(local).__enter__()
    res["varlen"] = {
        "segments": int(len(starts)), "partition_host_s": round(t_part, 3), "host_threads": os.cpu_count(),
        "partition_gpu_ms": round(t_part_dev, 2),
        "encode_ms": round(ev_time(lambda: lc.varlen_encode(x, vc.starts, lc.FIT_REFERENCE,
                                                            max_segment_len=vc.max_segment_len)), 3),
        "decode_ms": round(ev_time(lambda: vc.decode(out=out)), 3),
        "gather_ms_2^24": round(ev_time(lambda: vc.gather(idx, out=ra)), 3),
        "sum_ms": round(ev_time(lambda: vc.sum()), 3), "compressed_ratio": round(vc.nbytes / (8 * n), 5)}
    assert torch.equal(vc.decode(out=out), x) and torch.equal(vc.gather(idx, out=ra), x[idx])
    assert vc.sum() == int(x.sum().item()) & 0xFFFFFFFFFFFFFFFF
    del vc
    pc = lc.encode(x, lc.POLY2, 8192, lc.FIT_REFERENCE)
    res["poly2_8192"] = {
        "encode_ms_reference_fit": round(ev_time(lambda: lc.encode(x, lc.POLY2, 8192, lc.FIT_REFERENCE, payload=pc.payload)), 3),
        "encode_ms_exact_fit": round(ev_time(lambda: lc.encode(x, lc.POLY2, 8192, lc.FIT_EXACT, payload=pc.payload)), 3),
        "decode_ms": 0.0, "gather_ms_2^24": 0.0, "sum_ms": 0.0}
    pc = lc.encode(x, lc.POLY2, 8192, lc.FIT_REFERENCE)
    res["poly2_8192"]["decode_ms"] = round(ev_time(lambda: pc.decode(out=out)), 3)
    res["poly2_8192"]["gather_ms_2^24"] = round(ev_time(lambda: pc.gather(idx, out=ra)), 3)
    res["poly2_8192"]["sum_ms"] = round(ev_time(lambda: pc.sum()), 3)
    res["poly2_8192"]["compressed_ratio"] = round(pc.nbytes / (8 * n), 5)
    assert torch.equal(pc.decode(out=out), x) and torch.equal(pc.gather(idx, out=ra), x[idx])
    clk.__exit__(None, None, None)
    assert pc.sum() == int(x.sum().item()) & 0xFFFFFFFFFFFFFFFF
    lc.check()
    for k in res:
        r = res[k]
        r["decode_gbs"] = round(8 * n / (r["decode_ms"] / 1e3) / 1e9, 1)
        r["mlookups_s"] = round(RA_BATCH / (r["gather_ms_2^24"] / 1e3) / 1e6, 1)
        r["sum_gbs"] = round(8 * n / (r["sum_ms"] / 1e3) / 1e9, 1)
    if rank == 0:
        line = {"metric": f"variable-length and degree-2 LeCo on {n // 1_000_000}M u64: decode GB/s, random access, sum",
                "value": res["varlen"]["decode_gbs"], "unit": "GB/s", "n_gpus": world, "steps": max(3, args.steps // 4),
                "warmup": 1, "ms_per_step": res["varlen"]["decode_ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": {"workload": f"{n} u64 regime-switching (linear/quadratic/flat, sigma 2^8); varlen: coarse "
                                       "blocks of 2000, delta 12; poly2: 8192-value blocks", "keys": n},
                "clocks": clk.summary(), **res}
        print(json.dumps(line), flush=True)


def run_filter(args, world, rank, local):
    """Predicate pushdown on the decode workload's column (200M sorted u64
    keys, LeCo-fix, 4096-value blocks): filter_range at 50% and 1%
    selectivity with the zone map, and a close-range filter, each timed on the
    device; the reference's own filter loop (compiled headers) is timed on the
    host cores over the first blocks, and the GPU's indices there are checked
    against it."""
    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    x = workloads.piecewise_linear_u64(n, seed=2 + rank, device=dev)
    col = lc.encode(x, lc.LINEAR, BS, lc.FIT_REFERENCE)
    zmin, zmax = col.zonemap()
    xh = x.cpu().numpy().view(np.uint64)
    pay, off = col.to_host()
    stream = torch.cuda.current_stream()
    out = torch.empty(n + col.nblocks, dtype=torch.int32, device=dev)
    ws = torch.empty(int(lc.lib().leco_filter_workspace_bytes(n, BS)), dtype=torch.uint8, device=dev)
    reps = max(3, args.steps // 4)

    def ev_time(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    zmax_h = to_np_u64(zmax)
    res = {}
    with ClockSampler(local) as clk:
        for q in (0.5, 0.99):
            f = int(np.quantile(xh[:: max(1, n // 1_000_000)], q))
            ms = ev_time(lambda: col.filter_range(f, zone_max=zmax, zone_min=zmin, out=out, ws=ws, sync=False))
            _, c = col.filter_range(f, zone_max=zmax, zone_min=zmin, out=out, ws=ws)
            # algorithmic bytes: per block its offset, header and zone-map pair; 4 B per index
            # written (blocks whose bounds straddle the filter also read their fields: a few here)
            alg = (8 + 17 + 16) * col.nblocks + 4 * c
            res[f"range_q{q}"] = {"filter": f, "matches": c, "ms": round(ms, 4),
                                  "gvalues_s": round(n / ms / 1e6, 2), "alg_bytes": alg,
                                  "alg_gbs": round(alg / ms / 1e6, 1),
                                  "frac_of_hbm": round(alg / ms / 1e6 / peaks()[0], 3)}
        f = res["range_q0.5"]["filter"]
        ms = ev_time(lambda: col.filter_range(f, out=out, ws=ws, sync=False))
        _, c = col.filter_range(f, out=out, ws=ws)
        res["range_q0.5_no_zone_map"] = {"filter": f, "matches": c, "ms": round(ms, 4),
                                         "gvalues_s": round(n / ms / 1e6, 2)}
        base, f1, f2 = (1 << 31) - 1, 1 << 29, 1 << 30
        ms = ev_time(lambda: col.filter_range_close(f1, f2, base, zone_min=zmin, out=out, ws=ws, sync=False))
        _, c = col.filter_range_close(f1, f2, base, zone_min=zmin, out=out, ws=ws)
        alg = (8 + 17 + 8) * col.nblocks + 4 * c
        res["close"] = {"base": base, "f1": f1, "f2": f2, "matches": c, "ms": round(ms, 4),
                        "gvalues_s": round(n / ms / 1e6, 2), "alg_bytes": alg, "alg_gbs": round(alg / ms / 1e6, 1)}
    lc.check()
    # the reference's filter loop on the host, over the first blocks (bounded sample)
    cpu = {}
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import Reference

        R = Reference()
        nbs = min(col.nblocks, 4096)
        ns = min(n, nbs * BS)
        spay, soff = pay[: int(off[nbs])], off[: nbs + 1]
        f = res["range_q0.5"]["filter"]
        t0 = time.perf_counter()
        want = R.filter_column(0, spay, soff, ns, 8, BS, f, zmax_h[:nbs])
        t_cpu = time.perf_counter() - t0
        got, c = col.filter_range(f, zone_max=zmax, zone_min=zmin, out=out, ws=ws)
        g = got.cpu().numpy().view(np.uint32)
        assert np.array_equal(g[: len(want)], want), "filter_range differs from the reference on the sample"
        cpu = {"value": round(ns / t_cpu / 1e9, 4), "unit": "Gvalues/s", "cores": 1, "kind": "reference",
               "sample": f"first {nbs} blocks ({ns} keys), filter_range at the median, zone map, 1 thread "
                         "(the reference's loop is single-threaded)"}
    except (FileNotFoundError, OSError) as e:
        cpu = {"unavailable": str(e)}
    if rank == 0:
        head = res["range_q0.5"]
        line = {"metric": f"LeCo-fix predicate pushdown on {n // 1_000_000}M sorted u64 keys: filter_range Gvalues/s",
                "value": head["gvalues_s"], "unit": "Gvalues/s", "n_gpus": world, "steps": reps,
                "warmup": max(3, args.warmup), "ms_per_step": head["ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": {"workload": f"{n} u64 piecewise-linear keys, LeCo-fix blocks of {BS}, zone map",
                           "keys": n, "compressed_bytes": int(off[-1])},
                "clocks": clk.summary(), "cpu_baseline": cpu, **res}
        print(json.dumps(line), flush=True)


def run_gather(args, world, rank, local):
    """Random access alone on the decode workload's column (200M u64 keys,
    LeCo-fix, 4096-value blocks): the column is encoded, the keys and every
    temporary are released, and each step is one batch of 2^24 uniform
    lookups.  The device then holds only the compressed column, its directory,
    the index sets and the output (under 1 GB), which keeps an ncu capture of
    the gather kernel at the full column size small."""
    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    x = workloads.piecewise_linear_u64(n, seed=2 + rank, device=dev)
    col = lc.encode(x, lc.LINEAR, BS, lc.FIT_REFERENCE).compact()
    idx_sets = [torch.randint(0, n, (RA_BATCH,), device=dev, dtype=torch.int64) for _ in range(2)]
    want = [x[i] for i in idx_sets]
    del x
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    out = torch.empty(RA_BATCH, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream()
    for i in range(max(3, args.warmup)):
        col.gather(idx_sets[i % 2], out=out)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            ev[i][0].record(stream)
            col.gather(idx_sets[i % 2], out=out)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    lc.check()
    assert torch.equal(out, want[(args.steps - 1) % 2]), "random access mismatch"
    ms = [a.elapsed_time(b) for a, b in ev]
    mean = float(np.mean(ms))
    peak, _ = peaks()
    if rank == 0:
        ach = RA_BATCH * RA_DRAM_BYTES / (mean / 1e3) / 1e9
        line = {"metric": "LeCo-fix batched random access on 200M u64 keys: Glookups/s",
                "value": round(RA_BATCH / mean / 1e6, 2), "unit": "Glookups/s", "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": round(mean, 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": {"workload": f"{n} u64 piecewise-linear keys, LeCo-fix blocks of {BS}, 2^24 uniform lookups",
                           "keys": n, "compressed_bytes": col.nbytes, "device_bytes_held": int(torch.cuda.memory_allocated())},
                "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(ach / peak, 4), "algorithmic_bytes_per_lookup": RA_DRAM_BYTES},
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)


def per_block_calls(lc, x, threads: int, nblocks: int = 200):
    """The reference drivers' calling pattern: one call per 4096-value u64 LeCo
    block.  Times the C ABI's per-block calls (leco_block_encode / _decode /
    _random: host buffers, one launch and a synchronize each) against the
    compiled reference's encodeArray8_int / decodeArray8 / randomdecodeArray8 on
    one host thread, on the same blocks (microseconds per call)."""
    import ctypes

    R = reference_lib()
    L = lc.lib()
    xh = x[: nblocks * BS].cpu().numpy().view(np.uint64)
    blocks = [np.ascontiguousarray(xh[i * BS:(i + 1) * BS]) for i in range(nblocks)]
    buf = np.zeros(BS * 8 * 2 + 256, np.uint8)
    out = np.zeros(BS, np.uint64)
    v = np.zeros(1, np.uint64)
    P = ctypes.c_void_p
    imgs = []
    t0 = time.perf_counter()
    for b in blocks:
        nb = L.leco_block_encode(0, 8, P(b.ctypes.data), BS, lc.FIT_REFERENCE, P(buf.ctypes.data))
        imgs.append(buf[:nb].tobytes())
    t_enc = (time.perf_counter() - t0) / nblocks
    t0 = time.perf_counter()
    for img in imgs:
        a = np.frombuffer(img, np.uint8)
        lc._check(L.leco_block_decode(0, 8, P(a.ctypes.data), len(img), BS, P(out.ctypes.data)))
    t_dec = (time.perf_counter() - t0) / nblocks
    assert np.array_equal(out, blocks[-1])
    t0 = time.perf_counter()
    for i, img in enumerate(imgs):
        a = np.frombuffer(img, np.uint8)
        lc._check(L.leco_block_random(0, 8, P(a.ctypes.data), len(img), BS, (i * 997) % BS, P(v.ctypes.data)))
    t_ra = (time.perf_counter() - t0) / nblocks
    res = {"blocks": nblocks, "gpu_encode_us": round(t_enc * 1e6, 1), "gpu_decode_us": round(t_dec * 1e6, 1),
           "gpu_random_us": round(t_ra * 1e6, 1)}
    if R is not None:
        t0 = time.perf_counter()
        rimgs = [R.encode_block(0, b) for b in blocks]
        res["reference_encode_us"] = round((time.perf_counter() - t0) / nblocks * 1e6, 1)
        assert rimgs == imgs, "per-block images differ from the reference's"
        t0 = time.perf_counter()
        for img in rimgs:
            R.decode_block(0, img, BS, 8)
        res["reference_decode_us"] = round((time.perf_counter() - t0) / nblocks * 1e6, 1)
        t0 = time.perf_counter()
        for i, img in enumerate(rimgs):
            R.random_block(0, img, (i * 997) % BS, 8)
        res["reference_random_us"] = round((time.perf_counter() - t0) / nblocks * 1e6, 1)
        res["reference_threads"] = 1
    return res


def run_codecs(args, world, rank, local):
    """Each fixed-block codec (LeCo linear, FOR, Delta, degree-2) on the decode
    workload's column (200M u64 keys, 4096-value blocks) and on its low 32 bits
    as u32: bulk decode, 2^24 uniform lookups (2^20 for Delta, whose random
    access walks the block), compressed-domain sum, encode (reference fit);
    every result checked against the keys."""
    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    x64 = workloads.piecewise_linear_u64(n, seed=2 + rank, device=dev)
    stream = torch.cuda.current_stream()

    def ev(fn, reps=5):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    res = {}
    with ClockSampler(local) as clk:
        for s, x in ((8, x64), (4, (x64 & 0xFFFFFFFF).to(torch.int32))):
            out = torch.empty_like(x)
            for name, codec in (("leco", lc.LINEAR), ("for", lc.FOR), ("delta", lc.DELTA), ("poly2", lc.POLY2)):
                col = lc.encode(x, codec, BS, lc.FIT_REFERENCE)
                m = (1 << 20) if codec == lc.DELTA else RA_BATCH
                idx = torch.randint(0, n, (m,), device=dev)
                ra = torch.empty(m, dtype=x.dtype, device=dev)
                r = {"ratio": round(col.nbytes / (n * s), 5),
                     "encode_ms": round(ev(lambda: lc.encode(x, codec, BS, lc.FIT_REFERENCE, payload=col.payload), 3), 4),
                     "decode_ms": round(ev(lambda: col.decode(out=out)), 4),
                     "sum_ms": round(ev(lambda: col.sum()), 4),
                     "lookups": m, "gather_ms": round(ev(lambda: col.gather(idx, out=ra)), 4)}
                col = lc.encode(x, codec, BS, lc.FIT_REFERENCE)
                assert torch.equal(col.decode(out=out), x), (name, s)
                assert torch.equal(col.gather(idx, out=ra), x[idx]), (name, s)
                mask = 0xFFFFFFFFFFFFFFFF if s == 8 else 0xFFFFFFFF
                want = int((x.to(torch.int64) & mask).sum().item()) & 0xFFFFFFFFFFFFFFFF
                assert col.sum() == want, (name, s)
                r["decode_gbs"] = round(n * s / r["decode_ms"] / 1e6, 1)
                r["mlookups_s"] = round(m / r["gather_ms"] / 1e3, 1)
                res[f"{name}_u{8 * s}"] = r
                del col
    lc.check()
    res["per_block_calls"] = per_block_calls(lc, x64, threads=host_threads())
    if rank == 0:
        head = res["delta_u64"]
        line = {"metric": f"fixed-block codecs on {n // 1_000_000}M keys: decode GB/s, random access, sum, encode",
                "value": head["decode_gbs"], "unit": "GB/s", "n_gpus": world, "steps": 5, "warmup": 2,
                "ms_per_step": head["decode_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u64+u32", "data": "synthetic",
                "config": {"workload": f"{n} piecewise-linear keys (u64, and their low 32 bits as u32), {BS}-value "
                                       "blocks, each codec; value = Delta u64 decode", "keys": n},
                "clocks": clk.summary(), **res}
        print(json.dumps(line), flush=True)


def run_encode(args, world, rank, local):
    """LeCo-fix u64 encode of prefixes of the decode workload's column (1 block up to
    the whole 200M keys, 4096-value blocks) with the reference fit and the exact fit:
    the reference fit's fixed cost is its sequential add chain, 4096 steps for any
    number of blocks.  CUDA events, mean of 10 encodes after 3 untimed; each
    column's decode is checked against its keys."""
    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    x = workloads.piecewise_linear_u64(args.n, seed=2 + rank, device=dev)
    stream = torch.cuda.current_stream()

    def ev(fn, reps=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps * 1e3

    res = {}
    nb_all = (args.n + BS - 1) // BS
    with ClockSampler(local) as clk:
        for nblk in (1, 32, 128, 1024, 4096, 12208, nb_all):
            n = min(args.n, nblk * BS)
            xs = x[:n]
            col = lc.encode(xs, lc.LINEAR, BS, lc.FIT_REFERENCE)
            assert torch.equal(col.decode(), xs)
            r = {"keys": n,
                 "reference_fit_us": round(ev(lambda: lc.encode(xs, lc.LINEAR, BS, lc.FIT_REFERENCE, payload=col.payload)), 1),
                 "exact_fit_us": round(ev(lambda: lc.encode(xs, lc.LINEAR, BS, lc.FIT_EXACT, payload=col.payload)), 1)}
            r["reference_fit_gbs"] = round(n * 8 / r["reference_fit_us"] / 1e3, 1)
            res[f"blocks_{nblk}"] = r
            del col
    lc.check()
    if rank == 0:
        head = res[f"blocks_{nb_all}"]
        line = {"metric": f"LeCo-fix u64 encode GB/s of input, {args.n // 1_000_000}M keys, reference fit",
                "value": head["reference_fit_gbs"], "unit": "GB/s", "n_gpus": world, "steps": 10, "warmup": 3,
                "ms_per_step": round(head["reference_fit_us"] / 1e3, 4), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": {"workload": f"prefixes of {args.n} u64 piecewise-linear keys, {BS}-value blocks, "
                                       "LeCo-fix encode, reference and exact fit", "keys": args.n},
                "clocks": clk.summary(), **res}
        print(json.dumps(line), flush=True)


def to_np_u64(t):
    return t.cpu().numpy().view(np.uint64)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "batch":
        run_batch(args, world, rank, local)
        return
    if args.workload == "serve":
        run_serve(args, world, rank, local)
        return
    if args.workload == "varlen":
        run_varlen(args, world, rank, local)
        return
    if args.workload == "filter":
        run_filter(args, world, rank, local)
        return
    if args.workload == "gather":
        run_gather(args, world, rank, local)
        return
    if args.workload == "codecs":
        run_codecs(args, world, rank, local)
        return
    if args.workload == "encode":
        run_encode(args, world, rank, local)
        return

    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist

    n = args.n
    x = workloads.piecewise_linear_u64(n, seed=2 + rank, device=dev)
    stream = torch.cuda.current_stream()
    t_enc = {}
    cols = {}
    for mode, name in ((lc.FIT_REFERENCE, "reference"), (lc.FIT_EXACT, "exact")):
        col = lc.encode(x, lc.LINEAR, BS, mode)  # warm-up + correctness
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        e0.record(stream)
        for _ in range(reps):
            col = lc.encode(x, lc.LINEAR, BS, mode, payload=col.payload)
        e1.record(stream)
        torch.cuda.synchronize()
        t_enc[name] = e0.elapsed_time(e1) / reps
        cols[name] = col
    col = cols["reference"]
    lc.check()
    y = col.decode()
    assert torch.equal(y, x), "decode mismatch"
    gidx = torch.randint(0, n, (RA_BATCH,), device=dev, dtype=torch.int64)
    assert torch.equal(col.gather(gidx), x[gidx]), "random access mismatch"
    assert col.sum() == int(x.sum().item()) & 0xFFFFFFFFFFFFFFFF, "sum mismatch"
    del cols
    torch.cuda.synchronize()

    out = torch.empty_like(x)
    ra_out = torch.empty(RA_BATCH, dtype=torch.int64, device=dev)
    idx_sets = [torch.randint(0, n, (RA_BATCH,), device=dev, dtype=torch.int64) for _ in range(4)]
    for i in range(args.warmup):
        col.decode(out=out)
        col.gather(idx_sets[i % 4], out=ra_out)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for i in range(args.steps):
            a, b, c = ev[i]
            a.record(stream)
            col.decode(out=out)
            b.record(stream)
            col.gather(idx_sets[i % 4], out=ra_out)
            c.record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
    total_ms = t_start.elapsed_time(t_end)
    dec_ms = [a.elapsed_time(b) for a, b, _ in ev]
    ra_ms = [b.elapsed_time(c) for _, b, c in ev]
    lc.check()
    assert torch.equal(out, x)

    if pg:
        import torch.distributed as dist

        t = torch.tensor([total_ms, float(np.mean(dec_ms)), float(np.mean(ra_ms))], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, dec_mean, ra_mean = t.tolist()
    else:
        dec_mean, ra_mean = float(np.mean(dec_ms)), float(np.mean(ra_ms))

    comp = col.nbytes
    dec_bytes = n * 8
    value = world * dec_bytes / (dec_mean / 1e3) / 1e9
    ra_rate = world * RA_BATCH / (ra_mean / 1e3) / 1e6
    peak, peak_kind = peaks()
    alg_bytes = comp + (col.nblocks + 1) * 8 + dec_bytes  # payload + offsets read, values written
    ra_alg = RA_BATCH * RA_DRAM_BYTES
    achieved = alg_bytes / (dec_mean / 1e3) / 1e9

    # end-to-end through the public host-buffer API: pinned compressed bytes in,
    # pinned decoded values out, copies inside the timed region
    e2e = e2e_ra = None
    if not args.no_e2e:
        pay_h, off_h = col.to_host()
        pay_pin = torch.empty(len(pay_h) + 64, dtype=torch.uint8).pin_memory()
        pay_pin[: len(pay_h)].copy_(torch.from_numpy(pay_h))
        off_pin = torch.from_numpy(off_h.view(np.int64)).pin_memory()
        out_pin = torch.empty(n, dtype=torch.int64).pin_memory()
        L = lc.lib()
        import ctypes

        P = ctypes.c_void_p
        args_e2e = (0, 8, P(pay_pin.data_ptr()), P(off_pin.data_ptr()), n, BS, P(out_pin.data_ptr()))
        for _ in range(2):
            lc._check(L.leco_decode_host(*args_e2e))
        # each call timed alone; the median of nine (the host link and host memory are
        # shared on this machine: single calls have taken up to 1.7x the median)
        rep_s = []
        for _ in range(9):
            t0 = time.perf_counter()
            lc._check(L.leco_decode_host(*args_e2e))
            rep_s.append(time.perf_counter() - t0)
        e2e_s = float(np.median(rep_s))
        # the host link this run had: a plain device->host copy of the decoded size into the same buffer
        link_s = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out_pin.copy_(x, non_blocking=True)
            torch.cuda.synchronize()
            link_s.append(time.perf_counter() - t0)
        lc._check(L.leco_decode_host(*args_e2e))
        assert torch.equal(out_pin, x.cpu())
        # random access end to end: leco_gather_host uploads the compressed column and the
        # indices, builds the directory, gathers and copies the values back, every call
        idx_pin = idx_sets[0].cpu().pin_memory()
        ra_pin = torch.empty(RA_BATCH, dtype=torch.int64).pin_memory()
        args_ra = (0, 8, P(pay_pin.data_ptr()), P(off_pin.data_ptr()), n, BS, P(idx_pin.data_ptr()), RA_BATCH,
                   P(ra_pin.data_ptr()))
        lc._check(L.leco_gather_host(*args_ra))
        ra_s = []
        for _ in range(9):
            t0 = time.perf_counter()
            lc._check(L.leco_gather_host(*args_ra))
            ra_s.append(time.perf_counter() - t0)
        assert torch.equal(ra_pin, x[idx_sets[0]].cpu())
        e2e_ra = {"value": round(world * RA_BATCH / float(np.median(ra_s)) / 1e6, 2), "unit": "Mlookups/s",
                  "api": "leco_gather_host (pinned host buffers; column, indices and results cross PCIe every call)",
                  "statistic": "median of 9 calls", "call_ms": [round(t * 1e3, 2) for t in ra_s],
                  "h2d_bytes_per_call": int(comp + off_h.nbytes + RA_BATCH * 8), "d2h_bytes_per_call": RA_BATCH * 8}
        del idx_pin, ra_pin
        e2e = {"value": round(world * dec_bytes / e2e_s / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": int(comp + off_h.nbytes), "d2h_bytes_per_step": int(dec_bytes),
               "api": "leco_decode_host (pinned host buffers)", "statistic": "median of 9 calls",
               "call_ms": [round(t * 1e3, 2) for t in rep_s],
               "plain_d2h_copy_gbs": round(dec_bytes / float(np.median(link_s)) / 1e9, 3)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        R = reference_lib()
        if R is None:
            cpu = {"unavailable": "oracle/_ref/libleco_ref.so was not built"}
        else:
            # the same column through the reference on the host cores; its stream must be
            # this library's, byte for byte, over the whole column
            threads = host_threads()
            xh = x.cpu().numpy().view(np.uint64)
            rpay, roff = R.encode_column(0, xh, BS, threads=threads)
            gp, go = col.to_host()
            cpu = cpu_reference_baseline(R, xh, rpay, roff, threads)
            cpu["gpu_stream_identical_full_column"] = bool(np.array_equal(go, roff) and np.array_equal(gp[: len(rpay)], rpay))
            cpu["reference_compressed_ratio"] = round(len(rpay) / (n * 8), 5)
            del xh, rpay, gp

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": decode_config(n, world),
            "decode_ms": round(dec_mean, 4),
            "ra_mlookups_s": round(ra_rate, 1),
            "ra_batch_p50_us": round(float(np.percentile(ra_ms, 50)) * 1e3, 1),
            "ra_batch_p99_us": round(float(np.percentile(ra_ms, 99)) * 1e3, 1),
            "decode_p50_ms": round(float(np.percentile(dec_ms, 50)), 4),
            "decode_p99_ms": round(float(np.percentile(dec_ms, 99)), 4),
            "encode_gbs": {"fit_reference": round(dec_bytes / (t_enc['reference'] / 1e3) / 1e9, 2),
                           "fit_exact": round(dec_bytes / (t_enc['exact'] / 1e3) / 1e9, 2)},
            "compressed_ratio": round(comp / dec_bytes, 5),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": profile_traffic(),
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                         "kernel": DECODE_KERNEL, "algorithmic_bytes_per_launch": int(alg_bytes)},
            "roofline_gather": {"bound": "hbm", "achieved": round(ra_alg / (ra_mean / 1e3) / 1e9, 1), "peak": peak,
                                "unit": "GB/s", "frac": round(ra_alg / (ra_mean / 1e3) / 1e9 / peak, 4),
                                "traffic": profile_traffic("gather_kernel_leco_u64_200M.txt"),
                                "kernel": "gather_kernel",
                                "algorithmic_bytes_per_lookup": RA_DRAM_BYTES,
                                "algorithmic_bytes_per_launch": int(ra_alg),
                                "note": "per lookup: 8 B index read + 8 B value written + one 32 B payload sector; "
                                        "the 32 B directory sector is L2-resident (48,829 blocks x 32 B = 1.6 MB) "
                                        "and not counted"},
            "e2e": e2e,
            "e2e_random_access": e2e_ra,
            "cpu_baseline": cpu,
            "gpu_launches": args.steps * 2,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if pg:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
