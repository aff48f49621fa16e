"""Benchmark of the Zstd L2 batched match-find workload on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gcz|reference]

Workload (one "step"): Zstd L2 match finding over a 1 GiB synthetic input
(seed 2; 40% order-1 Markov / 40% copies with offsets log-uniform to 8 MiB /
20% random; 16384 independent 64 KiB windows; search depth 64, which behaves
exactly like depth 16) in one launch, producing the ZSTD_Sequence records
ZSTD_compressSequences consumes.  Each rank processes its own 1 GiB shard
(weak scaling, no collective on the data path).

`value`: input GB/s (1e9 B/s) with the input already in HBM (device entry
point), K steps timed with CUDA events on the launch stream; the input is
larger than L2 (126 MB), so no flush is needed between steps.
`e2e`: the same metric through the host-buffer C-ABI call
(gcz_zstd_match_find) from pinned memory: H2D of the input, kernels, D2H of
the sequences and per-window offsets, all inside the timed region.
`--impl reference`: the reference's path timed on this box -- its CPU
restatement (oracle port, all host threads) as `value`, plus the reference's
own kernels (PTX compiled from its sources, JIT-loaded) on the same GPU.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-compressor_b200"))
sys.path.insert(0, ROOT)

METRIC = "input GB/s per B200 (match-find, end-to-end); p50/p99 latency; ratio, bit-exact"
WORKLOAD = "zstd_l2_batched_1gib"
N_BYTES = 1 << 30
SEED = 2
DEPTH = 64
HBM_FALLBACK = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gcz", choices=["gcz", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3, help="0 skips the end-to-end leg")
    ap.add_argument("--bytes", type=int, default=N_BYTES, help="input bytes per GPU (profiling runs use less)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configs' keys (zstd_l1_16mib, ...)")
    ap.add_argument("--no-heavy-configs", action="store_true", help="skip the uneven-batch and serving keys")
    ap.add_argument("--untuned", action="store_true", help="library default schedule, not gcz/tuned/<GPU>.json")
    ap.add_argument("--algo", type=int, default=2, help="1: fused single-warp kernels, 2: sweep + second stage")
    ap.add_argument("--workload", default="zstd", choices=["zstd", "lzma2", "serving", "uneven", "frames", "tune"],
                    help="zstd: Zstd L2 batched 1 GiB (the reported line); lzma2: LZMA2 L1 1 GiB, seed 3; "
                         "serving: open-loop request stream; uneven: many files in one launch")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving: requests per second (Poisson)")
    ap.add_argument("--duration", type=float, default=60.0, help="serving: seconds of arrivals")
    ap.add_argument("--max-request", type=int, default=256 << 20, help="serving: largest request size")
    ap.add_argument("--max-batch", type=int, default=256 << 20, help="serving: largest batch (bytes of input)")
    ap.add_argument("--serve-warmup", default="zstd,lzma2", choices=["zstd,lzma2", "lzma2,zstd", "none"],
                    help="serving: warm-up requests before the stream, in order")
    ap.add_argument("--files", type=int, default=4096, help="uneven: number of files")
    ap.add_argument("--max-file", type=int, default=64 << 20, help="uneven: largest file size")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_mod

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod
    else:
        torch.cuda.set_device(local)
    return world, rank, local, dist


def barrier(dist, torch, local):
    if dist is not None:
        dist.barrier(device_ids=[local])
    torch.cuda.synchronize()


def max_over_ranks(dist, torch, value):
    from gcz import shards

    return value if dist is None else shards.max_over_ranks(value)


def sum_over_ranks(dist, torch, value):
    from gcz import shards

    return value if dist is None else shards.sum_over_ranks(value)


def measured_traffic(workload, n):
    """DRAM bytes per step from the committed ncu summary (1 GiB step), or None."""
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if n != N_BYTES or not os.path.exists(tfile):
        return None
    with open(tfile) as f:
        return json.load(f).get(workload)


def cpu_library_baselines(data, kind, threads):
    """Stock compressors at matched levels on the host cores, per 64 KiB window
    like the match-finder levels: libzstd ZSTD_compress level 1 (Zstd) or
    liblzma raw LZMA2 preset 9 (LZMA2), `threads` windows at a time.  nvCOMP is
    not part of this image, so its L0 baseline is reported unavailable."""
    from concurrent.futures import ThreadPoolExecutor

    from gcz import codecs

    if kind == "xz":
        wins, kind = [], "lzma2"
    else:
        wins = [data[o:o + 65536] for o in range(0, data.size, 65536)]
    if kind == "zstd":
        fn = lambda w: len(codecs.zstd_compress_level(w.tobytes(), 1))  # noqa: E731
        name = "libzstd 1.5.5 ZSTD_compress level 1"
    else:
        fn = lambda w: len(codecs.lzma2_raw_compress(w.tobytes(), 9))  # noqa: E731
        name = "liblzma 5.4.5 raw LZMA2 preset 9"
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        out = sum(ex.map(fn, wins))
    dt = time.perf_counter() - t0
    res = {"nvcomp_zstd_l0": {"unavailable": "nvCOMP is not installed in this image"}}
    if wins:
        res[name] = {"gbs": round(data.size / dt / 1e9, 4), "ratio": round(out / data.size, 4), "threads": threads,
                     "sample_bytes": int(data.size)}
    if kind == "zstd":
        # whole buffer, level 1, ZSTD_c_nbWorkers = threads (libzstd's own multithreading)
        import ctypes
        L = codecs.zstd()
        L.ZSTD_compress2.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
        L.ZSTD_compress2.restype = ctypes.c_size_t
        cctx = L.ZSTD_createCCtx()
        L.ZSTD_CCtx_setParameter(cctx, 100, 1)  # ZSTD_c_compressionLevel
        L.ZSTD_CCtx_setParameter(cctx, 400, threads)  # ZSTD_c_nbWorkers
        dst = np.empty(L.ZSTD_compressBound(data.size), np.uint8)
        t0 = time.perf_counter()
        r = L.ZSTD_compress2(cctx, dst.ctypes.data, dst.size, data.ctypes.data, data.size)
        dt = time.perf_counter() - t0
        L.ZSTD_freeCCtx(cctx)
        if not L.ZSTD_isError(r):
            res["libzstd 1.5.5 whole buffer level 1, nbWorkers"] = {
                "gbs": round(data.size / dt / 1e9, 4), "ratio": round(r / data.size, 4), "threads": threads,
                "sample_bytes": int(data.size)}
    else:
        # liblzma's multithreaded stream encoder at preset 9 (xz 5.4.5 CLI), 8 MiB blocks
        import shutil
        if shutil.which("xz"):
            t0 = time.perf_counter()
            pr = subprocess.run(["xz", "-9", f"-T{threads}", "--block-size=8MiB", "-c"], input=data.tobytes(),
                                capture_output=True, check=True)
            dt = time.perf_counter() - t0
            res["liblzma 5.4.5 stream encoder mt preset 9 (xz), 8 MiB blocks"] = {
                "gbs": round(data.size / dt / 1e9, 4), "ratio": round(len(pr.stdout) / data.size, 4),
                "threads": threads, "sample_bytes": int(data.size)}
    return res


def cpu_oracle_time(data, depth, threads):
    from oracle import oracle as orc

    t0 = time.perf_counter()
    seqs, off = orc.zstd_sequences(data, depth, threads=threads)
    dt = time.perf_counter() - t0
    return dt, int(off[-1])


def link_time(torch, dev, h_in, d_in, h_out, d_out, out_bytes, piece=64 << 20, reps=3):
    """Seconds for the PCIe traffic of one end-to-end step with no kernels:
    the input's H2D in `piece`-sized copies on one stream while `out_bytes` of
    results go D2H in matching pieces on another (full duplex, as in the
    pipeline).  Mean of `reps` runs after one warm-up, CUDA events."""
    src, dst = h_in.view(torch.uint8).reshape(-1), d_in.view(torch.uint8).reshape(-1)
    osrc, odst = d_out.view(torch.uint8).reshape(-1)[:out_bytes], h_out.view(torch.uint8).reshape(-1)[:out_bytes]
    n = src.numel()
    k = max((n + piece - 1) // piece, 1)
    opiece = (out_bytes + k - 1) // k
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    times = []
    for r in range(reps + 1):
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s_in)
        s_out.wait_event(e0)
        for i in range(k):
            with torch.cuda.stream(s_in):
                dst[i * piece:(i + 1) * piece].copy_(src[i * piece:(i + 1) * piece], non_blocking=True)
            if i * opiece < out_bytes:
                with torch.cuda.stream(s_out):
                    odst[i * opiece:(i + 1) * opiece].copy_(osrc[i * opiece:(i + 1) * opiece], non_blocking=True)
        s_in.wait_stream(s_out)
        e1.record(s_in)
        torch.cuda.synchronize(dev)
        if r:
            times.append(e0.elapsed_time(e1) / 1e3)
    return sum(times) / len(times)


def load_tuned(ctx, args):
    """The schedule the autotuner saved for this GPU model (gcz/tuned/), or the
    library defaults; --algo 1 forces the fused kernels.  Returns the knobs
    in effect."""
    from gcz import autotune

    src = "defaults"
    if args.algo == 2 and not args.untuned:
        if autotune.apply_tuned(ctx) is not None:
            src = "gcz/tuned/" + os.path.basename(autotune.tuned_path(ctx.device))
    ctx.set_option("algo", args.algo)
    knobs = {k: ctx.query(k) for k in ("algo", "sweep_warps", "sweep_groups", "sweep_prefetch", "parse_seg", "parse_ctas",
                                       "lzma_ctas", "lzma_threads", "slice_windows")}
    knobs["source"] = src
    return knobs


def time_steps(torch, stream, steps, fn, flush=None):
    """Mean milliseconds per call of fn() with CUDA events on `stream`.  With no
    `flush`, one event pair brackets all steps (inputs larger than L2).  With a
    flush, every step has its own pair and flush() writes a buffer larger than
    L2 just before it, outside the pair."""
    if flush is None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps
    pairs = []
    for _ in range(steps):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        pairs.append((a, b))
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in pairs) / steps


def zstd_bit_exact(data, d_seqs, d_off, depth, nsample=512):
    """Sequences of `nsample` windows spread over the input (first and last
    included) against the oracle, outside every timed region."""
    import gcz
    from oracle import oracle as orc

    n = data.size
    B = gcz.num_windows(n)
    idx = np.unique(np.linspace(0, B - 1, min(nsample, B)).astype(np.int64))
    off = d_off.cpu().numpy().astype(np.int64)
    got = d_seqs[:int(off[-1])].cpu().numpy().view(np.uint32)
    sub = np.concatenate([data[i * 65536:(i + 1) * 65536] for i in idx])  # ragged last window stays last
    o_seqs, o_off = orc.zstd_sequences(sub, depth, threads=os.cpu_count() or 1)
    o_off = o_off.astype(np.int64)
    bad = [int(i) for k, i in enumerate(idx)
           if not np.array_equal(got[off[i]:off[i + 1]], o_seqs[o_off[k]:o_off[k + 1]])]
    return {"equal": not bad, "windows_checked": int(idx.size), "windows_differing": bad[:8],
            "sequences_checked": int(o_off[-1]), "against": "oracle/oracle.c (pinned to the reference kernels)"}


def zstd_ratio(ctx, data, depth, threads):
    """Compression ratio of Zstd frames built from these sequences by the
    reference's own coder loop (ZSTD_compressSequences per 64 KiB window,
    compress_zstd_custom.rs:115-199) on a sample, next to the same loop fed
    with the oracle's (= the reference kernels') sequences."""
    from gcz import codecs
    from oracle import oracle as orc

    level = 2 if depth > 16 else 1
    blob, _ = ctx.zstd_compress_frames(data, level, threads)
    o_seqs, o_off = orc.zstd_sequences(data, depth, threads=threads)
    comp = codecs.SequenceCompressor()
    ref = bytearray()
    for b in range(o_off.size - 1):
        ref += comp.compress(data[b * 65536:(b + 1) * 65536], o_seqs[int(o_off[b]):int(o_off[b + 1])])
    comp.close()
    r, rr = len(blob) / data.size, len(ref) / data.size
    return {"value": round(r, 5), "reference_value": round(rr, 5), "delta_pp": round(100 * (r - rr), 4),
            "frames_identical": bytes(blob.tobytes()) == bytes(ref), "sample_bytes": int(data.size),
            "coder": "libzstd 1.5.5 ZSTD_compressSequences per window (param 1001 = 0, session reset)"}


def zstd_config1(ctx, torch, dev, steps, warmup):
    """Config 1, Zstd L1 plain: one 16 MiB input (seed 1), depth 16.  The input
    fits in L2, so every timed step follows a 512 MiB write that flushes it.
    e2e and its per-call latency go through the host-buffer call."""
    import gcz

    n, depth = 16 << 20, 16
    data = gcz.gen_synthetic(1, n, 8 << 20)
    B = gcz.num_windows(n)
    d_in = torch.from_numpy(data).to(dev)
    cap = int(gcz.L.gcz_zstd_max_sequences(n))
    d_seqs = torch.empty((cap, 4), dtype=torch.int32, device=dev)
    d_off = torch.empty(B + 1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    flush_buf = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    def step():
        ctx.zstd_match_find_device(d_in.data_ptr(), n, depth, d_seqs.data_ptr(), cap, d_off.data_ptr(), sp)

    for _ in range(max(warmup, 3)):
        step()
    ctx.sync(sp)
    nseq = int(d_off[-1].item())
    ctx.profile_start()
    ms = time_steps(torch, stream, steps, step, flush=lambda: flush_buf.zero_())
    kern_ms, kern_launches, _ = ctx.profile_stop()
    ctx.sync(sp)
    del flush_buf
    h_in = torch.from_numpy(data).pin_memory()
    h_seqs = torch.empty((cap, 4), dtype=torch.int32).pin_memory()
    h_off = torch.empty(B + 1, dtype=torch.int64).pin_memory()

    def e2e_step():
        rc = gcz.L.gcz_zstd_match_find(ctx.handle, h_in.data_ptr(), n, depth, h_seqs.data_ptr(), cap,
                                       h_off.data_ptr())
        if rc != 0:
            raise RuntimeError(gcz.L.gcz_last_error(ctx.handle).decode())

    for _ in range(3):
        e2e_step()
    lat = []
    for _ in range(steps):
        t0 = time.perf_counter()
        e2e_step()
        lat.append((time.perf_counter() - t0) * 1e3)
    assert int(h_off[-1].item()) == nseq
    step_ms = kern_ms / max(kern_launches, 1)
    alg = n + 16 * nseq + 8 * B
    peak, peak_kind = peaks()
    return {
        "workload": "zstd_l1_16mib", "input_bytes": n, "windows": B, "search_depth": depth, "sequences": nseq,
        "value": round(n / (ms / 1e3) / 1e9, 3), "unit": "GB/s", "ms_per_step": round(ms, 4),
        "value_is": "device-resident, L2 flushed before every step",
        "e2e": {"value": round(n / (statistics.mean(lat) / 1e3) / 1e9, 3), "unit": "GB/s",
                "h2d_bytes_per_step": n, "d2h_bytes_per_step": 16 * nseq + 8 * (B + 1)},
        "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3), "p99": round(float(np.percentile(lat, 99)), 3),
                       "calls": len(lat), "of": "gcz_zstd_match_find on the 16 MiB host buffer"},
        "roofline": {"bound": "hbm", "achieved": round(alg / (step_ms / 1e3) / 1e9, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(alg / (step_ms / 1e3) / 1e9 / peak, 4),
                     "peak_source": f"{peak_kind} hbm_gbs", "kernel_ms_per_step": round(step_ms, 4),
                     "algorithmic_bytes_per_step": alg},
        "bit_exact": zstd_bit_exact(data, d_seqs, d_off, depth, nsample=B),
    }


def run_gcz(args):
    import torch
    import gcz

    world, rank, local, dist = dist_setup(args)
    dev = torch.device("cuda", local)
    ctx = gcz.Context(local)
    tuned = load_tuned(ctx, args)
    n = args.bytes
    data = gcz.gen_synthetic(SEED + 1000 * rank, n, 8 << 20)
    B = gcz.num_windows(n)
    d_in = torch.from_numpy(data).to(dev)
    # Output capacity: 4 bytes of records per input byte is ample for this input
    # (about one sequence per 50 bytes); an overflow would raise in ctx.sync.
    cap = min(int(gcz.L.gcz_zstd_max_sequences(n)), max(n // 4, 1024))
    d_seqs = torch.empty((cap, 4), dtype=torch.int32, device=dev)
    d_off = torch.empty(B + 1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step():
        ctx.zstd_match_find_device(d_in.data_ptr(), n, DEPTH, d_seqs.data_ptr(), cap, d_off.data_ptr(), sp)

    for _ in range(max(args.warmup, 3)):
        step()
    ctx.sync(sp)
    nseq = int(d_off[-1].item())

    # ---- device-resident timing
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, torch, local)
    with Clocks(local) as clk:
        ctx.profile_start()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        kern_ms, kern_launches, all_launches = ctx.profile_stop()
    barrier(dist, torch, local)
    ctx.sync(sp)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(dist, torch, ms)
    value = world * n * args.steps / (ms_max / 1e3) / 1e9

    # ---- end-to-end through the host-buffer C-ABI call (pinned buffers)
    e2e_value = link_value = e2e_packed = None
    e2e_lat = []
    if args.e2e_steps > 0:
        h_in = torch.from_numpy(data).pin_memory()
        h_seqs = torch.empty((nseq + 1024, 4), dtype=torch.int32).pin_memory()
        h_off = torch.empty(B + 1, dtype=torch.int64).pin_memory()

        def e2e_step():
            rc = gcz.L.gcz_zstd_match_find(ctx.handle, h_in.data_ptr(), n, DEPTH, h_seqs.data_ptr(), nseq + 1024,
                                           h_off.data_ptr())
            if rc != 0:
                raise RuntimeError(gcz.L.gcz_last_error(ctx.handle).decode())

        e2e_step()
        barrier(dist, torch, local)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            t1 = time.perf_counter()
            e2e_step()
            e2e_lat.append((time.perf_counter() - t1) * 1e3)
        e2e_s = time.perf_counter() - t0
        barrier(dist, torch, local)
        e2e_max = max_over_ranks(dist, torch, e2e_s)
        e2e_value = round(world * n * args.e2e_steps / e2e_max / 1e9, 3)
        assert int(h_off[-1].item()) == nseq
        link_s = max_over_ranks(dist, torch, link_time(torch, dev, h_in, d_in, h_seqs, d_seqs, 16 * nseq))
        link_value = round(world * n / link_s / 1e9, 3)
        # the same call with 8-byte records (gcz_zstd_match_find_packed): half the bytes back
        h_rec = torch.empty(nseq + 1024, dtype=torch.int64).pin_memory()

        def e2e_packed_step():
            rc = gcz.L.gcz_zstd_match_find_packed(ctx.handle, h_in.data_ptr(), n, DEPTH, h_rec.data_ptr(),
                                                  nseq + 1024, h_off.data_ptr())
            if rc != 0:
                raise RuntimeError(gcz.L.gcz_last_error(ctx.handle).decode())

        e2e_packed_step()
        barrier(dist, torch, local)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_packed_step()
        pk_s = max_over_ranks(dist, torch, time.perf_counter() - t0)
        barrier(dist, torch, local)
        assert int(h_off[-1].item()) == nseq
        pk_link_s = max_over_ranks(dist, torch, link_time(torch, dev, h_in, d_in, h_seqs, d_seqs, 8 * nseq))
        e2e_packed = {"value": round(world * n * args.e2e_steps / pk_s / 1e9, 3), "unit": "GB/s",
                      "h2d_bytes_per_step": n, "d2h_bytes_per_step": 8 * nseq + 8 * (B + 1),
                      "call": "gcz_zstd_match_find_packed (8-byte records the caller expands to ZSTD_Sequence)",
                      "link_bound": round(world * n / pk_link_s / 1e9, 3)}
        del h_in, h_seqs, h_off, h_rec

    # ---- roofline of the match-find step (match kernels + offset scan + compaction)
    peak, peak_kind = peaks()
    step_ms = kern_ms / max(kern_launches, 1)
    alg_bytes = n + 16 * nseq + 8 * B  # input once + ZSTD_Sequence out + counts/offsets
    achieved = alg_bytes / (step_ms / 1e3) / 1e9
    traffic = measured_traffic(WORKLOAD, n)

    cpu = libs = exact = ratio = configs = None
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        # outside the timed regions: bit-exactness on sampled windows, then the
        # frames' ratio through the reference's coder loop
        exact = zstd_bit_exact(data, d_seqs, d_off, DEPTH)
        ratio = zstd_ratio(ctx, data[:64 << 20], DEPTH, threads)
        del d_seqs, d_off, d_in
        torch.cuda.empty_cache()
        if not args.no_cpu_baseline:
            sample = data[:256 << 20]
            dt, _ = cpu_oracle_time(sample, DEPTH, threads)
            cpu = {"value": round(sample.size / dt / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                   "sample": f"first 256 MiB of the same 1 GiB input (4096 windows), oracle/oracle.c on "
                             f"{threads} threads"}
            libs = cpu_library_baselines(data[:256 << 20], "zstd", threads)
            small = data[:16 << 20]
            dt1, _ = cpu_oracle_time(small, DEPTH, 1)
            libs["oracle single thread"] = {"gbs": round(small.size / dt1 / 1e9, 4), "threads": 1,
                                            "sample_bytes": int(small.size)}
        if not args.no_configs:
            # BASELINE's other configs at their stated sizes, each outside the
            # headline's timed region: 1 (Zstd L1, 16 MiB), 3 (LZMA2 L1, 1 GiB),
            # 4 (4096 uneven files, ~28 GB), 5 (Poisson serving, 60 s)
            del data
            configs = {"zstd_l1_16mib": zstd_config1(ctx, torch, dev, args.steps, args.warmup)}
            configs["lzma2_l1_1gib"] = measure_lzma2(args, ctx, torch, dev, None, 1, 0, local,
                                                     cpu_legs=not args.no_cpu_baseline)
            if not args.no_heavy_configs:
                with Clocks(local) as c4:
                    configs["uneven_batch"] = measure_uneven(ctx, torch, args.steps, args.files, args.max_file)
                configs["uneven_batch"]["clocks"] = c4.summary()
                with Clocks(local) as c5:
                    configs["serving"] = measure_serving(ctx, torch, args.rate, args.duration, args.max_request,
                                                         args.max_batch)
                configs["serving"]["clocks"] = c5.summary()

    total_launches = sum_over_ranks(dist, torch, all_launches)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
            "value_is": "device-resident: input already in HBM, every match-find kernel of the step, CUDA events "
                        "on the launch stream; e2e is the same step through the host-buffer call",
            "config": {"workload": WORKLOAD, "input_bytes_per_gpu": n, "windows_per_gpu": B, "window": 65536,
                       "search_depth": DEPTH, "sequences_per_gpu": nseq, "parallelism": f"replicas{world}",
                       "algo": args.algo, "schedule": tuned, "fallback_windows": ctx.query("fallback_windows"),
                       "l2": "input 1 GiB > 126 MB L2, no flush needed"},
            "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": n,
                    "d2h_bytes_per_step": 16 * nseq + 8 * (B + 1),
                    "call": "gcz_zstd_match_find (pinned host input, ZSTD_Sequence records and offsets back)",
                    "link_bound": {"value": link_value, "unit": "GB/s",
                                   "what": "plain pinned copies of the step's bytes, no kernels: the H2D of the "
                                           "input in 64 MiB pieces with the sequence records' D2H on a second "
                                           "stream"},
                    "frac_of_link": round(e2e_value / link_value, 3) if e2e_value and link_value else None},
            "e2e_packed": e2e_packed,
            "latency_ms": ({"p50": round(float(np.percentile(e2e_lat, 50)), 3),
                            "p99": round(float(np.percentile(e2e_lat, 99)), 3), "calls": len(e2e_lat),
                            "of": "the 1 GiB host-buffer call (serving latency: --workload serving)"}
                           if e2e_lat else None),
            "ratio": ratio,
            "bit_exact": exact,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs", "kernel_ms_per_step": round(step_ms, 4),
                         "algorithmic_bytes_per_step": alg_bytes},
            "cpu_baseline": cpu,
            "cpu_libraries": libs,
            "configs": configs,
            "gpu_launches": int(total_launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def measure_lzma2(args, ctx, torch, dev, dist, world, rank, local, cpu_legs=True):
    """Config 3, LZMA2 L1: 1 GiB (seed 3, copy offsets to 128 MiB), 16384
    windows, per-position packed matches + per-window has-match byte, timed
    device-resident; e2e through the host-buffer call, both as the triage the
    encoder consumes and with the per-position results."""
    import gcz

    n = args.bytes
    data = gcz.gen_synthetic(3 + 1000 * rank, n, 128 << 20)
    B = gcz.num_windows(n)
    d_in = torch.from_numpy(data).to(dev)
    d_packed = torch.empty(n, dtype=torch.int32, device=dev)
    d_has = torch.empty(B, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step():
        ctx.lzma2_match_find_device(d_in.data_ptr(), n, 32, d_packed.data_ptr(), d_has.data_ptr(), sp)

    for _ in range(max(args.warmup, 3)):
        step()
    ctx.sync(sp)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, torch, local)
    with Clocks(local) as clk:
        ctx.profile_start()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        kern_ms, kern_launches, all_launches = ctx.profile_stop()
    barrier(dist, torch, local)
    ctx.sync(sp)
    ms_max = max_over_ranks(dist, torch, e0.elapsed_time(e1))
    value = world * n * args.steps / (ms_max / 1e3) / 1e9
    # bit-exact on sampled windows against the oracle, outside the timed region
    from oracle import oracle as orc
    idx = np.unique(np.linspace(0, B - 1, min(512, B)).astype(np.int64))
    got = d_packed.cpu().numpy().view(np.uint32)
    has = d_has.cpu().numpy()
    sub = np.concatenate([data[i * 65536:(i + 1) * 65536] for i in idx])
    o_packed = orc.lzma_packed(sub, 32, threads=os.cpu_count() or 1)
    o_has = orc.has_matches(o_packed, sub.size)
    bad = [int(i) for k, i in enumerate(idx)
           if not np.array_equal(got[i * 65536:i * 65536 + 65536], o_packed[k * 65536:k * 65536 + 65536])
           or has[i] != o_has[k]]
    exact = {"equal": not bad, "windows_checked": int(idx.size), "windows_differing": bad[:8],
             "against": "oracle/oracle.c (pinned to the reference kernels)"}
    del got
    e2e_value = e2e_packed = None
    if args.e2e_steps > 0:
        h_in = torch.from_numpy(data).pin_memory()
        h_packed = torch.empty(n, dtype=torch.int32).pin_memory()
        h_has = torch.empty(B, dtype=torch.uint8).pin_memory()

        def e2e_run(packed_ptr):
            def e2e_step():
                rc = gcz.L.gcz_lzma2_match_find(ctx.handle, h_in.data_ptr(), n, 32, packed_ptr, h_has.data_ptr())
                if rc != 0:
                    raise RuntimeError(gcz.L.gcz_last_error(ctx.handle).decode())

            e2e_step()
            barrier(dist, torch, local)
            t0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                e2e_step()
            dt = time.perf_counter() - t0
            barrier(dist, torch, local)
            return round(world * n * args.e2e_steps / max_over_ranks(dist, torch, dt) / 1e9, 3)

        # The LZMA2 L1+ encoder consumes one bit per window (compress_lzma2_custom.rs:577):
        # the triage call (packed = NULL) is its end-to-end path; the per-position
        # results through the same call are reported beside it.
        e2e_value = e2e_run(None)
        has_triage = h_has.clone()
        e2e_packed = e2e_run(h_packed.data_ptr())
        assert torch.equal(has_triage, h_has)
        del h_in, h_packed, h_has
    del d_in, d_packed, d_has
    torch.cuda.empty_cache()
    libs = l1 = None
    if rank == 0 and world == 1 and cpu_legs:
        threads = os.cpu_count() or 1
        sample = data[:16 << 20]
        libs = cpu_library_baselines(sample, "lzma2", threads)
        mt = cpu_library_baselines(data[:64 << 20], "xz", threads)
        libs.update({k: v for k, v in mt.items() if k.startswith("liblzma 5.4.5 stream")})
        # LZMA2 L1 end to end on the sample: GPU triage, then the preset-9 coder
        # pool on every window with a match (compress_lzma2_custom.rs:570-597)
        from gcz import formats
        t0 = time.perf_counter()
        blob = formats.compress_lzma2(sample.tobytes(), device_id=local, workers=threads)
        dt = time.perf_counter() - t0
        l1 = {"gbs": round(sample.size / dt / 1e9, 4), "ratio": round(len(blob) / sample.size, 4),
              "coder_threads": threads, "sample_bytes": int(sample.size)}
    peak, peak_kind = peaks()
    step_ms = kern_ms / max(kern_launches, 1)
    alg_bytes = n + 4 * n + B  # input once + packed matches + has-match bytes
    achieved = alg_bytes / (step_ms / 1e3) / 1e9
    return {
        "metric": "input GB/s per B200 (LZMA2 L1 match-find)", "value": round(value, 3), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator)", "value_is": "device-resident, input 1 GiB > L2",
        "config": {"workload": "lzma2_l1_1gib", "input_bytes_per_gpu": n, "windows_per_gpu": B, "algo": args.algo},
        "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": n, "d2h_bytes_per_step": B,
                "call": "gcz_lzma2_match_find(packed=NULL): per-window has-match bytes"},
        "e2e_packed": {"value": e2e_packed, "unit": "GB/s", "h2d_bytes_per_step": n,
                       "d2h_bytes_per_step": 4 * n + B, "call": "gcz_lzma2_match_find: per-position matches"},
        "bit_exact": exact,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": measured_traffic("lzma2_l1_1gib", n),
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "kernel_ms_per_step": round(step_ms, 4), "algorithmic_bytes_per_step": alg_bytes},
        "cpu_libraries": libs, "lzma2_l1_nvlz_end_to_end": l1,
        "gpu_launches": int(all_launches), "clocks": clk.summary()}


def run_lzma2(args):
    """LZMA2 L1 workload on its own line (config 3)."""
    import torch
    import gcz

    world, rank, local, dist = dist_setup(args)
    dev = torch.device("cuda", local)
    ctx = gcz.Context(local)
    tuned = load_tuned(ctx, args)
    line = measure_lzma2(args, ctx, torch, dev, dist, world, rank, local, cpu_legs=not args.no_cpu_baseline)
    line["config"]["schedule"] = tuned
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def fill_pool(pool_np, seed, block=16 << 20):
    """A pinned payload pool of `block`-sized spans, each from the generator
    with its own Dirichlet(1,1,1) mix (Markov / copy / random fractions)."""
    import gcz
    from concurrent.futures import ThreadPoolExecutor

    n = pool_np.size
    nblk = (n + block - 1) // block
    mixes = np.random.default_rng(seed).dirichlet([1, 1, 1], size=nblk)

    def gen(i):
        o = i * block
        gcz.gen_synthetic(seed * 100003 + i, min(block, n - o), 8 << 20, tuple(mixes[i]), out=pool_np[o:o + block])

    with ThreadPoolExecutor(os.cpu_count() or 4) as ex:
        list(ex.map(gen, range(nblk)))


def measure_serving(ctx, torch, rate, duration, max_request, max_batch, budget=120 * 10**9, pool_bytes=4 << 30,
                    warm="zstd,lzma2"):
    """Config 5, serving: an open-loop Poisson stream against the request loop.
    Request sizes log-uniform 4 KiB..max_request, 70% Zstd L1 / 20% Zstd L2 /
    10% LZMA2 L1 (has-match bytes, what the LZMA2 encoder reads).  Payloads are
    slices of a pinned pool made of 16 MiB spans with their own Dirichlet mix;
    results go to a pinned ring freed in completion order.  Reports offered and
    served GB/s and the submit-to-completion p50/p99 the loop measured.
    `warm` names the kinds of the warm-up requests, in order ("none": no
    warm-up, the stream's first requests pay the first launches)."""
    import threading
    import gcz
    from gcz import serving

    pool = torch.empty(pool_bytes, dtype=torch.uint8, pin_memory=True)
    pool_np = pool.numpy()
    fill_pool(pool_np, 5)
    srv = serving.Server(ctx, hbm_budget=budget, max_batch_bytes=max_batch)
    slots, dev_bytes = srv.info()
    rng = np.random.default_rng(11)
    count = int(rate * duration)
    gaps = rng.exponential(1.0 / rate, size=count)
    sizes = np.exp(rng.uniform(np.log(4096), np.log(max_request), size=count)).astype(np.int64)
    u = rng.random(count)
    kinds = np.where(u < 0.9, serving.ZSTD, serving.LZMA2)
    depths = np.where(u < 0.7, 16, np.where(u < 0.9, 64, 32))
    offs = (rng.random(count) * (pool_bytes - sizes)).astype(np.int64)
    q = []
    lock = threading.Condition()
    # Zstd results get room for n/16 + 1024 sequences (this input averages one
    # sequence per ~50 bytes); a full ring holds the submitter back.
    ring_n = 8 << 30
    ring = torch.empty(ring_n, dtype=torch.uint8, pin_memory=True).numpy()
    rs = {"head": 0, "tail": 0, "stalls": 0}
    ring_cv = threading.Condition()

    def ring_alloc(nbytes):
        nbytes = (nbytes + 255) & ~255
        with ring_cv:
            h = rs["head"]
            if h % ring_n + nbytes > ring_n:
                h += ring_n - h % ring_n  # skip the ring's end
            if h + nbytes - rs["tail"] > ring_n:
                rs["stalls"] += 1
            while h + nbytes - rs["tail"] > ring_n:
                ring_cv.wait()
            rs["head"] = h + nbytes
            return h % ring_n, h + nbytes

    def ring_free(end):
        with ring_cv:
            rs["tail"] = end
            ring_cv.notify_all()

    lats = np.zeros(count)

    def waiter():
        i = 0
        while i < count:
            with lock:
                while len(q) <= i:
                    lock.wait()
                r, end = q[i]
            srv.wait(r)
            lats[i] = r.latency_ms
            ring_free(end)
            q[i] = None
            i += 1

    kinds_warm = {"zstd": serving.ZSTD, "lzma2": serving.LZMA2}
    if warm != "none":
        srv.warm_up(tuple(kinds_warm[k] for k in warm.split(",")))
    base = srv.stats()
    wt = threading.Thread(target=waiter)
    wt.start()
    t0 = time.perf_counter()
    nxt = t0
    late = 0.0
    for i in range(count):
        nxt += gaps[i]
        d = nxt - time.perf_counter()
        if d > 0:
            time.sleep(d)
        else:
            late = max(late, -d)
        n = int(sizes[i])
        nb = gcz.num_windows(n)
        if kinds[i] == serving.ZSTD:
            cap = n // 16 + 1024
            na, nbb = cap * 16, ((nb + 1) * 8 + 255) & ~255
            o, end = ring_alloc(na + nbb)
            r = srv.submit(serving.ZSTD, pool_np[offs[i]:offs[i] + n], int(depths[i]),
                           out_a=ring[o:o + na].view(np.uint32).reshape(cap, 4), cap=cap,
                           out_b=ring[o + na:o + na + (nb + 1) * 8].view(np.uint64))
        else:
            o, end = ring_alloc(nb)
            r = srv.submit(serving.LZMA2, pool_np[offs[i]:offs[i] + n], 32, out_b=ring[o:o + nb], packed=False)
        with lock:
            q.append((r, end))
            lock.notify()
    t_sub = time.perf_counter() - t0
    wt.join()
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    del ring, pool
    done = st["bytes"] - base["bytes"]
    return {
        "workload": "serving_poisson", "value": round(done / wall / 1e9, 3), "unit": "GB/s",
        "value_is": "input bytes completed / wall time from the first arrival to the last completion",
        "offered_gbs": round(float(sizes.sum()) / duration / 1e9, 3),
        "latency_ms": {"p50": round(float(np.percentile(lats, 50)), 3), "p99": round(float(np.percentile(lats, 99)), 3),
                       "max": round(float(lats.max()), 3), "of": "submit to completion, every request"},
        "rate_per_s": rate, "duration_s": duration, "requests": count, "size_range": [4096, max_request],
        "mix": "70% Zstd L1, 20% Zstd L2, 10% LZMA2 L1 (has-match bytes); 16 MiB pool spans with Dirichlet(1,1,1) mixes",
        "hbm_budget_bytes": budget, "max_batch_bytes": max_batch, "slots": slots, "device_bytes_held": dev_bytes,
        "batches": st["batches"] - base["batches"], "completed": st["completed"] - base["completed"],
        "submit_seconds": round(t_sub, 3), "wall_s": round(wall, 3), "ring_stalls": rs["stalls"],
        "max_submit_lag_s": round(late, 4), "warm_up": warm, "status": st["status"]}


def run_serving(args):
    """Config 5 on its own line (see measure_serving)."""
    import torch
    import gcz

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ctx = gcz.Context(local)
    with Clocks(local) as clk:
        res = measure_serving(ctx, torch, args.rate, args.duration, args.max_request, args.max_batch,
                              warm=args.serve_warmup)
    line = {"metric": "serving input GB/s per B200 (match-find, p50/p99 latency)", "n_gpus": 1,
            "higher_is_better": True, "dtype": "u8", "data": "synthetic (seeded pool)", **res,
            "config": {"workload": "serving_poisson"}, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def measure_uneven(ctx, torch, steps, files=4096, max_file=64 << 20, part_windows=32768):
    """Config 4, uneven batch: `files` files of log-uniform size 4 KiB..max_file
    with per-file Dirichlet(1,1,1) mixes, Zstd L1 (depth 16), device-resident.
    The slab does not fit one launch's scratch at 18 device bytes per input
    byte, so its window table is cut into parts of at most `part_windows`
    windows; all parts' launches are captured in one CUDA graph, and a step is
    one replay of it (every window of every file)."""
    import gcz
    from concurrent.futures import ThreadPoolExecutor

    sizes, mix = gcz.gen_file_sizes(4, files, 4096, max_file)
    foff, wins, slab = gcz.batch_layout(sizes)
    total = int(np.sum(sizes))
    dev = torch.device("cuda", torch.cuda.current_device())
    d_slab = torch.empty(slab + 64, dtype=torch.uint8, device=dev)
    # generate file by file into a pinned staging buffer, copy into the slab
    stage_n = 1 << 30
    stage = torch.empty(stage_n, dtype=torch.uint8, pin_memory=True)
    st_np = stage.numpy()
    order = np.argsort(foff)
    i = 0
    with ThreadPoolExecutor(os.cpu_count() or 4) as ex:
        while i < len(order):
            j, used, jobs = i, 0, []
            while j < len(order) and (used + int(sizes[order[j]]) <= stage_n or j == i):
                f = int(order[j])
                jobs.append((f, used))
                used += (int(sizes[f]) + 15) & ~15
                j += 1
            list(ex.map(lambda fu: gcz.gen_synthetic(4000 + fu[0], int(sizes[fu[0]]), 8 << 20, tuple(mix[fu[0]]),
                                                     out=st_np[fu[1]:fu[1] + int(sizes[fu[0]])]), jobs))
            for f, u in jobs:
                o, sz = int(foff[f]), int(sizes[f])
                d_slab[o:o + sz].copy_(stage[u:u + sz], non_blocking=True)
            torch.cuda.synchronize()
            i = j
    del stage, st_np
    # parts: contiguous window ranges, offsets rebased to the part's first byte
    parts = []
    for w0 in range(0, wins.size, part_windows):
        w1 = min(wins.size, w0 + part_windows)
        pw = wins[w0:w1].copy()
        base = int(pw["offset"][0])
        pw["offset"] -= base
        pbytes = int(pw["offset"][-1]) + int(pw["size"][-1])
        cap = sum(int(gcz.L.gcz_zstd_max_sequences(int(x))) for x in pw["size"]) // 4 + 1024
        parts.append({"base": base, "bytes": pbytes, "wins": torch.from_numpy(pw.view(np.uint8)).to(dev),
                      "n": int(pw.size), "cap": cap,
                      "seqs": torch.empty((cap, 4), dtype=torch.int32, device=dev),
                      "off": torch.empty(int(pw.size) + 1, dtype=torch.int64, device=dev)})
    st = torch.cuda.current_stream()

    def launch_all(stream):
        for p in parts:
            ctx.zstd_match_find_batch_device(d_slab.data_ptr() + p["base"], p["bytes"], p["wins"].data_ptr(), p["n"],
                                             16, p["seqs"].data_ptr(), p["cap"], p["off"].data_ptr(), stream)

    for _ in range(3):  # also sizes every scratch buffer, so the captured launches allocate nothing
        launch_all(st.cuda_stream)
    ctx.sync(st.cuda_stream)
    nseq = sum(int(p["off"][-1].item()) for p in parts)
    cs = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(cs):
        with torch.cuda.graph(g, stream=cs):
            launch_all(cs.cuda_stream)
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    ctx.sync(st.cuda_stream)
    ms = time_steps(torch, st, steps, g.replay)
    ctx.sync(st.cuda_stream)
    # one small file and the largest file against the oracle, outside the timed region
    from oracle import oracle as orc
    checked = []
    first_win = np.searchsorted(wins["offset"], foff)
    nwins = np.array([gcz.num_windows(int(x)) for x in sizes])
    inside = (first_win // part_windows) == ((first_win + nwins - 1) // part_windows)  # not cut by a part boundary
    by_size = [int(f) for f in np.argsort(sizes) if inside[f]]
    for f in (by_size[0], by_size[-1]):  # the smallest and the largest file that one part holds whole
        w_first, nwf = int(first_win[f]), int(nwins[f])
        k = w_first // part_windows
        p = parts[k]
        lw = w_first - k * part_windows
        off = p["off"].cpu().numpy().astype(np.int64)
        got = p["seqs"][off[lw]:off[lw + nwf]].cpu().numpy().view(np.uint32)
        data = d_slab[int(foff[f]):int(foff[f]) + int(sizes[f])].cpu().numpy()
        o_seqs, _ = orc.zstd_sequences(data, 16, threads=os.cpu_count() or 1)
        checked.append({"file": f, "bytes": int(sizes[f]), "equal": bool(np.array_equal(got, o_seqs))})
    res = {"workload": "uneven_batch", "value": round(total / (ms / 1e3) / 1e9, 3), "unit": "GB/s",
           "ms_per_step": round(ms, 3), "value_is": "device-resident, one CUDA graph replay per step",
           "files": files, "size_range": [4096, max_file], "input_bytes": total, "slab_bytes": int(slab),
           "windows": int(wins.size), "launch_parts": len(parts), "part_windows": part_windows,
           "sequences": nseq, "mix": "Dirichlet(1,1,1) per file", "search_depth": 16,
           "bit_exact": {"equal": all(c["equal"] for c in checked), "files_checked": checked,
                         "against": "oracle/oracle.c"}}
    del parts, d_slab, g
    torch.cuda.empty_cache()
    return res


def run_uneven(args):
    """Config 4 on its own line (see measure_uneven)."""
    import torch
    import gcz

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ctx = gcz.Context(local)
    with Clocks(local) as clk:
        res = measure_uneven(ctx, torch, args.steps, args.files, args.max_file)
    print(json.dumps({"metric": "uneven-batch input GB/s per B200 (Zstd L1 match-find)", **res,
                      "config": {"workload": "uneven_batch"}, "clocks": clk.summary()}), flush=True)


def run_reference(args):
    """Reference arm: the reference's path on this box, on the same workload
    (1 GiB, seed 2, depth 64), the same --steps/--warmup and the same metric.
    The reference has no CPU match finder, so `value` is its kernels' CPU
    restatement (the oracle port) on all host threads over the whole 1 GiB per
    step; `reference_kernels_b200` times the reference's own kernels (PTX from
    its sources, driver JIT) on the same GPU.  Nothing here loads libgcz.so:
    the input comes from the oracle's own build of the generator."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as orc

    n = args.bytes
    data = orc.gen_synthetic(SEED, n, 8 << 20)
    threads = os.cpu_count() or 1
    for _ in range(max(args.warmup, 3)):
        cpu_oracle_time(data, DEPTH, threads)
    times = [cpu_oracle_time(data, DEPTH, threads)[0] for _ in range(args.steps)]
    value = n * len(times) / sum(times) / 1e9
    refk = reference_kernels(data)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(sum(times) / len(times) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOAD, "input_bytes_per_gpu": n, "windows_per_gpu": (n + 65535) // 65536,
                   "window": 65536, "search_depth": DEPTH},
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"the whole {n >> 20} MiB input every step, oracle/oracle.c on {threads} threads "
                                   "(the reference has no CPU match finder; its kernels are timed below)"},
        "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_kernels_b200": refk,
    }
    print(json.dumps(line), flush=True)


def reference_kernels(data):
    """The reference's own kernels (PTX from its sources and flags, JIT on this
    GPU, grid = windows, block = 256) on the same bytes:
    - zstd_match_find over the whole input in one grid (kernel only), and its
      adapter pattern per 8 MiB chunk (alloc_zeros + H2D + launch + D2H of the
      sequence buffer, compress_zstd_custom.rs:79-116) on 128 MiB;
    - lzma2_match_find per 128 MiB pipeline chunk (pipeline_lzma2.rs:116-190)
      over the LZMA2 input (seed 3, offsets to 128 MiB), kernel only, and its
      adapter pattern (alloc_zeros of 64 B + 4 B per byte, H2D, launch, D2H of
      both buffers, compress_lzma2_custom.rs:508-540) on one chunk."""
    try:
        from oracle import ref_kernels
        from oracle import oracle as orc
        import torch

        if not ref_kernels.available() or not torch.cuda.is_available():
            return {"unavailable": "oracle/_ref not built or no GPU"}
        rk = ref_kernels.RefKernels(0)
        n = data.size
        d_in = rk.to_device(data)
        bufs = rk.zstd_alloc(n)
        rk.zstd_launch(d_in, n, bufs, DEPTH)  # JIT + warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rk.zstd_launch(d_in, n, bufs, DEPTH)
        e1.record()
        torch.cuda.synchronize()
        k_ms = e0.elapsed_time(e1)
        del bufs, d_in
        torch.cuda.empty_cache()
        chunk = 8 << 20
        sample = data[:128 << 20]
        t0 = time.perf_counter()
        for off in range(0, sample.size, chunk):
            part = sample[off:off + chunk]
            d = rk.to_device(part)
            b = rk.zstd_alloc(part.size)
            rk.zstd_launch(d, part.size, b, DEPTH)
            b[0].cpu()
            b[2].cpu()
        torch.cuda.synchronize()
        a_s = time.perf_counter() - t0
        res = {"zstd_kernel_only_gbs": round(n / (k_ms / 1e3) / 1e9, 4), "zstd_kernel_ms": round(k_ms, 3),
               "zstd_adapter_pattern_gbs": round(sample.size / a_s / 1e9, 4),
               "note": "PTX from the reference's own sources and flags, driver JIT; grid = windows, block = 256"}
        del sample
        torch.cuda.empty_cache()
        # LZMA2: 128 MiB chunks, one 8.5 GiB output allocation reused for the kernel-only timing
        lz = orc.gen_synthetic(3, n, 128 << 20)
        lchunk = 128 << 20
        lb = rk.lzma_alloc(min(lchunk, n))
        d = rk.to_device(lz[:lchunk])
        rk.lzma_launch(d, min(lchunk, n), lb)  # JIT + warm-up
        torch.cuda.synchronize()
        l_ms = 0.0
        for off in range(0, n, lchunk):
            part = lz[off:off + lchunk]
            d = rk.to_device(part)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            rk.lzma_launch(d, part.size, lb)
            b.record()
            torch.cuda.synchronize()
            l_ms += a.elapsed_time(b)
        del lb, d
        torch.cuda.empty_cache()
        t0 = time.perf_counter()
        part = lz[:lchunk]
        d = rk.to_device(part)
        b = rk.lzma_alloc(part.size)
        rk.lzma_launch(d, part.size, b)
        b[0].cpu()
        b[1].cpu()
        torch.cuda.synchronize()
        la_s = time.perf_counter() - t0
        del b, d
        torch.cuda.empty_cache()
        res.update({"lzma2_kernel_only_gbs": round(n / (l_ms / 1e3) / 1e9, 4), "lzma2_kernel_ms": round(l_ms, 3),
                    "lzma2_adapter_pattern_gbs": round(part.size / la_s / 1e9, 4),
                    "lzma2_note": "8 launches of 128 MiB (2048 windows each) over the 1 GiB LZMA2 input; the "
                                  "adapter pattern moves 8.5 GiB of zero-filled slots and counts back per chunk"})
        return res
    except Exception as e:  # report, never fail the arm
        return {"unavailable": f"{type(e).__name__}: {e}"}


def run_frames(args):
    """Zstd L2 frames end to end: 1 GiB host input (seed 2) -> one Zstd frame
    per 64 KiB window.  `value`: everything on the GPU
    (gcz_zstd_compress_frames_gpu: copy-in, match finding, entropy stage,
    copy-out of 32 MiB slices over four streams).  Beside it: the libzstd coder
    path (gcz_zstd_compress_frames: GPU sequences, ZSTD_compressSequences on
    all host cores) and, on a 64 MiB sample, the reference's schedule (GPU
    sequences, then one thread encoding window after window,
    compress_zstd_custom.rs:115-199)."""
    import ctypes
    import torch
    import gcz
    from gcz import codecs

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ctx = gcz.Context(local)
    n = args.bytes
    data = gcz.gen_synthetic(SEED, n, 8 << 20)
    h_in = torch.from_numpy(data).pin_memory()
    bound = int(gcz.L.gcz_zstd_frames_bound(n))
    h_out = torch.empty(bound, dtype=torch.uint8).pin_memory()
    nb = gcz.num_windows(n)
    sizes = np.zeros(nb, np.uint64)
    used = ctypes.c_size_t()
    threads = os.cpu_count() or 1

    def gpu_step():
        rc = gcz.L.gcz_zstd_compress_frames_gpu(ctx.handle, h_in.data_ptr(), n, 2, h_out.data_ptr(), bound,
                                                sizes.ctypes.data, ctypes.byref(used))
        if rc != 0:
            raise RuntimeError(gcz.L.gcz_last_error(ctx.handle).decode())

    def cpu_coder_step():
        rc = gcz.L.gcz_zstd_compress_frames(ctx.handle, h_in.data_ptr(), n, 2, 0, h_out.data_ptr(), bound,
                                            sizes.ctypes.data, ctypes.byref(used))
        if rc != 0:
            raise RuntimeError(gcz.L.gcz_last_error(ctx.handle).decode())

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            fn()
            times.append(time.perf_counter() - t0)
        return n * len(times) / sum(times) / 1e9, sum(times) / len(times)

    ctx.profile_start()
    value, sec = timed(gpu_step, args.steps, max(args.warmup, 3))
    _, _, launches = ctx.profile_stop()
    gpu_bytes = int(used.value)
    pool = sched = None
    if not args.no_cpu_baseline:  # the host-coder legs (skipped when profiling the GPU path)
        cpu_value, _ = timed(cpu_coder_step, 1, 1)
        cpu_bytes = int(used.value)
        pool = {"gbs": round(cpu_value, 3), "threads": threads, "compressed_bytes": cpu_bytes,
                "ratio": round(cpu_bytes / n, 4)}
        sample = data[:64 << 20]
        t0 = time.perf_counter()
        seqs, off = ctx.zstd_match_find(sample, DEPTH)
        t1 = time.perf_counter()
        comp = codecs.SequenceCompressor()
        for b in range(off.size - 1):
            comp.compress(sample[b * 65536:(b + 1) * 65536], seqs[int(off[b]):int(off[b + 1])])
        t2 = time.perf_counter()
        comp.close()
        sched = {"bytes": int(sample.size), "gpu_s": round(t1 - t0, 4), "serial_coder_s": round(t2 - t1, 3),
                 "gbs": round(sample.size / (t2 - t0) / 1e9, 4)}
    print(json.dumps({
        "metric": "Zstd L2 frames, input GB/s per B200 (end to end)", "value": round(value, 3),
        "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": round(1e3 * sec, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": {"workload": "zstd_l2_frames_1gib", "input_bytes": n, "windows": nb, "slice": "32 MiB, 4 slots",
                   "entropy_stage": "GPU: Huffman/RLE/raw literals, per-window RLE/FSE-compressed/predefined sequence tables, repeat codes",
                   "compressed_bytes": gpu_bytes, "ratio": round(gpu_bytes / n, 4)},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": n, "d2h_bytes_per_step": gpu_bytes},
        "libzstd_coder_pool": pool,
        "reference_schedule_sample": sched,
        "gpu_launches": int(launches)}), flush=True)


def run_tune(args):
    """Runs the autotuner (gcz/autotune.py) on samples of the Zstd (seed 2)
    and LZMA2 (seed 3) workloads and saves the winners for this GPU model."""
    import torch
    import gcz
    from gcz import autotune

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ctx = gcz.Context(local)
    n = min(args.bytes, 256 << 20)
    out = autotune.tune(ctx, gcz.gen_synthetic(SEED, n, 8 << 20), gcz.gen_synthetic(3, n, 128 << 20),
                        search_depth=DEPTH, reps=5)
    print(json.dumps({"workload": "tune", "sample_bytes": n, "best": out["best"], "saved": autotune.tuned_path(local),
                      "zstd": out["zstd"]["results"], "lzma2": out["lzma2"]["results"],
                      "host": out.get("host", {}).get("results")}), flush=True)


def main():
    args = parse()
    single = args.workload in ("serving", "uneven", "frames", "tune")
    if args.impl != "reference" and single and int(os.environ.get("RANK", "0")) != 0:
        return  # one-GPU workloads: rank 0 runs and prints, the other ranks have no work
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "lzma2":
        run_lzma2(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.workload == "uneven":
        run_uneven(args)
    elif args.workload == "frames":
        run_frames(args)
    elif args.workload == "tune":
        run_tune(args)
    else:
        run_gcz(args)


if __name__ == "__main__":
    main()
