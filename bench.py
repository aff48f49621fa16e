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

METRIC = "input GB/s per B200 (match-find, end-to-end)"
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
    ap.add_argument("--algo", type=int, default=2, help="1: fused single-warp kernels, 2: sweep + second stage")
    ap.add_argument("--workload", default="zstd", choices=["zstd", "lzma2", "serving", "uneven", "frames"],
                    help="zstd: Zstd L2 batched 1 GiB (the reported line); lzma2: LZMA2 L1 1 GiB, seed 3; "
                         "serving: open-loop request stream; uneven: many files in one launch")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving: requests per second (Poisson)")
    ap.add_argument("--duration", type=float, default=10.0, help="serving: seconds of arrivals")
    ap.add_argument("--max-request", type=int, default=64 << 20, help="serving: largest request size")
    ap.add_argument("--max-batch", type=int, default=256 << 20, help="serving: largest batch (bytes of input)")
    ap.add_argument("--files", type=int, default=4096, help="uneven: number of files")
    ap.add_argument("--max-file", type=int, default=8 << 20, help="uneven: largest file size")
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


def run_gcz(args):
    import torch
    import gcz

    world, rank, local, dist = dist_setup(args)
    dev = torch.device("cuda", local)
    ctx = gcz.Context(local)
    ctx.set_option("algo", args.algo)
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
    e2e_value = link_value = None
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
            e2e_step()
        e2e_s = time.perf_counter() - t0
        barrier(dist, torch, local)
        e2e_max = max_over_ranks(dist, torch, e2e_s)
        e2e_value = round(world * n * args.e2e_steps / e2e_max / 1e9, 3)
        assert int(h_off[-1].item()) == nseq
        link_s = max_over_ranks(dist, torch, link_time(torch, dev, h_in, d_in, h_seqs, d_seqs, 16 * nseq))
        link_value = round(world * n / link_s / 1e9, 3)

    # ---- roofline of the match-find step (match kernel + offset scan + compaction)
    peak, peak_kind = peaks()
    step_ms = kern_ms / max(kern_launches, 1)
    alg_bytes = n + 16 * nseq + 8 * B  # input once + ZSTD_Sequence out + counts/offsets
    achieved = alg_bytes / (step_ms / 1e3) / 1e9
    traffic = measured_traffic(WORKLOAD, n)

    cpu = libs = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = data[:256 << 20]
        dt, _ = cpu_oracle_time(sample, DEPTH, threads)
        cpu = {"value": round(sample.size / dt / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"first 256 MiB of the same 1 GiB input (4096 windows), oracle/oracle.c on {threads} threads"}
        libs = cpu_library_baselines(data[:256 << 20], "zstd", threads)
        small = data[:16 << 20]
        dt1, _ = cpu_oracle_time(small, DEPTH, 1)
        libs["oracle single thread"] = {"gbs": round(small.size / dt1 / 1e9, 4), "threads": 1,
                                        "sample_bytes": int(small.size)}

    total_launches = sum_over_ranks(dist, torch, all_launches)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD, "input_bytes_per_gpu": n, "windows_per_gpu": B, "window": 65536,
                       "search_depth": DEPTH, "sequences_per_gpu": nseq, "parallelism": f"replicas{world}",
                       "algo": args.algo, "fallback_windows": ctx.query("fallback_windows"),
                       "l2": "input 1 GiB > 126 MB L2, no flush needed"},
            "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": n,
                    "d2h_bytes_per_step": 16 * nseq + 8 * (B + 1),
                    "link_bound": {"value": link_value, "unit": "GB/s",
                                   "what": "plain pinned copies of the step's bytes, no kernels: the H2D of the "
                                           "input in 64 MiB pieces with the sequence records' D2H on a second "
                                           "stream"},
                    "frac_of_link": round(e2e_value / link_value, 3) if e2e_value and link_value else None},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs", "kernel_ms_per_step": round(step_ms, 4),
                         "algorithmic_bytes_per_step": alg_bytes},
            "cpu_baseline": cpu,
            "cpu_libraries": libs,
            "gpu_launches": int(total_launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_lzma2(args):
    """LZMA2 L1 workload: 1 GiB (seed 3, copy offsets to 128 MiB), 16384
    windows, per-position packed matches + per-window has-match byte."""
    import torch
    import gcz

    world, rank, local, dist = dist_setup(args)
    dev = torch.device("cuda", local)
    ctx = gcz.Context(local)
    ctx.set_option("algo", args.algo)
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
    ms_max = max_over_ranks(dist, torch, e0.elapsed_time(e1))
    value = world * n * args.steps / (ms_max / 1e3) / 1e9
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
    libs = l1 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
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
    if rank == 0:
        print(json.dumps({
            "metric": "input GB/s per B200 (LZMA2 L1 match-find)", "value": round(value, 3), "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator)",
            "config": {"workload": "lzma2_l1_1gib", "input_bytes_per_gpu": n, "windows_per_gpu": B, "algo": args.algo},
            "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": n, "d2h_bytes_per_step": B,
                    "call": "gcz_lzma2_match_find(packed=NULL): per-window has-match bytes"},
            "e2e_packed": {"value": e2e_packed, "unit": "GB/s", "h2d_bytes_per_step": n,
                           "d2h_bytes_per_step": 4 * n + B, "call": "gcz_lzma2_match_find: per-position matches"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": measured_traffic("lzma2_l1_1gib", n),
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "kernel_ms_per_step": round(step_ms, 4), "algorithmic_bytes_per_step": alg_bytes},
            "cpu_libraries": libs, "lzma2_l1_nvlz_end_to_end": l1,
            "gpu_launches": int(all_launches), "clocks": clk.summary()}), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_serving(args):
    """Open-loop Poisson stream against the library's request loop: request
    sizes log-uniform 4 KiB..max_request, 70% Zstd L1 / 20% Zstd L2 / 10% LZMA2
    L1, payloads are slices of a pinned 1 GiB synthetic pool.  Reports the
    completed input GB/s and submit-to-completion p50/p99 latency."""
    import threading
    import torch
    import gcz
    from gcz import serving

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ctx = gcz.Context(local)
    pool_n = 1 << 30
    pool = torch.empty(pool_n, dtype=torch.uint8, pin_memory=True)
    gcz.gen_synthetic(5, pool_n, 8 << 20, out=pool.numpy())
    srv = serving.Server(ctx, hbm_budget=120 * 10**9, max_batch_bytes=args.max_batch)
    rng = np.random.default_rng(11)
    count = int(args.rate * args.duration)
    gaps = rng.exponential(1.0 / args.rate, size=count)
    sizes = np.exp(rng.uniform(np.log(4096), np.log(args.max_request), size=count)).astype(np.int64)
    u = rng.random(count)
    kinds = np.where(u < 0.9, serving.ZSTD, serving.LZMA2)
    depths = np.where(u < 0.7, 16, np.where(u < 0.9, 64, 32))
    offs = (rng.random(count) * (pool_n - sizes)).astype(np.int64)
    pool_np = pool.numpy()
    q = []
    lock = threading.Condition()
    # Outputs go to one pinned ring, allocated in submission order and freed in
    # completion order (the waiter completes requests in order); a full ring
    # holds the submitter back.  Zstd results get room for n/16 + 1024
    # sequences (this input averages one sequence per ~50 bytes).
    ring_n = 4 << 30
    ring = torch.empty(ring_n, dtype=torch.uint8, pin_memory=True).numpy()
    rs = {"head": 0, "tail": 0}
    ring_cv = threading.Condition()

    def ring_alloc(nbytes):
        nbytes = (nbytes + 255) & ~255
        with ring_cv:
            h = rs["head"]
            if h % ring_n + nbytes > ring_n:
                h += ring_n - h % ring_n  # skip the ring's end
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

    # Warm-up outside the timed region: two largest batches of each kind, so both
    # slots of the loop hold their device buffers at full size.  The loop flips
    # slots on every batch, so the two of a kind go back to back (Z, Z, L, L);
    # alternating kinds would leave each slot warm for one kind only, and the
    # other kind's first batches there would allocate inside the timed region.
    wn = min(args.max_batch, pool_n)
    for kind in (serving.ZSTD, serving.ZSTD, serving.LZMA2, serving.LZMA2):
        if kind == serving.ZSTD:
            cap = wn // 16 + 1024
            r = srv.submit(kind, pool_np[:wn], 16, out_a=ring[:cap * 16].view(np.uint32).reshape(cap, 4), cap=cap,
                           out_b=ring[cap * 16:cap * 16 + (gcz.num_windows(wn) + 1) * 8].view(np.uint64))
        else:
            r = srv.submit(kind, pool_np[:wn], 32, out_b=ring[:gcz.num_windows(wn)], packed=False)
        srv.wait(r)
    base = srv.stats()

    wt = threading.Thread(target=waiter)
    wt.start()
    t0 = time.perf_counter()
    nxt = t0
    for i in range(count):
        nxt += gaps[i]
        d = nxt - time.perf_counter()
        if d > 0:
            time.sleep(d)
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
    wt.join()
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    done_bytes = st["bytes"] - base["bytes"]
    st["batches"] -= base["batches"]
    st["completed"] -= base["completed"]
    st["p50_ms"], st["p99_ms"] = float(np.percentile(lats, 50)), float(np.percentile(lats, 99))
    print(json.dumps({
        "metric": "serving input GB/s per B200 (match-find, p50/p99 latency)", "value": round(done_bytes / wall / 1e9, 3),
        "unit": "GB/s", "n_gpus": 1, "higher_is_better": True, "dtype": "u8", "data": "synthetic (seeded pool)",
        "config": {"workload": "serving_poisson", "rate_per_s": args.rate, "duration_s": args.duration,
                   "requests": count, "size_range": [4096, args.max_request], "mix": "70% zstd L1, 20% zstd L2, 10% lzma2 (has-match bytes only)",
                   "outputs": "pinned 4 GiB ring, freed in completion order", "offered_gbps": round(float(sizes.sum()) / args.duration / 1e9, 3), "hbm_budget_bytes": 120 * 10**9,
                   "max_batch_bytes": args.max_batch},
        "latency_ms": {"p50": round(st["p50_ms"], 3), "p99": round(st["p99_ms"], 3)},
        "batches": st["batches"], "completed": st["completed"], "wall_s": round(wall, 3)}), flush=True)


def run_uneven(args):
    """Uneven batch: many files of log-uniform size with per-file Dirichlet(1,1,1)
    mixes in one launch through the window-table entry point (device resident).
    Reports input GB/s of the launch."""
    import torch
    import gcz

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ctx = gcz.Context(local)
    sizes, mix = gcz.gen_file_sizes(4, args.files, 4096, args.max_file)
    foff, wins, slab = gcz.batch_layout(sizes)
    h_slab = torch.zeros(slab, dtype=torch.uint8).pin_memory()
    hs = h_slab.numpy()
    from concurrent.futures import ThreadPoolExecutor

    def gen(i):
        o, sz = int(foff[i]), int(sizes[i])
        gcz.gen_synthetic(4000 + i, sz, 8 << 20, tuple(mix[i]), out=hs[o:o + sz])

    with ThreadPoolExecutor(os.cpu_count() or 4) as ex:
        list(ex.map(gen, range(len(sizes))))
    d_slab = h_slab.cuda()
    d_wins = torch.from_numpy(wins.view(np.uint8)).cuda()
    cap = sum(int(gcz.L.gcz_zstd_max_sequences(int(x))) for x in sizes)
    d_seqs = torch.empty((cap, 4), dtype=torch.int32, device="cuda")
    d_off = torch.empty(wins.size + 1, dtype=torch.int64, device="cuda")
    st = torch.cuda.current_stream()

    def step():
        ctx.zstd_match_find_batch_device(d_slab.data_ptr(), slab, d_wins.data_ptr(), wins.size, 16,
                                         d_seqs.data_ptr(), cap, d_off.data_ptr(), st.cuda_stream)

    for _ in range(3):  # also sizes every buffer, so the captured launches allocate nothing
        step()
    ctx.sync(st.cuda_stream)
    # the whole batch as one CUDA graph (the launches of one match-find step)
    cs = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(cs):
        with torch.cuda.graph(g, stream=cs):
            ctx.zstd_match_find_batch_device(d_slab.data_ptr(), slab, d_wins.data_ptr(), wins.size, 16,
                                             d_seqs.data_ptr(), cap, d_off.data_ptr(), cs.cuda_stream)
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    ctx.sync(st.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        g.replay()
    e1.record(st)
    torch.cuda.synchronize()
    ctx.sync(st.cuda_stream)
    ms = e0.elapsed_time(e1) / args.steps
    total = int(np.sum(sizes))
    print(json.dumps({
        "metric": "uneven-batch input GB/s per B200 (Zstd L1 match-find, one launch)",
        "value": round(total / (ms / 1e3) / 1e9, 3), "unit": "GB/s", "ms_per_step": round(ms, 3),
        "config": {"workload": "uneven_batch", "files": args.files, "size_range": [4096, args.max_file],
                   "input_bytes": total, "windows": int(wins.size), "mix": "Dirichlet(1,1,1) per file",
                   "launch": "one CUDA graph replay per step"}}), flush=True)


def run_reference(args):
    """Reference arm: the reference's path on this box.  `value` = its CPU
    restatement (oracle port) on all host threads over a bounded sample of the
    workload; `reference_kernels_b200` = the reference's own kernels on the GPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import gcz

    n = N_BYTES
    data = gcz.gen_synthetic(SEED, n, 8 << 20)
    threads = os.cpu_count() or 1
    sample = data[:256 << 20]
    times = []
    for _ in range(max(args.warmup, 1)):
        cpu_oracle_time(sample[:16 << 20], DEPTH, threads)
    steps = max(1, min(args.steps, 5))
    for _ in range(steps):
        dt, _ = cpu_oracle_time(sample, DEPTH, threads)
        times.append(dt)
    value = sample.size * steps / sum(times) / 1e9
    refk = reference_kernels(data)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world, "steps": steps,
        "warmup": max(args.warmup, 1), "ms_per_step": round(sum(times) / steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOAD, "input_bytes_per_gpu": n, "window": 65536, "search_depth": DEPTH},
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"first 256 MiB of the 1 GiB input, oracle/oracle.c on {threads} threads "
                                   "(the reference has no CPU match finder; its kernels are timed below)"},
        "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_kernels_b200": refk,
    }
    print(json.dumps(line), flush=True)


def reference_kernels(data):
    """The reference's zstd_match_find PTX (JIT on this GPU) over the same
    1 GiB in one grid (kernel only), and its adapter pattern per 8 MiB chunk
    (alloc_zeros + H2D + launch + D2H of the sequence buffer) on a sample."""
    try:
        from oracle import ref_kernels
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
        # adapter pattern, 8 MiB chunks (compress_zstd_custom.rs:79-116), first 128 MiB
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
        return {"kernel_only_gbs": round(n / (k_ms / 1e3) / 1e9, 4), "kernel_ms_1gib": round(k_ms, 3),
                "adapter_pattern_gbs": round(sample.size / a_s / 1e9, 4),
                "note": "PTX from the reference's own sources and flags, driver JIT; grid=windows, block=256"}
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
                   "entropy_stage": "GPU: Huffman/RLE/raw literals, predefined-FSE sequences, repeat codes",
                   "compressed_bytes": gpu_bytes, "ratio": round(gpu_bytes / n, 4)},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": n, "d2h_bytes_per_step": gpu_bytes},
        "libzstd_coder_pool": pool,
        "reference_schedule_sample": sched,
        "gpu_launches": int(launches)}), flush=True)


def main():
    args = parse()
    single = args.workload in ("serving", "uneven", "frames")
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
    else:
        run_gcz(args)


if __name__ == "__main__":
    main()
