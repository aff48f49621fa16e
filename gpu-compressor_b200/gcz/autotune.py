"""Autotuner for the schedule-only knobs of libgcz.

Hash bits, window size and the parse rules are fixed by the reference (they
decide the sequences and matches); what may change is how the work is
scheduled:

  Zstd   "sweep_warps"  windows swept per CTA (4-7), one 32 KiB table each
         "sweep_groups" the sweep's grouping of lanes that share a hash bucket:
                        after a read-back (0: __match_any_sync, 1: ballots) or
                        one block ahead for every step (2, 3 likewise)
         "sweep_prefetch" how far ahead (0, 4 or 8 blocks of 128 bytes) the
                        read-back sweeps prefetch their input into L2
         "parse_seg"    speculative segment of the second stage: 2048, 4096 or
                        8192 bytes per warp (32, 16 or 8 warps per window), or
                        1024 bytes per 8-lane group (64 segments per window),
                        or 512 bytes per 4-lane group (128 segments)
         "parse_ctas"   second-stage CTAs per SM
  LZMA2  "lzma_ctas"    second-stage CTAs per SM (the sweep is shared)
         "lzma_threads" second-stage threads per CTA (256, 512 or 1024)
  host   "slice_windows" windows per slice of the host-buffer pipelines

tune_zstd() and tune_lzma2() time every candidate on a sample of the caller's
input with CUDA events, check that all of them give bit-identical results
(sequences and offsets; packed matches and has-match bytes), keep the fastest
and leave it set on the context.  tune() runs both (and the host slice size)
and saves the winners under tuned/<GPU model>.json; apply_tuned() loads that
file into a context.
"""
import hashlib
import json
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TUNED_DIR = os.path.join(HERE, "tuned")

# The fused single-warp kernels (algo 1) are a fallback family, several times
# slower on every input measured, and "algo" also switches LZMA2's kernels, so
# the search stays within the split kernels.
ZSTD_CANDIDATES = [
    {"algo": 2, "sweep_warps": sw, "sweep_groups": sg, "sweep_prefetch": pf, "parse_seg": seg, "parse_ctas": ctas}
    for sw in (7, 6, 5, 4)
    for sg, pf in ((0, 4), (0, 8), (0, 0), (1, 4), (1, 0), (2, 0), (3, 0))
    for seg, ctas_list in ((4096, (3, 2)), (1024, (3, 2)), (512, (3, 2)), (8192, (3, 2)), (2048, (1,)))
    for ctas in ctas_list
]
LZMA_CANDIDATES = [{"lzma_ctas": c, "lzma_threads": t} for t in (512, 256) for c in (3, 2, 1)] + [
    {"lzma_ctas": c, "lzma_threads": 1024} for c in (2, 1)]
SLICE_CANDIDATES = [256, 512, 1024, 2048]


def model_key(name):
    return re.sub(r"[^A-Za-z0-9]+", "_", name).strip("_")


def tuned_path(device=0):
    import torch

    return os.path.join(TUNED_DIR, model_key(torch.cuda.get_device_name(device)) + ".json")


def _apply(ctx, cfg):
    for k, v in cfg.items():
        ctx.set_option(k, v)


def _timed(torch, st, fn, reps):
    fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _u8(sample):
    return np.ascontiguousarray(np.frombuffer(memoryview(sample).cast("B"), dtype=np.uint8))


def tune_zstd(ctx, sample, search_depth=16, reps=3, candidates=None):
    """Fastest Zstd schedule on `sample` (host bytes, a representative slice
    of the workload, >= a few MiB); every candidate must give the same
    sequences and offsets."""
    import torch
    from . import L, num_windows

    data = _u8(sample)
    n = data.size
    dev = torch.device("cuda", ctx.device)
    d_in = torch.from_numpy(data).to(dev)
    cap = int(L.gcz_zstd_max_sequences(n))
    d_seqs = torch.empty((max(cap, 1), 4), dtype=torch.int32, device=dev)
    d_off = torch.empty(num_windows(n) + 1, dtype=torch.int64, device=dev)
    st = torch.cuda.current_stream(dev)
    results, digest = [], None

    def run():
        ctx.zstd_match_find_device(d_in.data_ptr(), n, search_depth, d_seqs.data_ptr(), cap, d_off.data_ptr(),
                                   st.cuda_stream)

    for cfg in candidates or ZSTD_CANDIDATES:
        _apply(ctx, cfg)
        run()
        ctx.sync(st.cuda_stream)
        total = int(d_off[-1].item())
        h = hashlib.sha256(d_seqs[:total].cpu().numpy().tobytes() + d_off.cpu().numpy().tobytes()).hexdigest()
        if digest is None:
            digest = h
        elif h != digest:
            raise AssertionError(f"schedule {cfg} changed the sequences")
        ms = _timed(torch, st, run, reps)
        ctx.sync(st.cuda_stream)
        results.append({"config": cfg, "ms": round(ms, 4), "gbps": round(n / (ms / 1e3) / 1e9, 3)})
    best = min(results, key=lambda r: r["ms"])
    _apply(ctx, best["config"])
    return {"best": best["config"], "best_gbps": best["gbps"], "results": results, "sample_bytes": n,
            "sequences_sha256": digest}


def tune_lzma2(ctx, sample, reps=3, candidates=None):
    """Fastest LZMA2 second-stage schedule on `sample`; every candidate must
    give the same per-position matches and has-match bytes."""
    import torch
    from . import num_windows

    data = _u8(sample)
    n = data.size
    dev = torch.device("cuda", ctx.device)
    d_in = torch.from_numpy(data).to(dev)
    d_packed = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    d_has = torch.empty(max(num_windows(n), 1), dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream(dev)
    results, digest = [], None

    def run():
        ctx.lzma2_match_find_device(d_in.data_ptr(), n, 32, d_packed.data_ptr(), d_has.data_ptr(), st.cuda_stream)

    for cfg in candidates or LZMA_CANDIDATES:
        _apply(ctx, cfg)
        run()
        ctx.sync(st.cuda_stream)
        h = hashlib.sha256(d_packed[:n].cpu().numpy().tobytes() + d_has.cpu().numpy().tobytes()).hexdigest()
        if digest is None:
            digest = h
        elif h != digest:
            raise AssertionError(f"schedule {cfg} changed the matches")
        ms = _timed(torch, st, run, reps)
        ctx.sync(st.cuda_stream)
        results.append({"config": cfg, "ms": round(ms, 4), "gbps": round(n / (ms / 1e3) / 1e9, 3)})
    best = min(results, key=lambda r: r["ms"])
    _apply(ctx, best["config"])
    return {"best": best["config"], "best_gbps": best["gbps"], "results": results, "sample_bytes": n,
            "matches_sha256": digest}


def tune_slices(ctx, sample, search_depth=16, reps=2, candidates=None):
    """Fastest host-pipeline slice size for gcz_zstd_match_find on a pinned
    copy of `sample` (H2D, kernels and D2H overlap slice by slice)."""
    import time
    import torch
    from . import L, num_windows

    data = _u8(sample)
    n = data.size
    h_in = torch.from_numpy(data).pin_memory()
    cap = n // 8 + 1024
    h_seqs = torch.empty((cap, 4), dtype=torch.int32).pin_memory()
    h_off = torch.empty(num_windows(n) + 1, dtype=torch.int64).pin_memory()
    results, digest = [], None
    for sw in candidates or SLICE_CANDIDATES:
        ctx.set_option("slice_windows", sw)

        def run():
            rc = L.gcz_zstd_match_find(ctx.handle, h_in.data_ptr(), n, search_depth, h_seqs.data_ptr(), cap,
                                       h_off.data_ptr())
            if rc != 0:
                raise RuntimeError(L.gcz_last_error(ctx.handle).decode())

        run()
        h = hashlib.sha256(h_off.numpy().tobytes() + h_seqs[:int(h_off[-1])].numpy().tobytes()).hexdigest()
        if digest is None:
            digest = h
        elif h != digest:
            raise AssertionError(f"slice size {sw} changed the sequences")
        t0 = time.perf_counter()
        for _ in range(reps):
            run()
        dt = (time.perf_counter() - t0) / reps
        results.append({"config": {"slice_windows": sw}, "ms": round(dt * 1e3, 3), "gbps": round(n / dt / 1e9, 3)})
    best = min(results, key=lambda r: r["ms"])
    ctx.set_option("slice_windows", best["config"]["slice_windows"])
    return {"best": best["config"], "best_gbps": best["gbps"], "results": results, "sample_bytes": n}


def tune(ctx, zstd_sample, lzma_sample=None, search_depth=16, reps=3, save=True, slices=True):
    """All knobs: the Zstd schedule (which fixes the shared sweep), then the
    LZMA2 second stage, then the host slice size.  Saves the winners as
    tuned/<GPU model>.json (with every candidate's time) unless save=False."""
    import torch

    out = {"gpu": torch.cuda.get_device_name(ctx.device), "zstd": tune_zstd(ctx, zstd_sample, search_depth, reps)}
    out["lzma2"] = tune_lzma2(ctx, lzma_sample if lzma_sample is not None else zstd_sample, reps)
    if slices:
        out["host"] = tune_slices(ctx, zstd_sample, search_depth)
    best = dict(out["zstd"]["best"])  # includes algo 2
    best.update(out["lzma2"]["best"])
    if slices:
        best.update(out["host"]["best"])
    out["best"] = best
    if save:
        os.makedirs(TUNED_DIR, exist_ok=True)
        with open(tuned_path(ctx.device), "w") as f:
            json.dump(out, f, indent=1)
    return out


def apply_tuned(ctx, path=None):
    """Set the knobs saved for this GPU model on `ctx`; returns them, or None
    when no tuned file exists (the context keeps its defaults)."""
    p = path or tuned_path(ctx.device)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        best = json.load(f)["best"]
    _apply(ctx, best)
    return best
