"""Uneven inputs in one launch: every window of a batch gives exactly what the
same input gives alone (and what the oracle gives), for Zstd and LZMA2; the
batch call replays inside a CUDA graph; the autotuner keeps results fixed."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _files(seed, count, max_size):
    import gcz

    sizes, mix = gcz.gen_file_sizes(seed, count, 1, max_size)
    return [gcz.gen_synthetic(seed * 1000 + i, int(s), 8 << 20, tuple(mix[i])) for i, s in enumerate(sizes)]


def test_zstd_files_equal_alone_and_oracle(ctx):
    files = _files(5, 120, 700000)
    files += [np.zeros(0, np.uint8), np.zeros(5, np.uint8), np.full(65536 * 2 + 3, 7, np.uint8)]
    seqs, offs = ctx.zstd_match_find_files(files, 16)
    w = 0
    for f in files:
        alone_s, alone_o = ctx.zstd_match_find(f, 16)
        o_s, o_o = orc.zstd_sequences(f, 16)
        nbf = alone_o.size - 1
        base = int(offs[w])
        np.testing.assert_array_equal(offs[w:w + nbf + 1] - base, alone_o)
        np.testing.assert_array_equal(seqs[base:int(offs[w + nbf])], alone_s)
        np.testing.assert_array_equal(alone_s, o_s)
        w += nbf
    assert w == offs.size - 1


def test_lzma2_batch_device_equals_alone(ctx):
    import torch
    import gcz

    files = _files(6, 60, 500000)
    foff, wins, slab = gcz.batch_layout([f.size for f in files])
    h_slab = np.zeros(slab, np.uint8)
    for o, f in zip(foff, files):
        h_slab[int(o):int(o) + f.size] = f
    d_slab = torch.from_numpy(h_slab).cuda()
    d_wins = torch.from_numpy(wins.view(np.uint8)).cuda()
    d_packed = torch.zeros(slab, dtype=torch.int32, device="cuda")
    d_has = torch.zeros(max(wins.size, 1), dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    ctx.lzma2_match_find_batch_device(d_slab.data_ptr(), slab, d_wins.data_ptr(), wins.size, 32, d_packed.data_ptr(),
                                      d_has.data_ptr(), st)
    ctx.sync(st)
    packed = d_packed.cpu().numpy().view(np.uint32)
    has = d_has.cpu().numpy()
    w = 0
    for o, f in zip(foff, files):
        alone_p, alone_h = ctx.lzma2_match_find(f, 32)
        np.testing.assert_array_equal(packed[int(o):int(o) + f.size], alone_p)
        np.testing.assert_array_equal(packed[int(o):int(o) + f.size], orc.lzma_packed(f, 32))
        np.testing.assert_array_equal(has[w:w + alone_h.size], alone_h)
        w += alone_h.size


def test_zstd_batch_replays_in_cuda_graph(ctx):
    import torch
    import gcz

    files = _files(7, 40, 400000)
    foff, wins, slab = gcz.batch_layout([f.size for f in files])
    h_slab = np.zeros(slab, np.uint8)
    for o, f in zip(foff, files):
        h_slab[int(o):int(o) + f.size] = f
    d_slab = torch.from_numpy(h_slab).cuda()
    d_wins = torch.from_numpy(wins.view(np.uint8)).cuda()
    cap = sum(int(gcz.L.gcz_zstd_max_sequences(f.size)) for f in files)
    d_seqs = torch.zeros((cap, 4), dtype=torch.int32, device="cuda")
    d_off = torch.zeros(wins.size + 1, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        ctx.zstd_match_find_batch_device(d_slab.data_ptr(), slab, d_wins.data_ptr(), wins.size, 16, d_seqs.data_ptr(),
                                         cap, d_off.data_ptr(), s.cuda_stream)  # allocates scratch once
    torch.cuda.synchronize()
    want_off = d_off.clone()
    want = d_seqs[:int(want_off[-1])].clone()
    d_seqs.zero_()
    d_off.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        ctx.zstd_match_find_batch_device(d_slab.data_ptr(), slab, d_wins.data_ptr(), wins.size, 16, d_seqs.data_ptr(),
                                         cap, d_off.data_ptr(), s.cuda_stream)
    for _ in range(2):
        d_seqs.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(d_off, want_off)
        assert torch.equal(d_seqs[:int(want_off[-1])], want)
    del g


def _defaults(ctx):
    for k, v in (("algo", 2), ("parse_ctas", 3), ("staged", 1), ("parse_seg", 1024), ("sweep_warps", 7), ("sweep_groups", 0),
                 ("sweep_prefetch", 4), ("lzma_ctas", 3), ("lzma_threads", 1024),
                 ("slice_windows", 512)):
        ctx.set_option(k, v)


def test_autotuner_covers_every_knob_and_keeps_results(ctx, tmp_path, monkeypatch):
    """Every Zstd schedule (kernel family, sweep warps, segment width, CTAs per
    SM) gives the same sequences and every LZMA2 schedule the same matches --
    the tuner checks that as it times them -- and the winners are saved per GPU
    model and loaded back into a fresh context.  Each timed schedule is also
    checked against the oracle on a few windows."""
    import gcz
    from gcz import autotune
    from oracle import oracle as orc

    monkeypatch.setattr(autotune, "TUNED_DIR", str(tmp_path))
    z = gcz.gen_synthetic(8, 8 << 20, 8 << 20)
    lz = gcz.gen_synthetic(9, 8 << 20, 128 << 20)
    try:
        out = autotune.tune(ctx, z, lz, reps=1, slices=True)
        assert len(out["zstd"]["results"]) == len(autotune.ZSTD_CANDIDATES)
        assert len(out["lzma2"]["results"]) == len(autotune.LZMA_CANDIDATES)
        assert set(out["best"]) >= {"algo", "lzma_ctas", "slice_windows"}
        for cfg in autotune.ZSTD_CANDIDATES[::5]:
            _defaults(ctx)
            for k, v in cfg.items():
                ctx.set_option(k, v)
            s, o = ctx.zstd_match_find(z[:4 * 65536], 16)
            os_, oo = orc.zstd_sequences(z[:4 * 65536], 16)
            np.testing.assert_array_equal(o, oo)
            np.testing.assert_array_equal(s, os_)
        c2 = gcz.Context(0)
        assert autotune.apply_tuned(c2) == out["best"]
        assert all(c2.query(k) == v for k, v in out["best"].items())
        c2.close()
    finally:
        _defaults(ctx)


def test_sharded_single_rank_uses_gpu_context(ctx):
    """Without a process group gcz.shards runs the whole input on this GPU."""
    import gcz
    from gcz import shards

    data = gcz.gen_synthetic(71, 3 * 65536 + 5, 8 << 20)
    s, o = shards.zstd_match_find_sharded(data, 16)
    s0, o0 = ctx.zstd_match_find(data, 16)
    np.testing.assert_array_equal(o, o0)
    np.testing.assert_array_equal(s, s0)
    p, h = shards.lzma2_match_find_sharded(data, 32)
    p0, h0 = ctx.lzma2_match_find(data, 32)
    np.testing.assert_array_equal(p, p0)
    np.testing.assert_array_equal(h, h0)


def test_host_pipeline_uneven_slices(ctx):
    """1500 windows + a ragged tail: the host-buffer pipeline cuts ramped slices
    of unequal size; results equal one device call and the oracle."""
    import torch
    import gcz

    n = 1500 * 65536 + 777
    data = gcz.gen_synthetic(91, n, 8 << 20)
    seqs, off = ctx.zstd_match_find(data, 16)
    d_in = torch.from_numpy(data).cuda()
    cap = int(gcz.L.gcz_zstd_max_sequences(n))
    d_seqs = torch.empty((cap, 4), dtype=torch.int32, device="cuda")
    d_off = torch.empty(gcz.num_windows(n) + 1, dtype=torch.int64, device="cuda")
    ctx.zstd_match_find_device(d_in.data_ptr(), n, 16, d_seqs.data_ptr(), cap, d_off.data_ptr(), 0)
    ctx.sync(0)
    o_dev = d_off.cpu().numpy().astype(np.uint64)
    np.testing.assert_array_equal(off, o_dev)
    np.testing.assert_array_equal(seqs, d_seqs[:int(o_dev[-1])].cpu().numpy().view(np.uint32))
    sub = data[:300 * 65536]
    o_s, o_o = orc.zstd_sequences(sub, 16, threads=16)
    np.testing.assert_array_equal(off[:301], o_o)
    np.testing.assert_array_equal(seqs[:int(o_o[-1])], o_s)
    packed, has = ctx.lzma2_match_find(data, 32)
    np.testing.assert_array_equal(packed[:sub.size], orc.lzma_packed(sub, 32, threads=16))
    np.testing.assert_array_equal(has, ctx.lzma2_triage(data, 32))
