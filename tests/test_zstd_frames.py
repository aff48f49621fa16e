"""GPU Zstd entropy stage.  CPU part: the test-side restatement of the frame
encoder (zstd_frames_ref) produces frames stock libzstd decodes, on the
oracle's sequences.  GPU part: the GPU frames equal the restatement's byte for
byte and decode with stock libzstd, through the host and the device calls."""
import ctypes

import numpy as np
import pytest

import cases
import zstd_frames_ref as zr
from oracle import oracle as orc

W = 65536

INPUTS = [
    {"kind": "synthetic", "n": 3 * W + 999, "seed": 41},
    {"kind": "text", "n": 70000, "seed": 42},
    {"kind": "zeros", "n": 100000},
    {"kind": "random", "n": 70000, "seed": 3},
    {"kind": "zipf", "n": 2 * W + 300, "seed": 4},   # all 256 byte values: FSE-coded Huffman weights
    {"kind": "fib", "n": W + 5000, "seed": 5},       # Fibonacci counts: code lengths limited to 11
    {"kind": "zipf", "n": 900, "seed": 6},           # one Huffman stream
]


def _build(spec):
    rng = np.random.default_rng(spec.get("seed", 0))
    n = spec["n"]
    if spec["kind"] == "zeros":
        return np.zeros(n, np.uint8)
    if spec["kind"] == "random":
        return np.frombuffer(rng.bytes(n), np.uint8).copy()
    if spec["kind"] == "zipf":
        p = 1.0 / np.arange(1, 257) ** 1.1
        return rng.permutation(256)[rng.choice(256, n, p=p / p.sum())].astype(np.uint8)
    if spec["kind"] == "fib":
        f = [1, 1]
        while len(f) < 24:
            f.append(f[-1] + f[-2])
        p = np.array(f, float)
        return (rng.choice(24, n, p=p / p.sum()) + 150).astype(np.uint8)
    return cases.build(spec)


def _ref_frames(data, depth=16):
    seqs, off = orc.zstd_sequences(data, depth)
    out = []
    for b in range(off.size - 1):
        s = seqs[int(off[b]):int(off[b + 1])]
        out.append(zr.encode_frame(data[b * W:(b + 1) * W].tobytes(), [(x[0], x[1], x[2]) for x in s]))
    return out


@pytest.mark.parametrize("spec", INPUTS + [{"kind": "synthetic", "n": n, "seed": 7} for n in (1, 5, 255, 256, 257)],
                         ids=lambda s: f"{s['kind']}-{s['n']}")
def test_reference_frames_decode_with_libzstd(spec):
    from gcz import codecs

    data = _build(spec)
    for b, f in enumerate(_ref_frames(data)):
        win = data[b * W:(b + 1) * W]
        assert codecs.zstd_decompress(f, win.size) == win.tobytes()


def test_reference_frames_use_every_table_mode():
    """Across these inputs the sequence fields get all three table modes:
    RLE (one sequence), FSE-compressed (most windows) and predefined (few
    sequences with many distinct codes, where a description costs more than
    it saves)."""
    from gcz import codecs

    for k in zr.MODE_USES:
        zr.MODE_USES[k] = 0
    for spec in INPUTS + [{"kind": "synthetic", "n": 2000, "seed": 9}, {"kind": "text", "n": 3000, "seed": 10}]:
        data = _build(spec)
        for b, f in enumerate(_ref_frames(data)):
            win = data[b * W:(b + 1) * W]
            assert codecs.zstd_decompress(f, win.size) == win.tobytes()
    assert all(v > 0 for v in zr.MODE_USES.values()), zr.MODE_USES


def test_reference_frames_ratio_within_a_tenth_of_a_point_of_libzstd():
    """On the bench generator's data the frames' size is within 0.1 percentage
    point of libzstd's own frames for the same sequences (ZSTD_compressSequences
    per window, the reference's coder loop)."""
    import gcz
    from gcz import codecs

    data = gcz.gen_synthetic(2, 2 << 20, 8 << 20)
    seqs, off = orc.zstd_sequences(data, 64)
    comp = codecs.SequenceCompressor()
    ours = ref = 0
    for b in range(off.size - 1):
        win = data[b * W:(b + 1) * W]
        s = seqs[int(off[b]):int(off[b + 1])]
        ref += len(comp.compress(win, s))
        f = zr.encode_frame(win.tobytes(), [(x[0], x[1], x[2]) for x in s])
        assert codecs.zstd_decompress(f, win.size) == win.tobytes()
        ours += len(f)
    comp.close()
    assert 100.0 * (ours - ref) / data.size <= 0.1, (ours / data.size, ref / data.size)


def _split(blob, sizes):
    out, pos = [], 0
    for s in sizes.tolist():
        out.append(blob[pos:pos + s].tobytes())
        pos += s
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("spec", INPUTS + [{"kind": "synthetic", "n": n, "seed": 7} for n in (1, 5, 255, 256, 257)],
                         ids=lambda s: f"{s['kind']}-{s['n']}")
def test_gpu_frames_equal_reference_frames(ctx, spec):
    data = _build(spec)
    blob, sizes = ctx.zstd_compress_frames_gpu(data, 1)
    assert _split(blob, sizes) == _ref_frames(data)


@pytest.mark.gpu
def test_gpu_frames_large_decode_and_level2(ctx):
    """70 MiB + ragged tail: more than one 64 MiB pipeline slice; every frame
    decodes; level 2 gives the same bytes as level 1."""
    import gcz
    from gcz import codecs

    n = 70 * (1 << 20) + 4321
    data = gcz.gen_synthetic(17, n, 8 << 20)
    blob, sizes = ctx.zstd_compress_frames_gpu(data, 1)
    frames = _split(blob, sizes)
    assert len(frames) == gcz.num_windows(n)
    for b in range(0, len(frames), 7):
        win = data[b * W:(b + 1) * W]
        assert codecs.zstd_decompress(frames[b], win.size) == win.tobytes()
    assert 0.3 < blob.size / n < 0.9
    blob2, sizes2 = ctx.zstd_compress_frames_gpu(data, 2)
    assert np.array_equal(sizes, sizes2) and np.array_equal(blob, blob2)
    # a spot check of full equality against the restatement
    sub = data[:4 * W]
    assert frames[:4] == _ref_frames(sub)


@pytest.mark.gpu
def test_gpu_frames_pipeline_slices_do_not_change_bytes():
    """The host pipeline rotates its slices over four slots and finishes them
    in order.  Whatever the slice size -- one window per slice (every slot
    reused hundreds of times), odd sizes, or the whole input in one slice --
    the frames and the size table are the same bytes."""
    import gcz

    n = 20 * (1 << 20) + 999
    data = gcz.gen_synthetic(31, n, 8 << 20)
    c = gcz.Context(0)
    try:
        c.set_option("frames_slice_windows", 1 << 20)  # one slice
        blob, sizes = c.zstd_compress_frames_gpu(data, 1)
        assert sizes.size == gcz.num_windows(n) and int(sizes.sum()) == blob.size
        for fsw in (1, 7, 64, 512):
            c.set_option("frames_slice_windows", fsw)
            b2, s2 = c.zstd_compress_frames_gpu(data, 1)
            assert np.array_equal(s2, sizes), fsw
            assert np.array_equal(b2, blob), fsw
    finally:
        c.close()


@pytest.mark.gpu
def test_device_entropy_stage_on_oracle_sequences(ctx):
    import torch
    import gcz

    data = gcz.gen_synthetic(23, 5 * W + 77, 8 << 20)
    seqs, off = orc.zstd_sequences(data, 16)
    d_src = torch.from_numpy(data).cuda()
    d_seqs = torch.from_numpy(seqs.astype(np.int32).reshape(-1, 4)).cuda()
    d_off = torch.from_numpy(off.astype(np.int64)).cuda()
    cap = int(gcz.L.gcz_zstd_frames_bound(data.size))
    d_out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    nb = gcz.num_windows(data.size)
    d_foff = torch.empty(nb + 1, dtype=torch.int64, device="cuda")
    for _ in range(2):  # second call reuses the scratch
        ctx.zstd_encode_frames_device(d_src.data_ptr(), data.size, d_seqs.data_ptr(), d_off.data_ptr(),
                                      d_out.data_ptr(), cap, d_foff.data_ptr(), 0)
        ctx.sync(0)
        foff = d_foff.cpu().numpy().astype(np.uint64)
        blob = d_out[:int(foff[-1])].cpu().numpy()
        assert _split(blob, np.diff(foff)) == _ref_frames(data)


@pytest.mark.gpu
def test_device_entropy_stage_rejects_bad_sequences(ctx):
    """An offset reaching before the window start: the kernel's own check turns
    it into a raw frame and an error status, reported as GCZ_EINVAL."""
    import torch
    import gcz

    data = gcz.gen_synthetic(24, W, 8 << 20)
    seqs = np.array([[5000, 10, 8, 0]], np.int32)  # match at position 10 with offset 5000
    off = np.array([0, 1], np.int64)
    d_src = torch.from_numpy(data).cuda()
    d_seqs = torch.from_numpy(seqs).cuda()
    d_off = torch.from_numpy(off).cuda()
    cap = int(gcz.L.gcz_zstd_frames_bound(W))
    d_out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    d_foff = torch.empty(2, dtype=torch.int64, device="cuda")
    ctx.zstd_encode_frames_device(d_src.data_ptr(), W, d_seqs.data_ptr(), d_off.data_ptr(), d_out.data_ptr(), cap,
                                  d_foff.data_ptr(), 0)
    with pytest.raises(gcz.GczError) as e:
        ctx.sync(0)
    assert e.value.code == -1
    # the context stays usable
    blob, sizes = ctx.zstd_compress_frames_gpu(data, 1)
    assert _split(blob, sizes) == _ref_frames(data)


@pytest.mark.gpu
def test_gpu_frames_empty_and_capacity(ctx):
    import gcz

    blob, sizes = ctx.zstd_compress_frames_gpu(np.zeros(0, np.uint8))
    assert blob.size == 0 and sizes.size == 0
    data = gcz.gen_synthetic(5, 3 * W, 8 << 20)
    out = np.empty(1000, np.uint8)
    fs = np.zeros(3, np.uint64)
    used = ctypes.c_size_t()
    rc = gcz.L.gcz_zstd_compress_frames_gpu(ctx.handle, data.ctypes.data, data.size, 1, out.ctypes.data, out.size,
                                            fs.ctypes.data, ctypes.byref(used))
    assert rc == -4 and used.value == 0


@pytest.mark.gpu
def test_gpu_frames_for_file_batches(ctx):
    """Many files in one launch of each kernel (window table): every file's
    frames equal the ones the single-buffer call gives for it and decode with
    stock libzstd; the device batch call gives the same bytes."""
    import torch
    import gcz
    from gcz import codecs

    rng = np.random.default_rng(8)
    sizes = [0, 1, 300, 65535, 65536, 65537, (3 << 20) | 5, 131072, 70000]
    files = [gcz.gen_synthetic(300 + i, s, 8 << 20, tuple(rng.dirichlet([1, 1, 1]))) for i, s in enumerate(sizes)]
    files[4] = _build({"kind": "zipf", "n": 65536, "seed": 9})
    res = ctx.zstd_compress_files_gpu(files, 1)
    assert len(res) == len(files)
    for f, frames in zip(files, res):
        blob, fs = ctx.zstd_compress_frames_gpu(f, 1)
        assert frames == _split(blob, fs)
        for b in (0, len(frames) - 1):
            if frames:
                win = f[b * W:(b + 1) * W]
                assert codecs.zstd_decompress(frames[b], win.size) == win.tobytes()
    # device form
    foff, wins, slab = gcz.batch_layout([f.size for f in files])
    h_slab = np.zeros(slab, np.uint8)
    for o, f in zip(foff, files):
        h_slab[int(o):int(o) + f.size] = f
    d_slab = torch.from_numpy(h_slab).cuda()
    d_wins = torch.from_numpy(wins.view(np.uint8)).cuda()
    cap = sum(int(gcz.L.gcz_zstd_max_sequences(f.size)) for f in files)
    d_seqs = torch.empty((max(cap, 1), 4), dtype=torch.int32, device="cuda")
    d_off = torch.empty(wins.size + 1, dtype=torch.int64, device="cuda")
    ctx.zstd_match_find_batch_device(d_slab.data_ptr(), slab, d_wins.data_ptr(), wins.size, 16, d_seqs.data_ptr(), cap,
                                     d_off.data_ptr(), 0)
    fb = sum(int(gcz.L.gcz_zstd_frames_bound(f.size)) for f in files)
    d_out = torch.empty(fb, dtype=torch.uint8, device="cuda")
    d_foff = torch.empty(wins.size + 1, dtype=torch.int64, device="cuda")
    ctx.zstd_encode_frames_batch_device(d_slab.data_ptr(), slab, d_wins.data_ptr(), wins.size, d_seqs.data_ptr(),
                                        d_off.data_ptr(), d_out.data_ptr(), fb, d_foff.data_ptr(), 0)
    ctx.sync(0)
    foffs = d_foff.cpu().numpy().astype(np.uint64)
    blob = d_out[:int(foffs[-1])].cpu().numpy()
    assert _split(blob, np.diff(foffs)) == [fr for frames in res for fr in frames]
