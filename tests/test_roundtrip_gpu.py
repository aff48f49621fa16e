"""End to end on the GPU: frames built from the GPU sequences are byte-identical
to frames built from the oracle's, decode through stock libzstd / liblzma, and
the containers round-trip."""
import numpy as np
import pytest

import cases
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_zstd_frames_identical_to_oracle_and_decode(ctx):
    """Zstd L1 plain shape (16 MiB, seed 1): compress_chunk_zstd_custom."""
    import gcz
    from gcz import codecs

    data = gcz.gen_synthetic(1, 16 << 20, 8 << 20)
    frames, sizes = gcz.compress_chunk_zstd_custom(data, 0, 1)
    o_seqs, o_off = orc.zstd_sequences(data, 16, threads=16)
    comp = codecs.SequenceCompressor()
    total = 0
    for b, f in enumerate(frames):
        win = data[b * 65536:(b + 1) * 65536]
        assert f == comp.compress(win, o_seqs[int(o_off[b]):int(o_off[b + 1])])
        assert codecs.zstd_decompress(f, win.size) == win.tobytes()
        total += len(f)
    comp.close()
    assert sizes == [len(f) for f in frames]
    ratio = total / data.size
    assert 0.0 < ratio < 1.0


def test_level2_equals_level1(ctx):
    import gcz

    data = gcz.gen_synthetic(9, 3 << 20, 8 << 20)
    assert gcz.compress_chunk_zstd_custom(data, 0, 1) == gcz.compress_chunk_zstd_custom(data, 0, 2)


def test_nvzs_container_round_trip(ctx):
    from gcz import formats
    import gcz

    data = gcz.gen_synthetic(12, 2 << 20 | 777, 8 << 20)
    blob = formats.compress_zstd(data.tobytes(), level=1)
    assert formats.decompress(blob) == data.tobytes()


def _de_bruijn_window():
    # every 2-byte pair exactly once: no position of the window has a match
    k, n = 256, 2
    a = [0] * k * n
    seq = []

    def db(t, p):
        if t > n:
            if n % p == 0:
                seq.extend(a[1:p + 1])
        else:
            a[t] = a[t - p]
            db(t + 1, p)
            for j in range(a[t - p] + 1, k):
                a[t] = j
                db(t + 1, t)

    db(1, 1)
    return np.array(seq, dtype=np.uint8)


def test_nvlz_container_round_trip_and_raw_triage(ctx):
    """LZMA2 L1: a window with no match becomes raw LZMA2 chunks without
    liblzma (compress_lzma2_custom.rs:577-585); the others use preset 9."""
    import gcz
    from gcz import formats

    db = _de_bruijn_window()
    assert db.size == 65536
    text = cases.build({"kind": "text", "n": 65536 + 5000, "seed": 43})
    data = np.concatenate([text[:65536], db, text[65536:]])
    packed, has = ctx.lzma2_match_find(data)
    assert list(has) == [1, 0, 1]
    blob = formats.compress_lzma2(data.tobytes(), workers=3)
    _, _, _, chunks = formats.read_container(blob)
    assert chunks[1][0] == 0x01 and len(chunks[1]) == 65536 + 4  # raw chunk + end marker
    assert formats.decompress(blob) == data.tobytes()


def test_gpu_find_matches_then_encode(ctx):
    import gcz
    from gcz import codecs

    data = gcz.gen_synthetic(13, 4 * 65536, 128 << 20)
    md = gcz.gpu_find_matches(data, 0)
    for i in range(md.num_sub_blocks):
        sub = data[i * 65536:(i + 1) * 65536]
        block = gcz.encode_single_sub_block(sub, md.match_counts_of(i))
        assert codecs.lzma2_raw_decompress(block) == sub.tobytes()


@pytest.mark.parametrize("n,level,threads", [(40 * 65536 * 16 + 77, 1, 0), (5 * 65536 + 3, 2, 1), (1, 1, 3)])
def test_native_frames_equal_serial_libzstd(ctx, n, level, threads):
    """gcz_zstd_compress_frames (slices over GPU + coder pool) gives, window by
    window, the frame the serial ZSTD_compressSequences loop gives for the
    oracle's sequences; the 40 MiB case crosses the 32 MiB slice boundary."""
    import gcz
    from gcz import codecs

    data = gcz.gen_synthetic(200 + n % 97, n, 8 << 20)
    blob, sizes = ctx.zstd_compress_frames(data, level, threads)
    assert sizes.size == gcz.num_windows(n) and int(sizes.sum()) == blob.size
    o_seqs, o_off = orc.zstd_sequences(data, gcz.search_depth_for_level(level), threads=16)
    comp = codecs.SequenceCompressor()
    pos = 0
    for b in range(sizes.size):
        win = data[b * 65536:(b + 1) * 65536]
        f = blob[pos:pos + int(sizes[b])].tobytes()
        pos += int(sizes[b])
        assert f == comp.compress(win, o_seqs[int(o_off[b]):int(o_off[b + 1])]), b
        if b % 37 == 0:
            assert codecs.zstd_decompress(f, win.size) == win.tobytes()
    comp.close()


def test_native_frames_empty_and_capacity(ctx):
    import ctypes
    import gcz

    blob, sizes = ctx.zstd_compress_frames(np.zeros(0, np.uint8))
    assert blob.size == 0 and sizes.size == 0
    data = gcz.gen_synthetic(5, 3 * 65536, 8 << 20)
    out = np.empty(1000, np.uint8)
    fs = np.zeros(3, np.uint64)
    used = ctypes.c_size_t()
    rc = gcz.L.gcz_zstd_compress_frames(ctx.handle, data.ctypes.data, data.size, 1, 2, out.ctypes.data, out.size,
                                        fs.ctypes.data, ctypes.byref(used))
    assert rc == -4 and used.value == 0  # GCZ_ECAPACITY
    assert b"too small" in gcz.L.gcz_last_error(ctx.handle)


def test_nvzs_gpu_frames_and_file_batches_round_trip(ctx):
    import gcz
    from gcz import formats

    data = gcz.gen_synthetic(14, 3 * 65536 + 11, 8 << 20)
    assert formats.decompress(formats.compress_zstd_gpu(data.tobytes())) == data.tobytes()
    files = [gcz.gen_synthetic(15 + i, s, 8 << 20).tobytes() for i, s in enumerate([0, 5, 70000, 200000])]
    blobs = formats.compress_zstd_files(files)
    assert [formats.decompress(b) for b in blobs] == files


@pytest.mark.gpu
@pytest.mark.parametrize("gpu_coder", [False, True])
def test_c_example_writes_decodable_nvzs(ctx, tmp_path, gpu_coder):
    """gpu-compressor_b200/examples/gcz_compress.c, built with gcc against the C
    ABI only, writes an NVZS container that decodes to the input."""
    import os
    import subprocess
    import gcz
    from gcz import formats

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "gpu-compressor_b200", "gcz")
    exe = tmp_path / "gcz_compress"
    subprocess.run(["gcc", "-O2", "-I", os.path.join(root, "include"),
                    os.path.join(root, "gpu-compressor_b200", "examples", "gcz_compress.c"),
                    "-L", libdir, "-lgcz", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    data = gcz.gen_synthetic(31, 5 * 65536 + 123, 8 << 20)
    src, dst = tmp_path / "in.bin", tmp_path / "out.nvzs"
    src.write_bytes(data.tobytes())
    args = [str(exe), "-l", "2"] + (["-g"] if gpu_coder else []) + [str(src), str(dst)]
    subprocess.run(args, check=True, capture_output=True)
    assert formats.decompress(dst.read_bytes()) == data.tobytes()
