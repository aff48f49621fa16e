"""NVZS / NVLZ containers and the CPU codec stages (no GPU)."""
import numpy as np
import pytest

import cases
from oracle import oracle as orc


def test_container_round_trip_and_layout():
    from gcz import formats

    chunks = [b"abc", b"", b"x" * 70000]
    blob = formats.write_container(formats.MAGIC_ZSTD, 123456, 65536, chunks)
    assert blob[:4] == b"NVZS" and len(blob) == 28 + 8 * 3 + sum(map(len, chunks))
    assert int.from_bytes(blob[4:12], "little") == 123456
    assert int.from_bytes(blob[12:20], "little") == 65536
    assert int.from_bytes(blob[20:28], "little") == 3
    assert formats.read_container(blob) == (b"NVZS", 123456, 65536, chunks)


@pytest.mark.parametrize("bad", [b"", b"NVZX" + b"\0" * 24, b"NVZS" + b"\0" * 16 + (5).to_bytes(8, "little")])
def test_container_rejects_bad_input(bad):
    from gcz import formats

    with pytest.raises(ValueError):
        formats.read_container(bad)


def test_sequences_from_oracle_compress_and_decode():
    """The CPU half of compress_chunk_zstd_custom: oracle sequences through
    ZSTD_compressSequences decode back to the window (stock libzstd)."""
    from gcz import codecs

    data = cases.build({"kind": "synthetic", "n": 3 * 65536 + 999, "seed": 41})
    seqs, off = orc.zstd_sequences(data, 16)
    comp = codecs.SequenceCompressor()
    for b in range(off.size - 1):
        win = data[b * 65536:(b + 1) * 65536]
        frame = comp.compress(win, seqs[int(off[b]):int(off[b + 1])])
        assert codecs.zstd_decompress(frame, win.size) == win.tobytes()
    comp.close()


def test_lzma2_raw_paths_decode():
    from gcz import codecs

    data = cases.build({"kind": "text", "n": 70000, "seed": 42}).tobytes()
    assert codecs.lzma2_raw_decompress(codecs.lzma2_raw_compress(data[:65536])) == data[:65536]
    # uncompressed chunks + end marker (emit_raw_lzma2_chunks, compress_lzma2_custom.rs:325-338)
    raw = codecs.lzma2_raw_chunks(data)
    assert raw[0] == 0x01 and raw[65536 + 3] == 0x02 and raw[-1] == 0x00
    assert codecs.lzma2_raw_decompress(raw) == data


def test_frames_bound_is_sum_of_compress_bounds():
    import gcz
    from gcz import codecs

    zb = codecs.zstd().ZSTD_compressBound
    for n in [0, 1, 65535, 65536, 65537, 3 * 65536 + 5, 1 << 30]:
        want = sum(zb(min(65536, n - o)) for o in range(0, n, 65536))
        assert gcz.L.gcz_zstd_frames_bound(n) == want


def test_write_container_frames_matches_write_container():
    from gcz import formats

    chunks = [b"ab", b"", b"xyz" * 9]
    assert formats.write_container_frames(formats.MAGIC_ZSTD, 99, 65536, [len(c) for c in chunks],
                                          b"".join(chunks)) == formats.write_container(formats.MAGIC_ZSTD, 99,
                                                                                        65536, chunks)
