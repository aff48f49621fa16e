"""Shared test helpers: sequence decoding and match validation."""
import numpy as np


def decode_window(window_bytes, seqs):
    """Rebuild a window from ZSTD_Sequence records (offset, litLength,
    matchLength, rep) with the literals taken from the original bytes; the
    trailing literals are implicit (compress_zstd_custom.rs:155-156).  Returns
    the rebuilt bytes -- equal to the input iff every match is genuine."""
    src = bytes(window_bytes)
    out = bytearray()
    pos = 0
    for off, ll, ml, _rep in np.asarray(seqs, dtype=np.int64).reshape(-1, 4):
        out += src[pos:pos + ll]
        pos += ll
        start = len(out) - off
        assert off >= 1 and start >= 0, (off, len(out))
        for i in range(ml):
            out.append(out[start + i])
        pos += ml
    assert pos <= len(src)
    out += src[pos:]
    return bytes(out)


def check_lzma_packed(data, packed, window=65536):
    """Every recorded match is genuine and stays inside its window."""
    d = np.asarray(data, dtype=np.uint8)
    idx = np.nonzero(packed)[0]
    for q in idx:
        v = int(packed[q])
        dist, ln = v & 0xFFFF, v >> 16
        w0 = (q // window) * window
        assert 2 <= ln <= 273
        assert q - dist >= w0
        assert q + ln <= min(w0 + window, d.size)
        assert bytes(d[q - dist:q - dist + ln]) == bytes(d[q:q + ln]) or dist < ln
        # overlapping copy (dist < len): byte-by-byte semantics
        for i in range(ln):
            assert d[q + i] == d[q - dist + i]
