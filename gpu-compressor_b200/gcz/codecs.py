"""CPU entropy stages the reference runs after its kernels, through the same
system libraries it links or dlopens: libzstd (ZSTD_compressSequences,
compress_zstd_custom.rs:16-40,157-199) and liblzma (raw LZMA2 preset 9,
compress_lzma2.rs:89-133, here through Python's lzma module which binds the
same liblzma).  No headers are needed; prototypes are declared here.
"""
import ctypes
import ctypes.util
import lzma

import numpy as np

ZSTD_RESET_SESSION_ONLY = 1
ZSTD_CONTENTSIZE_ERROR = 2**64 - 2
ZSTD_CONTENTSIZE_UNKNOWN = 2**64 - 1

_zstd = None


def zstd():
    global _zstd
    if _zstd is None:
        name = ctypes.util.find_library("zstd") or "libzstd.so.1"
        L = ctypes.CDLL(name)
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        L.ZSTD_createCCtx.restype = vp
        L.ZSTD_freeCCtx.argtypes = [vp]
        L.ZSTD_freeCCtx.restype = sz
        L.ZSTD_CCtx_reset.argtypes = [vp, ctypes.c_uint]
        L.ZSTD_CCtx_reset.restype = sz
        L.ZSTD_CCtx_setParameter.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.ZSTD_CCtx_setParameter.restype = sz
        L.ZSTD_compressSequences.argtypes = [vp, vp, sz, vp, sz, vp, sz]
        L.ZSTD_compressSequences.restype = sz
        L.ZSTD_isError.argtypes = [sz]
        L.ZSTD_isError.restype = ctypes.c_uint
        L.ZSTD_getErrorName.argtypes = [sz]
        L.ZSTD_getErrorName.restype = ctypes.c_char_p
        L.ZSTD_compressBound.argtypes = [sz]
        L.ZSTD_compressBound.restype = sz
        L.ZSTD_compress.argtypes = [vp, sz, vp, sz, ctypes.c_int]
        L.ZSTD_compress.restype = sz
        L.ZSTD_decompress.argtypes = [vp, sz, vp, sz]
        L.ZSTD_decompress.restype = sz
        L.ZSTD_getFrameContentSize.argtypes = [vp, sz]
        L.ZSTD_getFrameContentSize.restype = ctypes.c_ulonglong
        _zstd = L
    return _zstd


class SequenceCompressor:
    """One ZSTD_CCtx used the way compress_chunk_zstd_custom uses it: parameter
    1001 set to 0 once (:128), a session reset before every window (:161),
    ZSTD_compressSequences with the window's sequences and bytes (:163-171),
    and ZSTD_compress level 1 as the fallback on error (:173-190)."""

    def __init__(self):
        L = zstd()
        self.L = L
        self.cctx = L.ZSTD_createCCtx()
        if not self.cctx:
            raise MemoryError("ZSTD_createCCtx failed")
        L.ZSTD_CCtx_setParameter(self.cctx, 1001, 0)

    def close(self):
        if self.cctx:
            self.L.ZSTD_freeCCtx(self.cctx)
            self.cctx = None

    def __del__(self):
        self.close()

    def compress(self, window_bytes, seqs):
        """window_bytes: bytes-like; seqs: u32[k, 4] ZSTD_Sequence records."""
        L = self.L
        src = np.frombuffer(window_bytes, dtype=np.uint8) if not isinstance(window_bytes, np.ndarray) else window_bytes
        src = np.ascontiguousarray(src, dtype=np.uint8)
        sq = np.ascontiguousarray(seqs, dtype=np.uint32)
        bound = L.ZSTD_compressBound(src.size)
        out = np.empty(bound, np.uint8)
        L.ZSTD_CCtx_reset(self.cctx, ZSTD_RESET_SESSION_ONLY)
        ret = L.ZSTD_compressSequences(self.cctx, out.ctypes.data, bound, sq.ctypes.data if sq.size else None,
                                       sq.shape[0] if sq.ndim == 2 else 0, src.ctypes.data, src.size)
        if L.ZSTD_isError(ret):
            fb = L.ZSTD_compress(out.ctypes.data, bound, src.ctypes.data, src.size, 1)
            if L.ZSTD_isError(fb):
                raise RuntimeError("zstd: " + L.ZSTD_getErrorName(ret).decode())
            ret = fb
        return out[:ret].tobytes()


def zstd_decompress(frame, size_hint=None):
    L = zstd()
    f = np.frombuffer(frame, dtype=np.uint8)
    size = L.ZSTD_getFrameContentSize(f.ctypes.data, f.size)
    if size in (ZSTD_CONTENTSIZE_ERROR, ZSTD_CONTENTSIZE_UNKNOWN):
        size = size_hint if size_hint is not None else 1 << 20
    out = np.empty(max(int(size), 1), np.uint8)
    r = L.ZSTD_decompress(out.ctypes.data, out.size, f.ctypes.data, f.size)
    if L.ZSTD_isError(r):
        raise RuntimeError("zstd decompress: " + L.ZSTD_getErrorName(r).decode())
    return out[:r].tobytes()


def zstd_compress_level(data, level=1):
    L = zstd()
    src = np.frombuffer(data, dtype=np.uint8)
    bound = L.ZSTD_compressBound(src.size)
    out = np.empty(bound, np.uint8)
    r = L.ZSTD_compress(out.ctypes.data, bound, src.ctypes.data, src.size, level)
    if L.ZSTD_isError(r):
        raise RuntimeError("zstd: " + L.ZSTD_getErrorName(r).decode())
    return out[:r].tobytes()


# ----------------------------------------------------------------- LZMA2

LZMA2_RAW_FILTERS_P9 = [{"id": lzma.FILTER_LZMA2, "preset": 9}]


def lzma2_raw_compress(data, preset=9):
    """Raw LZMA2 stream of `data` at `preset` (compress_chunk_lzma2, compress_lzma2.rs:85-133)."""
    return lzma.compress(bytes(data), format=lzma.FORMAT_RAW, filters=[{"id": lzma.FILTER_LZMA2, "preset": preset}])


def lzma2_raw_decompress(stream, dict_size=64 << 20):
    """Raw LZMA2 decode (decompress_chunk_lzma2, compress_lzma2.rs:135-172)."""
    return lzma.decompress(bytes(stream), format=lzma.FORMAT_RAW,
                           filters=[{"id": lzma.FILTER_LZMA2, "dict_size": dict_size}])


def lzma2_raw_chunks(data):
    """Uncompressed LZMA2 chunks of <= 64 KiB plus the 0x00 end marker
    (emit_raw_lzma2_chunks + push(0), compress_lzma2_custom.rs:325-338,579-585)."""
    out = bytearray()
    off, first = 0, True
    while off < len(data):
        n = min(len(data) - off, 65536)
        out.append(0x01 if first else 0x02)
        us = n - 1
        out.append((us >> 8) & 0xFF)
        out.append(us & 0xFF)
        out += data[off:off + n]
        off += n
        first = False
    out.append(0x00)
    return bytes(out)
