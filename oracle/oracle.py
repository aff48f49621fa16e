"""ctypes front end of the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: the checker the B200 kernels are compared against.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
GEN_PATH = os.path.join(HERE, "_build", "libgen.so")
WINDOW = 65536
MAX_SEQS = WINDOW // 3  # compress_zstd_custom.rs:55

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
        L.oracle_zstd_match_find.argtypes = [vp, u64, u32, u32, u32, vp, vp, vp, vp, ctypes.c_int]
        L.oracle_zstd_match_find.restype = None
        L.oracle_lzma2_match_find.argtypes = [vp, u64, u32, u32, u32, vp, vp, vp, ctypes.c_int]
        L.oracle_lzma2_match_find.restype = None
        _lib = L
    return _lib


_gen = None


def gen_synthetic(seed, n, max_offset=8 << 20, mix=(0.4, 0.4, 0.2)):
    """The seeded synthetic input (include/gcz_gen.h) from _build/libgen.so,
    byte for byte what gcz.gen_synthetic gives, without loading libgcz.so."""
    global _gen
    if _gen is None:
        if not os.path.exists(GEN_PATH):
            build()
        g = ctypes.CDLL(GEN_PATH)
        g.gcz_gen_synthetic.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double]
        g.gcz_gen_synthetic.restype = None
        _gen = g
    out = np.empty(n, np.uint8)
    if n:
        _gen.gcz_gen_synthetic(seed, out.ctypes.data, n, max_offset, float(mix[0]), float(mix[1]), float(mix[2]))
    return out


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _u8(buf):
    return np.ascontiguousarray(np.frombuffer(buf, dtype=np.uint8) if not isinstance(buf, np.ndarray) else buf,
                                dtype=np.uint8)


def num_windows(n, window=WINDOW):
    return (n + window - 1) // window


def zstd_ref_layout(buf, search_depth=16, window=WINDOW, max_seqs=None, literals=True, threads=8):
    """Outputs of zstd_match_find in its own layout (zstd_compress.cu:179-190):
    (sequences u32[B, max_seqs, 3], literals u8[B*window] or None, seq_counts u32[B], lit_counts u32[B]).
    Unwritten slots are zero, as after the reference host's alloc_zeros."""
    a = _u8(buf)
    n = a.size
    if max_seqs is None:
        max_seqs = window // 3
    B = num_windows(n, window)
    seqs = np.zeros((max(B, 1), max_seqs, 3), np.uint32)
    lits = np.zeros(max(B, 1) * window, np.uint8) if literals else None
    sc = np.zeros(max(B, 1), np.uint32)
    lc = np.zeros(max(B, 1), np.uint32)
    lib().oracle_zstd_match_find(_ptr(a), n, window, search_depth, max_seqs, _ptr(seqs), _ptr(lits), _ptr(sc),
                                 _ptr(lc), threads)
    return seqs[:B], (lits[:B * window] if literals else None), sc[:B], lc[:B]


def zstd_sequences(buf, search_depth=16, window=WINDOW, threads=8):
    """Compact ZSTD_Sequence records (offset, litLength, matchLength, rep) as u32[N, 4]
    plus per-window offsets u64[B+1] -- what compress_zstd_custom.rs:137-153 builds."""
    a = _u8(buf)
    n = a.size
    B = num_windows(n, window)
    slice_windows = 2048  # bounds the strided scratch to ~0.5 GB
    parts, counts = [], []
    for b0 in range(0, B, slice_windows):
        b1 = min(B, b0 + slice_windows)
        seqs, _, sc, _ = zstd_ref_layout(a[b0 * window:min(n, b1 * window)], search_depth, window,
                                         literals=False, threads=threads)
        mask = np.arange(seqs.shape[1])[None, :] < sc[:, None]
        s = seqs[mask]  # row-major: window by window, in order
        part = np.zeros((s.shape[0], 4), np.uint32)
        part[:, 0] = s[:, 2]
        part[:, 1] = s[:, 0]
        part[:, 2] = s[:, 1] + 3
        parts.append(part)
        counts.append(sc)
    offsets = np.zeros(B + 1, np.uint64)
    if B:
        offsets[1:] = np.cumsum(np.concatenate(counts), dtype=np.uint64)
    out = np.concatenate(parts) if parts else np.zeros((0, 4), np.uint32)
    return out, offsets


def lzma_packed(buf, search_depth=32, window=WINDOW, threads=8):
    """Per-position len<<16|dist (0 = no match), u32[n]."""
    a = _u8(buf)
    n = a.size
    packed = np.zeros(max(n, 1), np.uint32)
    lib().oracle_lzma2_match_find(_ptr(a), n, window, 8, search_depth, None, None, _ptr(packed), threads)
    return packed[:n]


def lzma_ref_layout(buf, max_matches=8, search_depth=32, window=WINDOW, threads=8):
    """Outputs of lzma2_match_find in its own layout (lzma2_match_find.cu:54-63):
    (matches u32[B*window, max_matches, 2] zero-filled, counts u32[B*window])."""
    a = _u8(buf)
    n = a.size
    B = num_windows(n, window)
    match = np.zeros((max(B, 1) * window, max_matches, 2), np.uint32)
    counts = np.zeros(max(B, 1) * window, np.uint32)
    lib().oracle_lzma2_match_find(_ptr(a), n, window, max_matches, search_depth, _ptr(match), _ptr(counts), None,
                                  threads)
    return match[:B * window], counts[:B * window]


def has_matches(packed, n, window=WINDOW):
    """any(match_counts > 0) per window (compress_lzma2_custom.rs:577)."""
    B = num_windows(n, window)
    out = np.zeros(B, np.uint8)
    for b in range(B):
        out[b] = 1 if np.any(packed[b * window:(b + 1) * window]) else 0
    return out
