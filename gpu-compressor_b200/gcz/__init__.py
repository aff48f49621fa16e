"""gcz -- host side of the B200 match finders (libgcz) in the shape of
gpu-compressor's codec adapters.

    ctx = gcz.Context(device=0)
    seqs, offsets = ctx.zstd_match_find(data, search_depth=16)   # ZSTD_Sequence u32[N,4]
    packed, has = ctx.lzma2_match_find(data)                      # len<<16|dist per position

    frames, sizes = gcz.compress_chunk_zstd_custom(data, device_id=0, level=1)
    md = gcz.gpu_find_matches(data, device_id=0)                  # GpuMatchData
    block = gcz.encode_single_sub_block(sub, md.match_counts_of(i))

The adapter functions keep the names, arguments and results of the Rust
functions they stand in for (compress_zstd_custom.rs:47-203,
compress_lzma2_custom.rs:472-597); errors raise GczError.  All compute runs in
libgcz.so on the GPU -- there is no CPU fallback.
"""
import ctypes
import threading
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import WINDOW, ZSTD_MAX_SEQ_PER_WINDOW, LZMA2_MAX_MATCHES, LZMA2_SEARCH_DEPTH
from . import codecs

__all__ = [
    "Context", "GczError", "GpuMatchData", "compress_chunk_zstd_custom", "gpu_find_matches",
    "encode_single_sub_block", "search_depth_for_level", "gen_synthetic", "gen_file_sizes", "num_windows",
    "WINDOW", "ZSTD_MAX_SEQ_PER_WINDOW", "LZMA2_MAX_MATCHES", "LZMA2_SEARCH_DEPTH",
]

L = _lib.load()


class GczError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gcz error {code}: {msg}")
        self.code = code


def _u8(data):
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data.reshape(-1).view(np.uint8))
    return np.frombuffer(memoryview(data).cast("B"), dtype=np.uint8)


def _ptr(a):
    return a.ctypes.data if a is not None and a.size else None


def num_windows(n):
    return int(L.gcz_num_windows(n))


def search_depth_for_level(level):
    return int(L.gcz_zstd_search_depth_for_level(level))


CUDA_STREAM_LEGACY = 1  # (cudaStream_t)0x1


def _stream(s):
    """None -> the context's own stream; 0 (torch's default-stream handle) ->
    cudaStreamLegacy, so work stays ordered with torch's default stream."""
    if s is None:
        return None
    s = int(s)
    return CUDA_STREAM_LEGACY if s == 0 else s


class Context:
    """One device context of libgcz (gcz_create): stream and staging buffers
    are created once and reused across calls."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        rc = L.gcz_create(int(device), ctypes.byref(h))
        if rc != 0:
            raise GczError(rc, f"gcz_create(device={device}) failed")
        self._h = h
        self.device = int(device)
        self._lib = L  # kept for close() during interpreter shutdown, when module globals are gone

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gcz_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc):
        if rc != 0:
            raise GczError(rc, L.gcz_last_error(self._h).decode(errors="replace"))

    def set_option(self, key, value):
        self._check(L.gcz_set_option(self._h, key.encode(), int(value)))

    def query(self, key):
        v = ctypes.c_long()
        self._check(L.gcz_query(self._h, key.encode(), ctypes.byref(v)))
        return v.value

    def sync(self, stream=None):
        self._check(L.gcz_sync(self._h, _stream(stream)))

    # ------------------------------------------------------------ Zstd
    def zstd_match_find(self, data, search_depth=16):
        """ZSTD_Sequence records u32[N, 4] (offset, litLength, matchLength, rep)
        and per-window offsets u64[B+1]."""
        src = _u8(data)
        n = src.size
        cap = int(L.gcz_zstd_max_sequences(n))
        seqs = np.empty((max(cap, 1), 4), np.uint32)
        offsets = np.zeros(num_windows(n) + 1, np.uint64)
        self._check(L.gcz_zstd_match_find(self._h, _ptr(src), n, search_depth, seqs.ctypes.data, cap,
                                          offsets.ctypes.data))
        return seqs[:int(offsets[-1])], offsets

    def zstd_match_find_packed(self, data, search_depth=16):
        """8-byte records u64[N] (litLength | (matchLength-3) << 16 | offset << 32)
        and per-window offsets u64[B+1]; expand_packed() gives ZSTD_Sequence records."""
        src = _u8(data)
        n = src.size
        cap = int(L.gcz_zstd_max_sequences(n))
        recs = np.empty(max(cap, 1), np.uint64)
        offsets = np.zeros(num_windows(n) + 1, np.uint64)
        self._check(L.gcz_zstd_match_find_packed(self._h, _ptr(src), n, search_depth, recs.ctypes.data, cap,
                                                 offsets.ctypes.data))
        return recs[:int(offsets[-1])], offsets

    def zstd_match_find_device(self, d_src, n, search_depth, d_seqs, capacity, d_offsets, stream=None):
        """Device pointers (ints); enqueue only."""
        self._check(L.gcz_zstd_match_find_device(self._h, d_src, n, search_depth, d_seqs, capacity, d_offsets,
                                                 _stream(stream)))

    def zstd_match_find_ref_layout_device(self, d_input, d_sequences, d_literals, d_seq_counts, d_lit_counts,
                                          chunk_size, num_chunks, total_input_size, search_depth,
                                          max_sequences_per_chunk, stream=None):
        self._check(L.gcz_zstd_match_find_ref_layout_device(
            self._h, d_input, d_sequences, d_literals, d_seq_counts, d_lit_counts, chunk_size, num_chunks,
            total_input_size, search_depth, max_sequences_per_chunk, _stream(stream)))

    # ------------------------------------------------------------ LZMA2
    def lzma2_match_find(self, data, search_depth=LZMA2_SEARCH_DEPTH):
        """packed u32[n] (len<<16 | dist, 0 = none) and has_matches u8[B]."""
        src = _u8(data)
        n = src.size
        packed = np.empty(max(n, 1), np.uint32)
        has = np.zeros(max(num_windows(n), 1), np.uint8)
        self._check(L.gcz_lzma2_match_find(self._h, _ptr(src), n, search_depth, packed.ctypes.data,
                                           has.ctypes.data))
        return packed[:n], has[:num_windows(n)]

    def lzma2_triage(self, data, search_depth=LZMA2_SEARCH_DEPTH):
        """has_matches u8[B] only: the per-window bit the LZMA2 L1+ encoder
        consumes (compress_lzma2_custom.rs:577); no per-position results cross
        back to the host."""
        src = _u8(data)
        n = src.size
        has = np.zeros(max(num_windows(n), 1), np.uint8)
        self._check(L.gcz_lzma2_match_find(self._h, _ptr(src), n, search_depth, None, has.ctypes.data))
        return has[:num_windows(n)]

    def lzma2_match_find_device(self, d_src, n, search_depth, d_packed, d_has, stream=None):
        self._check(L.gcz_lzma2_match_find_device(self._h, d_src, n, search_depth, d_packed, d_has, _stream(stream)))

    def lzma2_find_matches(self, data, max_matches=LZMA2_MAX_MATCHES):
        """GpuMatchData arrays (zero-filled, de-interleaved)."""
        src = _u8(data)
        n = src.size
        B = num_windows(n)
        counts = np.empty(B * WINDOW, np.uint32)
        dists = np.empty(B * WINDOW * max_matches, np.uint32)
        lens = np.empty(B * WINDOW * max_matches, np.uint32)
        self._check(L.gcz_lzma2_find_matches(self._h, _ptr(src), n, max_matches, _ptr(dists), _ptr(lens),
                                             _ptr(counts)))
        return dists, lens, counts

    def lzma2_match_find_ref_layout_device(self, d_input, d_matches, d_counts, sub_block_size, num_sub_blocks,
                                           total_input_size, max_matches_per_pos, search_depth, stream=None):
        self._check(L.gcz_lzma2_match_find_ref_layout_device(self._h, d_input, d_matches, d_counts, sub_block_size,
                                                             num_sub_blocks, total_input_size, max_matches_per_pos,
                                                             search_depth, _stream(stream)))

    # ------------------------------------------------------------ batches
    def zstd_match_find_files(self, files, search_depth=16):
        """Many host inputs in one launch: ZSTD_Sequence records u32[N, 4] and
        per-window offsets u64[W+1] (windows of all files, in file order)."""
        arrs = [_u8(f) for f in files]
        k = len(arrs)
        sizes = (ctypes.c_size_t * k)(*[a.size for a in arrs])
        ptrs = (ctypes.c_void_p * k)(*[a.ctypes.data if a.size else None for a in arrs])
        nb = int(L.gcz_batch_num_windows(sizes, k))
        cap = sum(int(L.gcz_zstd_max_sequences(a.size)) for a in arrs)
        seqs = np.empty((max(cap, 1), 4), np.uint32)
        offsets = np.zeros(nb + 1, np.uint64)
        self._check(L.gcz_zstd_match_find_files(self._h, ptrs, sizes, k, search_depth, seqs.ctypes.data, cap,
                                                offsets.ctypes.data))
        return seqs[:int(offsets[-1])], offsets

    def zstd_match_find_batch_device(self, d_slab, slab_bytes, d_windows, num_windows, search_depth, d_seqs,
                                     capacity, d_offsets, stream=None):
        self._check(L.gcz_zstd_match_find_batch_device(self._h, d_slab, slab_bytes, d_windows, num_windows,
                                                       search_depth, d_seqs, capacity, d_offsets, _stream(stream)))

    def lzma2_match_find_batch_device(self, d_slab, slab_bytes, d_windows, num_windows, search_depth, d_packed,
                                      d_has, stream=None):
        self._check(L.gcz_lzma2_match_find_batch_device(self._h, d_slab, slab_bytes, d_windows, num_windows,
                                                        search_depth, d_packed, d_has, _stream(stream)))

    # ------------------------------------------------------------ frames
    def zstd_compress_frames(self, data, level=1, threads=0):
        """One Zstd frame per 64 KiB window (GPU sequences, libzstd
        ZSTD_compressSequences on `threads` CPU threads, 0 = all cores):
        (frames bytes back to back, frame sizes u64[B])."""
        src = _u8(data)
        n = src.size
        out = np.empty(max(int(L.gcz_zstd_frames_bound(n)), 1), np.uint8)
        sizes = np.zeros(max(num_windows(n), 1), np.uint64)
        used = ctypes.c_size_t()
        self._check(L.gcz_zstd_compress_frames(self._h, _ptr(src), n, level, threads, out.ctypes.data, out.size,
                                               sizes.ctypes.data, ctypes.byref(used)))
        return out[:used.value], sizes[:num_windows(n)]

    def zstd_compress_frames_gpu(self, data, level=1):
        """One Zstd frame per 64 KiB window, encoded on the GPU (raw, RLE or
        Huffman literals; RLE, FSE-compressed or predefined sequence tables): (frames back to back,
        frame sizes u64[B])."""
        src = _u8(data)
        n = src.size
        out = np.empty(max(int(L.gcz_zstd_frames_bound(n)), 1), np.uint8)
        sizes = np.zeros(max(num_windows(n), 1), np.uint64)
        used = ctypes.c_size_t()
        self._check(L.gcz_zstd_compress_frames_gpu(self._h, _ptr(src), n, level, out.ctypes.data, out.size,
                                                   sizes.ctypes.data, ctypes.byref(used)))
        return out[:used.value], sizes[:num_windows(n)]

    def zstd_compress_files_gpu(self, files, level=1):
        """GPU frames of many host files in one launch of each kernel: a list
        with, per file, the list of its frames (one per 64 KiB window)."""
        arrs = [_u8(f) for f in files]
        k = len(arrs)
        sizes = (ctypes.c_size_t * k)(*[a.size for a in arrs])
        ptrs = (ctypes.c_void_p * k)(*[a.ctypes.data if a.size else None for a in arrs])
        nb = int(L.gcz_batch_num_windows(sizes, k))
        bound = sum(int(L.gcz_zstd_frames_bound(a.size)) for a in arrs)
        out = np.empty(max(bound, 1), np.uint8)
        fs = np.zeros(max(nb, 1), np.uint64)
        used = ctypes.c_size_t()
        self._check(L.gcz_zstd_compress_files_gpu(self._h, ptrs, sizes, k, level, out.ctypes.data, out.size,
                                                  fs.ctypes.data, ctypes.byref(used)))
        res, pos, w = [], 0, 0
        for a in arrs:
            frames = []
            for _ in range(num_windows(a.size)):
                s = int(fs[w])
                frames.append(out[pos:pos + s].tobytes())
                pos += s
                w += 1
            res.append(frames)
        return res

    def zstd_encode_frames_batch_device(self, d_slab, slab_bytes, d_windows, num_windows, d_seqs, d_seq_offsets,
                                        d_out, out_capacity, d_frame_offsets, stream=None):
        self._check(L.gcz_zstd_encode_frames_batch_device(self._h, d_slab, slab_bytes, d_windows, num_windows, d_seqs,
                                                          d_seq_offsets, d_out, out_capacity, d_frame_offsets,
                                                          _stream(stream)))

    def zstd_encode_frames_device(self, d_src, n, d_seqs, d_seq_offsets, d_out, out_capacity, d_frame_offsets,
                                  stream=None):
        self._check(L.gcz_zstd_encode_frames_device(self._h, d_src, n, d_seqs, d_seq_offsets, d_out, out_capacity,
                                                    d_frame_offsets, _stream(stream)))

    # ------------------------------------------------------------ timing
    def profile_start(self):
        self._check(L.gcz_profile_start(self._h))

    def profile_stop(self):
        ms, k, a = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64()
        self._check(L.gcz_profile_stop(self._h, ctypes.byref(ms), ctypes.byref(k), ctypes.byref(a)))
        return ms.value, k.value, a.value


_contexts = {}
_ctx_lock = threading.Lock()


def context(device_id=0):
    """The process-wide Context of a device (created on first use)."""
    with _ctx_lock:
        c = _contexts.get(device_id)
        if c is None:
            c = _contexts[device_id] = Context(device_id)
        return c


# ---------------------------------------------------------------- adapters

def compress_chunk_zstd_custom(chunk_data, device_id=0, level=1):
    """compress_chunk_zstd_custom (compress_zstd_custom.rs:47-203): GPU match
    finding per 64 KiB window, then one Zstd frame per window through libzstd's
    ZSTD_compressSequences (gcz_zstd_compress_frames: a pool of CPU coder
    threads encodes one slice while the GPU matches the next).  Returns
    (frames, sizes)."""
    data = _u8(chunk_data)
    blob, fsizes = context(device_id).zstd_compress_frames(data, level)
    frames, pos = [], 0
    for s in fsizes.tolist():
        frames.append(blob[pos:pos + s].tobytes())
        pos += s
    return frames, [len(f) for f in frames]


@dataclass
class GpuMatchData:
    """compress_lzma2_custom.rs:472-479."""
    match_distances: np.ndarray
    match_lengths: np.ndarray
    match_counts: np.ndarray
    num_sub_blocks: int
    sub_block_size: int
    max_matches: int

    def match_counts_of(self, i):
        return self.match_counts[i * self.sub_block_size:(i + 1) * self.sub_block_size]


def gpu_find_matches(chunk_data, device_id=0):
    """gpu_find_matches (compress_lzma2_custom.rs:483-560)."""
    data = _u8(chunk_data)
    d, l, c = context(device_id).lzma2_find_matches(data, LZMA2_MAX_MATCHES)
    return GpuMatchData(d, l, c, num_windows(data.size), WINDOW, LZMA2_MAX_MATCHES)


def encode_single_sub_block(sub_data, match_counts, match_distances=None, match_lengths=None, max_matches=8):
    """encode_single_sub_block (compress_lzma2_custom.rs:570-597): raw LZMA2
    chunks when the GPU found no match in the window, else liblzma preset 9."""
    has = bool(np.any(np.asarray(match_counts)))
    data = bytes(_u8(sub_data))
    if not has:
        return codecs.lzma2_raw_chunks(data)
    try:
        return codecs.lzma2_raw_compress(data, 9)
    except Exception:  # liblzma error -> raw, like the reference (:589-595)
        return codecs.lzma2_raw_chunks(data)


# ---------------------------------------------------------------- inputs

def gen_synthetic(seed, n, max_offset=8 << 20, mix=(0.4, 0.4, 0.2), out=None):
    """Seeded synthetic bytes (include/gcz_gen.h)."""
    if out is None:
        out = np.empty(n, np.uint8)
    if n:
        L.gcz_gen_synthetic(seed, out.ctypes.data, n, max_offset, float(mix[0]), float(mix[1]), float(mix[2]))
    return out


def expand_packed(records):
    """ZSTD_Sequence records u32[N, 4] (offset, litLength, matchLength, rep = 0)
    from gcz_zstd_match_find_packed's 8-byte records: the caller-side loop."""
    r = np.asarray(records, dtype=np.uint64)
    out = np.zeros((r.size, 4), np.uint32)
    out[:, 0] = (r >> np.uint64(32)).astype(np.uint32)
    out[:, 1] = (r & np.uint64(0xFFFF)).astype(np.uint32)
    out[:, 2] = ((r >> np.uint64(16)) & np.uint64(0xFFFF)).astype(np.uint32) + 3
    return out


WINDOW_DTYPE = np.dtype([("offset", "<u8"), ("size", "<u4"), ("file", "<u4")])  # gcz_window


def batch_layout(sizes):
    """(file offsets u64[k], window table (WINDOW_DTYPE)[W], slab bytes) of a batch."""
    sizes = [int(x) for x in sizes]
    k = len(sizes)
    cs = (ctypes.c_size_t * k)(*sizes)
    nb = int(L.gcz_batch_num_windows(cs, k))
    foff = np.zeros(max(k, 1), np.uint64)
    wins = np.zeros(max(nb, 1), WINDOW_DTYPE)
    slab = ctypes.c_uint64()
    rc = L.gcz_batch_layout(cs, k, foff.ctypes.data, wins.ctypes.data, ctypes.byref(slab))
    if rc != 0:
        raise GczError(rc, "gcz_batch_layout failed")
    return foff[:k], wins[:nb], slab.value


def gen_file_sizes(seed, count, min_size=4096, max_size=64 << 20):
    sizes = np.empty(count, np.uint64)
    mix = np.empty((count, 3), np.float64)
    if count:
        L.gcz_gen_file_sizes(seed, count, min_size, max_size, sizes.ctypes.data, mix.ctypes.data)
    return sizes, mix
