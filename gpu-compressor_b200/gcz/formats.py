"""NVZS / NVLZ containers and whole-buffer compress / decompress on top of the
GPU match finders.

Container (pipeline.rs:196-203,245-253; pipeline_lzma2.rs:347-354,391-396):
    magic  b"NVZS" (Zstd) or b"NVLZ" (LZMA2)          4 bytes
    original size                                      u64 LE
    chunk size (65536 for the match-finder levels)     u64 LE
    number of chunks                                   u64 LE
    compressed size of every chunk                     u64 LE each
    the chunks, in order
Each chunk of a match-finder level is one independent 64 KiB window: a Zstd
frame (ZSTD_compressSequences over the GPU sequences) or a raw LZMA2 stream
(liblzma preset 9, or raw chunks when the GPU found no match in the window).
"""
import os
import struct
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import codecs

MAGIC_ZSTD = b"NVZS"
MAGIC_LZMA2 = b"NVLZ"
HEADER = struct.Struct("<4sQQQ")
WINDOW = 65536


def write_container(magic, orig_size, chunk_size, chunks):
    """Serialise chunks into one NVZS/NVLZ byte string."""
    parts = [HEADER.pack(magic, orig_size, chunk_size, len(chunks))]
    parts.append(struct.pack(f"<{len(chunks)}Q", *[len(c) for c in chunks]) if chunks else b"")
    parts.extend(chunks)
    return b"".join(parts)


def read_container(blob):
    """(magic, orig_size, chunk_size, [chunk bytes])."""
    mv = memoryview(blob)
    if len(mv) < HEADER.size:
        raise ValueError("truncated header")
    magic, orig, chunk_size, n = HEADER.unpack_from(mv, 0)
    if magic not in (MAGIC_ZSTD, MAGIC_LZMA2):
        raise ValueError("Invalid file format (expected NVZS or NVLZ)")
    off = HEADER.size
    if len(mv) < off + 8 * n:
        raise ValueError("truncated size table")
    sizes = struct.unpack_from(f"<{n}Q", mv, off) if n else ()
    off += 8 * n
    chunks = []
    for s in sizes:
        if off + s > len(mv):
            raise ValueError("truncated chunk")
        chunks.append(bytes(mv[off:off + s]))
        off += s
    return magic, orig, chunk_size, chunks


def write_container_frames(magic, orig_size, chunk_size, sizes, blob):
    """write_container for chunks already laid out back to back in `blob`."""
    sizes = [int(x) for x in sizes]
    head = HEADER.pack(magic, orig_size, chunk_size, len(sizes))
    return head + (struct.pack(f"<{len(sizes)}Q", *sizes) if sizes else b"") + bytes(blob)


def compress_zstd(data, level=1, device_id=0, threads=0):
    """NVZS with one Zstd frame per 64 KiB window (the Zstd L1/L2 path);
    `threads` CPU coder threads (0 = all cores)."""
    from . import context

    buf = np.frombuffer(memoryview(data).cast("B"), dtype=np.uint8)
    if buf.size == 0:
        return write_container(MAGIC_ZSTD, 0, WINDOW, [])
    blob, sizes = context(device_id).zstd_compress_frames(buf, level, threads)
    return write_container_frames(MAGIC_ZSTD, buf.size, WINDOW, sizes, blob)


def compress_zstd_gpu(data, level=1, device_id=0):
    """NVZS with frames built on the GPU (gcz_zstd_compress_frames_gpu): the
    same container, decodable by the same reader and stock libzstd."""
    from . import context

    buf = np.frombuffer(memoryview(data).cast("B"), dtype=np.uint8)
    if buf.size == 0:
        return write_container(MAGIC_ZSTD, 0, WINDOW, [])
    blob, sizes = context(device_id).zstd_compress_frames_gpu(buf, level)
    return write_container_frames(MAGIC_ZSTD, buf.size, WINDOW, sizes, blob)


def compress_zstd_files(files, level=1, device_id=0):
    """One NVZS container per file for a whole batch, with one launch of each
    GPU kernel for all of them (gcz_zstd_compress_files_gpu)."""
    from . import context

    bufs = [np.frombuffer(memoryview(f).cast("B"), dtype=np.uint8) for f in files]
    frames = context(device_id).zstd_compress_files_gpu(bufs, level)
    return [write_container(MAGIC_ZSTD, b.size, WINDOW, fr) for b, fr in zip(bufs, frames)]


def compress_lzma2(data, device_id=0, workers=None):
    """NVLZ with one raw LZMA2 stream per 64 KiB window (the LZMA2 L1+ path):
    the GPU decides per window whether liblzma preset 9 runs at all, a pool of
    min(ncpu, 8) encoder threads does the coding (pipeline_lzma2.rs:226-245)."""
    from . import context, encode_single_sub_block, num_windows

    buf = np.frombuffer(memoryview(data).cast("B"), dtype=np.uint8)
    if buf.size == 0:
        return write_container(MAGIC_LZMA2, 0, WINDOW, [])
    has = context(device_id).lzma2_triage(buf)
    nb = num_windows(buf.size)
    workers = workers or min(os.cpu_count() or 1, 8)

    def enc(b):
        sub = buf[b * WINDOW:(b + 1) * WINDOW]
        return encode_single_sub_block(sub, np.array([has[b]], np.uint32))

    with ThreadPoolExecutor(workers) as ex:
        chunks = list(ex.map(enc, range(nb)))
    return write_container(MAGIC_LZMA2, buf.size, WINDOW, chunks)


def decompress(blob):
    """Original bytes of an NVZS/NVLZ container, through stock libzstd / liblzma."""
    magic, orig, chunk_size, chunks = read_container(blob)
    out = bytearray()
    for i, c in enumerate(chunks):
        want = min(chunk_size, orig - i * chunk_size)
        if magic == MAGIC_ZSTD:
            out += codecs.zstd_decompress(c, want)
        else:
            out += codecs.lzma2_raw_decompress(c)
    if len(out) != orig:
        raise ValueError(f"decoded {len(out)} bytes, header says {orig}")
    return bytes(out)
