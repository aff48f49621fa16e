"""Python front end of the libgcz request loop (gcz_server_* in include/gcz.h)."""
import ctypes
import threading

import numpy as np

from . import L, GczError, num_windows, _u8

ZSTD, LZMA2, ZSTD_FRAMES = 0, 1, 2


class Request:
    """One submitted request; keeps its input and output buffers alive.

    out_a / out_b may be supplied (e.g. pinned, reused buffers): Zstd needs
    out_a u32[cap, 4] and out_b u64[windows+1]; LZMA2 takes out_a u32[n] or
    None (only the per-window has-match bytes, what the LZMA2 consumer reads)
    and out_b u8[windows]; ZSTD_FRAMES (frames built on the GPU) needs out_a
    u8[cap] and out_b u64[windows] (frame sizes)."""

    def __init__(self, kind, data, depth, out_a=None, out_b=None, cap=None, packed=True):
        self.kind = kind
        self.data = _u8(data)
        self.depth = depth
        n = self.data.size
        nb = num_windows(n)
        if kind == ZSTD:
            self.cap = int(L.gcz_zstd_max_sequences(n)) if cap is None else int(cap)
            self.out_a = np.empty((max(self.cap, 1), 4), np.uint32) if out_a is None else out_a
            self.out_b = np.zeros(nb + 1, np.uint64) if out_b is None else out_b
        elif kind == ZSTD_FRAMES:
            self.cap = int(L.gcz_zstd_frames_bound(n)) if cap is None else int(cap)
            self.out_a = np.empty(max(self.cap, 1), np.uint8) if out_a is None else out_a
            self.out_b = np.zeros(max(nb, 1), np.uint64) if out_b is None else out_b
        else:
            self.cap = n
            self.out_a = (np.empty(max(n, 1), np.uint32) if out_a is None else out_a) if packed else None
            self.out_b = np.zeros(max(nb, 1), np.uint8) if out_b is None else out_b
        self.id = None
        self.latency_ms = None

    def result(self):
        nb = num_windows(self.data.size)
        if self.kind == ZSTD:
            return self.out_a[:int(self.out_b[nb])], self.out_b[:nb + 1]
        if self.kind == ZSTD_FRAMES:  # the frames, one per window
            frames, pos = [], 0
            for s in self.out_b[:nb].tolist():
                frames.append(self.out_a[pos:pos + s].tobytes())
                pos += s
            return frames
        return (self.out_a[:self.data.size] if self.out_a is not None else None), self.out_b[:nb]


class Server:
    def __init__(self, ctx, hbm_budget=120 * 10**9, max_batch_bytes=0, max_batch_requests=0):
        h = ctypes.c_void_p()
        rc = L.gcz_server_create(ctx.handle, int(hbm_budget), int(max_batch_bytes), int(max_batch_requests),
                                 ctypes.byref(h))
        if rc != 0:
            raise GczError(rc, L.gcz_last_error(ctx.handle).decode(errors="replace"))
        self._h = h
        self._lock = threading.Lock()
        self.ctx = ctx
        self._lib = L  # kept for close() during interpreter shutdown

    @property
    def max_batch_bytes(self):
        return int(L.gcz_server_max_batch_bytes(self._h))

    def warm_up(self, kinds=(ZSTD, LZMA2)):
        """Grow both slots' device buffers to a full batch of each kind before
        latency-sensitive traffic: two max-size requests per kind, back to
        back, because the worker alternates slots on every batch.  The device
        buffers are sized from byte and window counts, not from the content, so
        zero bytes do (with small host outputs: zero windows give one sequence,
        or one tiny frame, each)."""
        n = self.max_batch_bytes
        nb = num_windows(n)
        data = np.zeros(n, np.uint8)
        for kind in kinds:
            for _ in range(2):
                if kind == ZSTD:
                    r = self.submit(kind, data, out_a=np.empty((4 * nb, 4), np.uint32), cap=4 * nb)
                elif kind == ZSTD_FRAMES:
                    r = self.submit(kind, data, out_a=np.empty(64 * nb, np.uint8), cap=64 * nb)
                else:
                    r = self.submit(kind, data, packed=False)
                self.wait(r)

    def submit(self, kind, data, depth=None, **outputs):
        depth = (32 if kind == LZMA2 else 16) if depth is None else depth
        r = Request(kind, data, depth, **outputs)
        rid = ctypes.c_uint64()
        rc = L.gcz_server_submit(self._h, kind, depth, r.data.ctypes.data if r.data.size else None, r.data.size,
                                 r.out_a.ctypes.data if r.out_a is not None else None, r.cap,
                                 r.out_b.ctypes.data, ctypes.byref(rid))
        if rc != 0:
            raise GczError(rc, "gcz_server_submit failed")
        r.id = rid.value
        return r

    def wait(self, r, timeout_s=600.0):
        lat = ctypes.c_double()
        rc = L.gcz_server_wait(self._h, r.id, float(timeout_s), ctypes.byref(lat))
        if rc != 0:
            raise GczError(rc, f"request {r.id} failed")
        r.latency_ms = lat.value
        return r.result()

    def stats(self):
        c, b, nb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        p50, p99 = ctypes.c_double(), ctypes.c_double()
        rc = L.gcz_server_stats(self._h, ctypes.byref(c), ctypes.byref(b), ctypes.byref(nb), ctypes.byref(p50),
                                ctypes.byref(p99))
        return {"completed": c.value, "bytes": b.value, "batches": nb.value, "p50_ms": p50.value,
                "p99_ms": p99.value, "status": rc}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gcz_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
