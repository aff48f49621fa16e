"""Python front end of the libgcz request loop (gcz_server_* in include/gcz.h)."""
import ctypes
import threading

import numpy as np

from . import L, GczError, num_windows, _u8
from ._lib import GCZ_ETIMEOUT

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
        self._live = {}  # id -> Request until a wait collects it: its buffers are in use until then
        self.ctx = ctx
        self._lib = L  # kept for close() during interpreter shutdown

    @property
    def max_batch_bytes(self):
        return int(L.gcz_server_max_batch_bytes(self._h))

    def info(self):
        """(slots, device bytes held): every slot's buffers are allocated at creation."""
        slots, dev = ctypes.c_uint32(), ctypes.c_uint64()
        rc = L.gcz_server_info(self._h, ctypes.byref(slots), ctypes.byref(dev))
        if rc != 0:
            raise GczError(rc, "gcz_server_info failed")
        return slots.value, dev.value

    def warm_up(self, kinds=(ZSTD, LZMA2)):
        """One max-size request of each kind, so that the first requests that
        matter do not pay for first-launch costs (module loading, shared-memory
        carve-out).  Device buffers are allocated at creation already.  The
        buffers are sized from byte and window counts, not from the content, so
        zero bytes do (with small host outputs: zero windows give one sequence,
        or one tiny frame, each)."""
        n = self.max_batch_bytes
        nb = num_windows(n)
        data = np.zeros(n, np.uint8)
        for kind in kinds:
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
        with self._lock:
            self._live[r.id] = r
        return r

    def selftest_wait_timeout(self, max_iterations=1 << 12):
        """Submit a failure-detection probe (gcz_server_selftest_wait_timeout):
        its batch's bounded wait runs out and the batch reports GCZ_EDEVICE."""
        r = Request(LZMA2, np.zeros(0, np.uint8), 32, packed=False)
        rid = ctypes.c_uint64()
        rc = L.gcz_server_selftest_wait_timeout(self._h, int(max_iterations), ctypes.byref(rid))
        if rc != 0:
            raise GczError(rc, "gcz_server_selftest_wait_timeout failed")
        r.id = rid.value
        with self._lock:
            self._live[r.id] = r
        return r

    def wait(self, r, timeout_s=600.0):
        """The request's result.  GczError with code GCZ_ETIMEOUT when timeout_s
        passed first: the request stays in the loop, and the server keeps its
        buffers alive until a later wait collects it."""
        lat = ctypes.c_double()
        rc = L.gcz_server_wait(self._h, r.id, float(timeout_s), ctypes.byref(lat))
        if rc != GCZ_ETIMEOUT:
            with self._lock:
                self._live.pop(r.id, None)
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
            self._lib.gcz_server_destroy(self._h)  # finishes every submitted request first
            self._h = None
            self._live = {}

    def __del__(self):
        self.close()
