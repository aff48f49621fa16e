"""Runs the reference's own match-finding kernels on the GPU.

TEST INFRASTRUCTURE ONLY.  _ref/*.ptx are compiled (make -C oracle ref) from
the reference's unmodified zstd_compress.cu / lzma2_match_find.cu with its own
flags (build.rs:59-95); the CUDA driver JIT-compiles them for the GPU at load,
exactly as cudarc's load_ptx does in the reference.  Launch shapes follow its
adapters: grid = windows, block = 256 (compress_zstd_custom.rs:91-111,
compress_lzma2_custom.rs:518-536).  Outputs are zero-initialised first, like
the reference's alloc_zeros.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ZSTD_PTX = os.path.join(REF_DIR, "zstd_compress.ptx")
LZMA_PTX = os.path.join(REF_DIR, "lzma2_match_find.ptx")
RUNNER = os.path.join(REF_DIR, "libref_runner.so")


def available():
    return all(os.path.exists(p) for p in (ZSTD_PTX, LZMA_PTX, RUNNER))


class RefKernels:
    def __init__(self, device=0):
        import torch

        self.torch = torch
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        torch.zeros(1, device=self.device)  # make the primary context current
        L = ctypes.CDLL(RUNNER)
        u32, u64 = ctypes.c_uint32, ctypes.c_uint64
        L.ref_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.ref_load.restype = ctypes.c_int
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_zstd_launch.argtypes = [u64, u64, u64, u64, u64, u32, u32, u32, u32, u32, u64]
        L.ref_zstd_launch.restype = ctypes.c_int
        L.ref_lzma_launch.argtypes = [u64, u64, u64, u32, u32, u32, u32, u32, u64]
        L.ref_lzma_launch.restype = ctypes.c_int
        if L.ref_load(ZSTD_PTX.encode(), LZMA_PTX.encode(), device) != 0:
            raise RuntimeError("reference kernels: " + L.ref_last_error().decode())
        self.L = L

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("reference kernels: " + self.L.ref_last_error().decode())

    def to_device(self, buf):
        t = self.torch
        a = np.ascontiguousarray(buf, dtype=np.uint8)
        d = t.empty(max(a.size, 1) + 64, dtype=t.uint8, device=self.device)
        if a.size:
            d[:a.size].copy_(t.from_numpy(a))
        return d

    def zstd_launch(self, d_in, n, bufs, search_depth=16, window=65536, max_seqs=None):
        """Launch on device buffers (bufs from zstd_alloc); returns nothing."""
        t = self.torch
        if max_seqs is None:
            max_seqs = window // 3
        B = (n + window - 1) // window
        seqs, lits, sc, lc = bufs
        st = t.cuda.current_stream(self.device).cuda_stream
        self._check(self.L.ref_zstd_launch(d_in.data_ptr(), seqs.data_ptr(), lits.data_ptr(), sc.data_ptr(),
                                           lc.data_ptr(), window, B, n, search_depth, max_seqs, st))

    def zstd_alloc(self, n, window=65536, max_seqs=None):
        t = self.torch
        if max_seqs is None:
            max_seqs = window // 3
        B = max((n + window - 1) // window, 1)
        return (t.zeros(B * max_seqs * 3, dtype=t.int32, device=self.device),
                t.zeros(B * window, dtype=t.uint8, device=self.device),
                t.zeros(B, dtype=t.int32, device=self.device),
                t.zeros(B, dtype=t.int32, device=self.device))

    def zstd(self, buf, search_depth=16, window=65536, max_seqs=None):
        """(sequences u32[B, max_seqs, 3], literals u8[B*window], seq_counts u32[B], lit_counts u32[B])."""
        t = self.torch
        n = int(np.asarray(buf).size)
        if max_seqs is None:
            max_seqs = window // 3
        B = (n + window - 1) // window
        d_in = self.to_device(buf)
        bufs = self.zstd_alloc(n, window, max_seqs)
        if B:
            self.zstd_launch(d_in, n, bufs, search_depth, window, max_seqs)
        t.cuda.synchronize(self.device)
        seqs, lits, sc, lc = (x.cpu().numpy().view(np.uint32) if x.dtype == t.int32 else x.cpu().numpy()
                              for x in bufs)
        return seqs.reshape(-1, max_seqs, 3)[:B], lits[:B * window], sc[:B], lc[:B]

    def lzma_alloc(self, n, window=65536, max_matches=8):
        t = self.torch
        B = max((n + window - 1) // window, 1)
        return (t.zeros(B * window * max_matches * 2, dtype=t.int32, device=self.device),
                t.zeros(B * window, dtype=t.int32, device=self.device))

    def lzma_launch(self, d_in, n, bufs, max_matches=8, search_depth=32, window=65536):
        t = self.torch
        B = (n + window - 1) // window
        m, c = bufs
        st = t.cuda.current_stream(self.device).cuda_stream
        self._check(self.L.ref_lzma_launch(d_in.data_ptr(), m.data_ptr(), c.data_ptr(), window, B, n, max_matches,
                                           search_depth, st))

    def lzma(self, buf, max_matches=8, search_depth=32, window=65536):
        """(matches u32[B*window, max_matches, 2], counts u32[B*window])."""
        t = self.torch
        n = int(np.asarray(buf).size)
        B = (n + window - 1) // window
        d_in = self.to_device(buf)
        bufs = self.lzma_alloc(n, window, max_matches)
        if B:
            self.lzma_launch(d_in, n, bufs, max_matches, search_depth, window)
        t.cuda.synchronize(self.device)
        m, c = (x.cpu().numpy().view(np.uint32) for x in bufs)
        return m.reshape(-1, max_matches, 2)[:B * window], c[:B * window]
