"""Input cases for the golden fixtures and the parity tests.

Each case is (name, spec) where spec describes how to build the bytes
deterministically (numpy PCG64 or the gcz synthetic generator) and the kernel
parameters to run it with.  The fixtures store a sha256 of every input so a
change in how inputs are built is caught instead of silently comparing
different data.
"""
import hashlib

import numpy as np


def _periodic(period, n, seed):
    rng = np.random.default_rng(seed)
    pat = rng.integers(0, 256, size=period, dtype=np.uint8)
    return np.resize(pat, n).astype(np.uint8)


def _rep_dense(n, seed):
    """Copies at a handful of recurring offsets separated by 1-3 literal bytes,
    so that the repeat-offset path (zstd_compress.cu:259-275) fires often."""
    rng = np.random.default_rng(seed)
    out = bytearray(rng.integers(0, 256, size=64, dtype=np.uint8).tobytes())
    offs = [7, 19, 33, 64]
    while len(out) < n:
        for _ in range(int(rng.integers(1, 4))):
            out.append(int(rng.integers(0, 256)))
        off = offs[int(rng.integers(0, len(offs)))]
        ln = int(rng.integers(3, 24))
        for _ in range(ln):
            out.append(out[-off])
    return np.frombuffer(bytes(out[:n]), dtype=np.uint8).copy()


def _text_like(n, seed):
    rng = np.random.default_rng(seed)
    words = [bytes(rng.integers(97, 123, size=int(rng.integers(2, 9)), dtype=np.uint8)) for _ in range(300)]
    out = bytearray()
    while len(out) < n:
        out += words[int(rng.zipf(1.3)) % len(words)] + b" "
    return np.frombuffer(bytes(out[:n]), dtype=np.uint8).copy()


def build(spec):
    kind = spec["kind"]
    n = spec["n"]
    seed = spec.get("seed", 0)
    if kind == "zeros":
        return np.zeros(n, np.uint8)
    if kind == "const":
        return np.full(n, spec.get("byte", 0x41), np.uint8)
    if kind == "random":
        return np.random.default_rng(seed).integers(0, 256, size=n, dtype=np.uint8)
    if kind == "periodic":
        return _periodic(spec["period"], n, seed)
    if kind == "rep_dense":
        return _rep_dense(n, seed)
    if kind == "text":
        return _text_like(n, seed)
    if kind == "small_alpha":
        return np.random.default_rng(seed).integers(0, spec.get("alpha", 4), size=n, dtype=np.uint8)
    if kind == "synthetic":
        import gcz

        return gcz.gen_synthetic(seed, n, spec.get("max_offset", 8 << 20), tuple(spec.get("mix", (0.4, 0.4, 0.2))))
    raise ValueError(kind)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# (name, spec).  Kernel parameters: window (chunk / sub-block size), zstd
# search depth and max sequences, lzma max matches and search depth.
CASES = []


def _add(name, **spec):
    spec.setdefault("window", 65536)
    spec.setdefault("zdepth", 16)
    spec.setdefault("max_seqs", spec["window"] // 3)
    spec.setdefault("lmax", 8)
    spec.setdefault("ldepth", 32)
    CASES.append((name, spec))


for _n in range(0, 10):
    _add(f"zeros_{_n}", kind="zeros", n=_n)
    _add(f"random_{_n}", kind="random", n=_n, seed=100 + _n)
_add("const_5", kind="const", n=5, byte=7)
_add("zeros_win_plus_17", kind="zeros", n=65536 + 17)
_add("random_win_minus_1", kind="random", n=65535, seed=1)
_add("random_win_plus_1", kind="random", n=65537, seed=2)
_add("text_40k", kind="text", n=40000, seed=3)
_add("small_alpha4_30k", kind="small_alpha", n=30000, seed=4, alpha=4)
_add("rep_dense_64k", kind="rep_dense", n=65536, seed=5)
_add("rep_dense_20k_greedy", kind="rep_dense", n=20000, seed=6, zdepth=1)
for _p in (1, 2, 3, 4, 5, 7, 8, 13, 31, 32, 33, 64, 100, 255, 256, 300):
    _add(f"periodic_{_p}", kind="periodic", n=3000, period=_p, seed=_p)
_add("synthetic_s1_160k", kind="synthetic", n=160000, seed=1)
_add("synthetic_s2_100k_w4096", kind="synthetic", n=100000, seed=2, window=4096)
_add("synthetic_s3_70k_copyheavy", kind="synthetic", n=70000, seed=3, mix=(0.1, 0.8, 0.1))
_add("text_30k_maxseqs_40", kind="text", n=30000, seed=7, max_seqs=40)
_add("text_30k_w1024", kind="text", n=30000, seed=8, window=1024)
_add("synthetic_s4_50k_ldepth0", kind="synthetic", n=50000, seed=4, ldepth=0)
_add("synthetic_s5_50k_lmax2", kind="synthetic", n=50000, seed=5, lmax=2)
