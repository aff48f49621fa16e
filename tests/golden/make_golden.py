"""Generate tests/golden/reference_outputs.npz by running the REFERENCE's own
kernels (oracle/_ref: PTX compiled from its unmodified sources, JIT-loaded by
the driver) on a GPU, for every case in cases.py.

    make -C oracle ref            # in a checkout next to the reference sources
    python tests/golden/make_golden.py OUT.npz   # on a machine with a GPU

Stored per case: input sha256; Zstd seq_counts, lit_counts, the sequences
({ll, ml-3, off} triples, concatenated), sha256 of the literal bytes; LZMA2
counts and the packed (len<<16|dist) first slot, plus checks that the
reference never filled a second slot.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "gpu-compressor_b200"))
sys.path.insert(0, HERE)

import cases  # noqa: E402
from oracle.ref_kernels import RefKernels  # noqa: E402


def main(out_path):
    rk = RefKernels(0)
    store = {}
    meta = []
    for name, spec in cases.CASES:
        data = cases.build(spec)
        n = data.size
        W = spec["window"]
        seqs, lits, sc, lc = rk.zstd(data, spec["zdepth"], W, spec["max_seqs"])
        B = sc.size
        flat = np.concatenate([seqs[b, :sc[b]] for b in range(B)]) if B else np.zeros((0, 3), np.uint32)
        # literal bytes actually written: lit_counts[b] per window at stride W
        lit_bytes = b"".join(lits[b * W:b * W + lc[b]].tobytes() for b in range(B))
        m, c = rk.lzma(data, spec["lmax"], spec["ldepth"], W)
        assert int(c.max(initial=0)) <= 1, name
        extra = m[:, 1:, :] if m.shape[1] > 1 else np.zeros((0,), np.uint32)
        assert not np.any(extra), name
        packed = np.where(c[:n] > 0, (m[:n, 0, 1] << 16) | m[:n, 0, 0], 0).astype(np.uint32)
        assert not np.any(c[n:]), name
        store[f"{name}/zstd_seqs"] = flat.astype(np.uint32)
        store[f"{name}/zstd_seq_counts"] = sc.astype(np.uint32)
        store[f"{name}/zstd_lit_counts"] = lc.astype(np.uint32)
        store[f"{name}/lzma_packed"] = packed
        meta.append({"name": name, "spec": spec, "input_sha256": cases.sha(data),
                     "literals_sha256": cases.sha(np.frombuffer(lit_bytes, np.uint8)), "n": int(n)})
        print(f"{name:32s} n={n:7d} windows={B:4d} seqs={int(sc.sum()):6d} lzma_matches={int(c.sum()):7d}")
    store["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(out_path, **store)
    print("wrote", out_path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_outputs.npz"))
