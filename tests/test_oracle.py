"""The CPU oracle (oracle/oracle.c) against the reference kernels' own outputs
(tests/golden/reference_outputs.npz, produced on a B200 by make_golden.py from
the reference's unmodified PTX), plus self-consistency checks."""
import numpy as np
import pytest

import cases
from oracle import oracle as orc
from helpers import decode_window, check_lzma_packed


def _golden_cases(golden):
    z, meta = golden
    return [(m, z) for m in meta]


def test_golden_covers_all_cases(golden):
    _, meta = golden
    assert [m["name"] for m in meta] == [n for n, _ in cases.CASES]


@pytest.mark.parametrize("name,spec", cases.CASES, ids=[n for n, _ in cases.CASES])
def test_oracle_zstd_matches_reference(golden, name, spec):
    z, meta = golden
    m = next(x for x in meta if x["name"] == name)
    data = cases.build(spec)
    assert cases.sha(data) == m["input_sha256"]
    W = spec["window"]
    seqs, lits, sc, lc = orc.zstd_ref_layout(data, spec["zdepth"], W, spec["max_seqs"], literals=True, threads=4)
    np.testing.assert_array_equal(sc, z[f"{name}/zstd_seq_counts"])
    np.testing.assert_array_equal(lc, z[f"{name}/zstd_lit_counts"])
    flat = np.concatenate([seqs[b, :sc[b]] for b in range(sc.size)]) if sc.size else np.zeros((0, 3), np.uint32)
    np.testing.assert_array_equal(flat.reshape(-1, 3), z[f"{name}/zstd_seqs"].reshape(-1, 3))
    lit_bytes = b"".join(lits[b * W:b * W + lc[b]].tobytes() for b in range(sc.size))
    assert cases.sha(np.frombuffer(lit_bytes, np.uint8)) == m["literals_sha256"]


@pytest.mark.parametrize("name,spec", cases.CASES, ids=[n for n, _ in cases.CASES])
def test_oracle_lzma_matches_reference(golden, name, spec):
    z, _ = golden
    data = cases.build(spec)
    packed = orc.lzma_packed(data, spec["ldepth"], spec["window"], threads=4)
    np.testing.assert_array_equal(packed, z[f"{name}/lzma_packed"])


def test_oracle_lzma_ref_layout_matches_packed():
    data = cases.build({"kind": "synthetic", "n": 70000, "seed": 9})
    m, c = orc.lzma_ref_layout(data, 8, 32)
    packed = orc.lzma_packed(data, 32)
    n = data.size
    assert not np.any(c[n:])
    assert not np.any(m[:, 1:, :])
    np.testing.assert_array_equal(np.where(c[:n] > 0, (m[:n, 0, 1] << 16) | m[:n, 0, 0], 0), packed)


@pytest.mark.parametrize("kind,seed", [("synthetic", 11), ("text", 12), ("rep_dense", 13), ("periodic", 14)])
def test_oracle_zstd_sequences_rebuild_input(kind, seed):
    spec = {"kind": kind, "n": 150000, "seed": seed, "period": 37}
    data = cases.build(spec)
    seqs, offsets = orc.zstd_sequences(data, 16)
    for b in range(offsets.size - 1):
        win = data[b * 65536:(b + 1) * 65536]
        s = seqs[int(offsets[b]):int(offsets[b + 1])]
        assert decode_window(win, s) == win.tobytes()


def test_oracle_lzma_matches_are_genuine():
    data = cases.build({"kind": "synthetic", "n": 140000, "seed": 21})
    check_lzma_packed(data, orc.lzma_packed(data, 32))


def test_oracle_thread_count_does_not_change_results():
    data = cases.build({"kind": "synthetic", "n": 300000, "seed": 22})
    a = orc.zstd_sequences(data, 16, threads=1)
    b = orc.zstd_sequences(data, 16, threads=7)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(orc.lzma_packed(data, threads=1), orc.lzma_packed(data, threads=5))


def test_oracle_depth_16_equals_64():
    """search_depth is only tested as > 1 (zstd_compress.cu:278): L1 == L2."""
    data = cases.build({"kind": "synthetic", "n": 200000, "seed": 23})
    a = orc.zstd_sequences(data, 16)
    b = orc.zstd_sequences(data, 64)
    np.testing.assert_array_equal(a[0], b[0])


def test_planted_mistake_is_caught():
    """A deliberately wrong oracle result (one sequence length changed) no
    longer rebuilds the input: the rebuild check has teeth."""
    data = cases.build({"kind": "text", "n": 20000, "seed": 24})
    seqs, offsets = orc.zstd_sequences(data, 16)
    bad = seqs.copy()
    k = int(np.argmax(bad[:, 2] > 4))
    bad[k, 2] += 1
    win = data[:65536]
    with pytest.raises(AssertionError):
        assert decode_window(win, bad[int(offsets[0]):int(offsets[1])]) == win.tobytes()


def test_oracle_generator_build_matches_the_package_generator():
    """oracle/_build/libgen.so (what the CPU baselines use, so that they never
    load the product library) gives the same bytes as gcz.gen_synthetic."""
    import gcz

    for seed, n, max_off in ((1, 1 << 20, 8 << 20), (3, 3 * 65536 + 5, 128 << 20), (7, 1, 8 << 20)):
        assert np.array_equal(orc.gen_synthetic(seed, n, max_off), gcz.gen_synthetic(seed, n, max_off))
