"""Zstd match finder on the GPU vs the reference kernels (golden fixtures and,
when oracle/_ref is present, the reference PTX run side by side) and vs the
CPU oracle -- bit-exact."""
import numpy as np
import pytest

import cases
from oracle import oracle as orc
from helpers import decode_window

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def run_ref_layout(ctx, data, window, depth, max_seqs):
    """gcz_zstd_match_find_ref_layout_device on torch buffers; numpy results."""
    t = _torch()
    n = data.size
    B = (n + window - 1) // window
    d_in = t.empty(max(n, 1) + 64, dtype=t.uint8, device="cuda")
    if n:
        d_in[:n].copy_(t.from_numpy(data))
    seqs = t.zeros(max(B, 1) * max_seqs * 3, dtype=t.int32, device="cuda")
    lits = t.zeros(max(B, 1) * window, dtype=t.uint8, device="cuda")
    sc = t.zeros(max(B, 1), dtype=t.int32, device="cuda")
    lc = t.zeros(max(B, 1), dtype=t.int32, device="cuda")
    if B:
        ctx.zstd_match_find_ref_layout_device(d_in.data_ptr(), seqs.data_ptr(), lits.data_ptr(), sc.data_ptr(),
                                              lc.data_ptr(), window, B, n, depth, max_seqs,
                                              t.cuda.current_stream().cuda_stream)
    ctx.sync(t.cuda.current_stream().cuda_stream)
    t.cuda.synchronize()
    return (seqs.cpu().numpy().view(np.uint32).reshape(-1, max_seqs, 3)[:B], lits.cpu().numpy()[:B * window],
            sc.cpu().numpy().view(np.uint32)[:B], lc.cpu().numpy().view(np.uint32)[:B])


@pytest.mark.parametrize("algo,staged,seg", [(2, 1, 4096), (2, 1, 1024), (2, 1, 512), (2, 1, 2048), (2, 1, 8192),
                                             (1, 1, 4096), (1, 0, 4096)],
                         ids=["split", "split-group1k", "split-group512", "split-seg2k", "split-seg8k", "fused-staged",
                              "fused-l1"])
@pytest.mark.parametrize("name,spec", cases.CASES, ids=[n for n, _ in cases.CASES])
def test_ref_layout_matches_reference_golden(ctx, golden, name, spec, algo, staged, seg):
    z, meta = golden
    m = next(x for x in meta if x["name"] == name)
    data = cases.build(spec)
    assert cases.sha(data) == m["input_sha256"]
    W = spec["window"]
    ctx.set_option("algo", algo)
    ctx.set_option("staged", staged)
    ctx.set_option("parse_seg", seg)
    try:
        seqs, lits, sc, lc = run_ref_layout(ctx, data, W, spec["zdepth"], spec["max_seqs"])
    finally:
        ctx.set_option("algo", 2)
        ctx.set_option("staged", 1)
        ctx.set_option("parse_seg", 1024)
    np.testing.assert_array_equal(sc, z[f"{name}/zstd_seq_counts"])
    np.testing.assert_array_equal(lc, z[f"{name}/zstd_lit_counts"])
    flat = np.concatenate([seqs[b, :sc[b]] for b in range(sc.size)]) if sc.size else np.zeros((0, 3), np.uint32)
    np.testing.assert_array_equal(flat.reshape(-1, 3), z[f"{name}/zstd_seqs"].reshape(-1, 3))
    lit_bytes = b"".join(lits[b * W:b * W + lc[b]].tobytes() for b in range(sc.size))
    assert cases.sha(np.frombuffer(lit_bytes, np.uint8)) == m["literals_sha256"]


@pytest.mark.parametrize("name,spec", [c for c in cases.CASES if c[1]["window"] == 65536 and c[1]["max_seqs"] == 21845],
                         ids=[n for n, s in cases.CASES if s["window"] == 65536 and s["max_seqs"] == 21845])
def test_compact_host_api_matches_oracle(ctx, name, spec):
    data = cases.build(spec)
    seqs, offsets = ctx.zstd_match_find(data, spec["zdepth"])
    o_seqs, o_off = orc.zstd_sequences(data, spec["zdepth"])
    np.testing.assert_array_equal(offsets, o_off)
    np.testing.assert_array_equal(seqs, o_seqs)


@pytest.mark.parametrize("algo,seg,sweep,pf", [(2, 4096, 0, 4), (2, 1024, 0, 4), (2, 512, 0, 4), (2, 1024, 0, 0),
                                                (2, 1024, 0, 8), (2, 1024, 1, 4), (2, 1024, 1, 0), (2, 1024, 2, 0),
                                                (2, 1024, 3, 0), (1, 4096, 0, 4)],
                         ids=["split", "split-group1k", "split-group512", "sweep-no-prefetch", "sweep-prefetch8",
                              "sweep-ballots", "sweep-ballots-no-prefetch", "sweep-ahead", "sweep-ahead-ballots",
                              "fused"])
@pytest.mark.parametrize("seed,n,mix", [(1, 16 << 20, (0.4, 0.4, 0.2)), (31, 5 << 20, (0.05, 0.9, 0.05)),
                                        (32, 3 << 20 | 12345, (0.9, 0.05, 0.05)), (33, 2 << 20, (0.0, 0.0, 1.0)),
                                        (34, 2 << 20, (0.0, 1.0, 0.0))])
def test_synthetic_vs_oracle(ctx, seed, n, mix, algo, seg, sweep, pf):
    """Zstd L1 plain workload shape (16 MiB, seed 1) and skewed mixes, over the
    kernel families, segment layouts, sweep groupings and sweep prefetch
    distances."""
    import gcz

    data = gcz.gen_synthetic(seed, n, 8 << 20, mix)
    ctx.set_option("algo", algo)
    ctx.set_option("parse_seg", seg)
    ctx.set_option("sweep_groups", sweep)
    ctx.set_option("sweep_prefetch", pf)
    try:
        seqs, offsets = ctx.zstd_match_find(data, 16)
    finally:
        ctx.set_option("algo", 2)
        ctx.set_option("parse_seg", 1024)
        ctx.set_option("sweep_groups", 0)
        ctx.set_option("sweep_prefetch", 4)
    o_seqs, o_off = orc.zstd_sequences(data, 16, threads=16)
    np.testing.assert_array_equal(offsets, o_off)
    np.testing.assert_array_equal(seqs, o_seqs)


def test_against_reference_ptx_16mib(ctx):
    """Reference kernels run on the same GPU on the 16 MiB Zstd L1 input: equal outputs."""
    from oracle import ref_kernels

    if not ref_kernels.available():
        pytest.skip("oracle/_ref not built")
    import gcz

    rk = ref_kernels.RefKernels(0)
    data = gcz.gen_synthetic(1, 16 << 20, 8 << 20)
    r_seqs, r_lits, r_sc, r_lc = rk.zstd(data, 16)
    g_seqs, g_lits, g_sc, g_lc = run_ref_layout(ctx, data, 65536, 16, 21845)
    np.testing.assert_array_equal(g_sc, r_sc)
    np.testing.assert_array_equal(g_lc, r_lc)
    for b in range(r_sc.size):
        np.testing.assert_array_equal(g_seqs[b, :r_sc[b]], r_seqs[b, :r_sc[b]])
        np.testing.assert_array_equal(g_lits[b * 65536:b * 65536 + r_lc[b]], r_lits[b * 65536:b * 65536 + r_lc[b]])


def test_device_api_full_size_1gib(ctx):
    """Zstd L2 batched workload (1 GiB, seed 2, depth 64) through the device
    entry point: equal to the multithreaded oracle; sampled windows rebuild."""
    t = _torch()
    import gcz

    n = 1 << 30
    data = gcz.gen_synthetic(2, n, 8 << 20)
    d_in = t.from_numpy(data).cuda()
    B = gcz.num_windows(n)
    cap = int(gcz.L.gcz_zstd_max_sequences(n))
    d_seqs = t.empty((cap, 4), dtype=t.int32, device="cuda")
    d_off = t.empty(B + 1, dtype=t.int64, device="cuda")
    st = t.cuda.current_stream().cuda_stream
    ctx.zstd_match_find_device(d_in.data_ptr(), n, 64, d_seqs.data_ptr(), cap, d_off.data_ptr(), st)
    ctx.sync(st)
    off = d_off.cpu().numpy().view(np.uint64)
    total = int(off[-1])
    seqs = d_seqs[:total].cpu().numpy().view(np.uint32)
    del d_seqs
    o_seqs, o_off = orc.zstd_sequences(data, 64, threads=32)
    np.testing.assert_array_equal(off, o_off)
    np.testing.assert_array_equal(seqs, o_seqs)
    rng = np.random.default_rng(0)
    for b in rng.choice(B, 8, replace=False):
        win = data[b * 65536:(b + 1) * 65536]
        assert decode_window(win, seqs[int(off[b]):int(off[b + 1])]) == win.tobytes()


def test_capacity_error_is_reported(ctx):
    import gcz

    data = gcz.gen_synthetic(5, 1 << 20, 8 << 20)
    seqs = np.empty((10, 4), np.uint32)
    offsets = np.zeros(17, np.uint64)
    rc = gcz.L.gcz_zstd_match_find(ctx.handle, data.ctypes.data, data.size, 16, seqs.ctypes.data, 10,
                                   offsets.ctypes.data)
    assert rc == gcz._lib.GCZ_ECAPACITY


def test_invalid_arguments(ctx):
    import gcz

    t = _torch()
    buf = t.zeros(1024, dtype=t.uint8, device="cuda")
    out = t.zeros(4096, dtype=t.int32, device="cuda")
    # misaligned device input
    rc = gcz.L.gcz_zstd_match_find_ref_layout_device(ctx.handle, buf.data_ptr() + 1, out.data_ptr(), None,
                                                     out.data_ptr(), None, 65536, 1, 100, 16, 100, None)
    assert rc == gcz._lib.GCZ_EINVAL
    # window not a multiple of 16 / too large
    for w in (1000, 65552, 0):
        rc = gcz.L.gcz_zstd_match_find_ref_layout_device(ctx.handle, buf.data_ptr(), out.data_ptr(), None,
                                                         out.data_ptr(), None, w, 1, 100, 16, 100, None)
        assert rc == gcz._lib.GCZ_EINVAL


def test_loaded_kernel_image_is_sm100(ctx):
    """The kernels the runtime loaded from libgcz.so were compiled for sm_100a
    (binaryVersion 100 from cudaFuncGetAttributes), not JIT-compiled from PTX."""
    assert ctx.query("binary_version") == 100


def test_packed_records_expand_to_the_sequences(ctx):
    """gcz_zstd_match_find_packed's 8-byte records expand (caller-side) to
    exactly gcz_zstd_match_find's ZSTD_Sequence records, with the same window
    offsets, across the host pipeline's slices."""
    import gcz

    for seed, n in ((61, 5 * 65536 + 77), (62, 70 << 20)):
        data = gcz.gen_synthetic(seed, n, 8 << 20)
        s, o = ctx.zstd_match_find(data, 64)
        r, o2 = ctx.zstd_match_find_packed(data, 64)
        np.testing.assert_array_equal(o2, o)
        np.testing.assert_array_equal(gcz.expand_packed(r), s)
