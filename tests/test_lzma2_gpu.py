"""LZMA2 match finder on the GPU vs the reference kernels (golden fixtures,
the reference PTX side by side) and vs the CPU oracle -- bit-exact."""
import numpy as np
import pytest

import cases
from oracle import oracle as orc
from helpers import check_lzma_packed

pytestmark = pytest.mark.gpu


def run_ref_layout(ctx, data, window, max_matches, depth):
    import torch as t

    n = data.size
    B = (n + window - 1) // window
    d_in = t.empty(max(n, 1) + 64, dtype=t.uint8, device="cuda")
    if n:
        d_in[:n].copy_(t.from_numpy(data))
    m = t.zeros(max(B, 1) * window * max_matches * 2, dtype=t.int32, device="cuda")
    c = t.full((max(B, 1) * window,), 7, dtype=t.int32, device="cuda")  # every count must be written
    st = t.cuda.current_stream().cuda_stream
    if B:
        ctx.lzma2_match_find_ref_layout_device(d_in.data_ptr(), m.data_ptr(), c.data_ptr(), window, B, n,
                                               max_matches, depth, st)
    ctx.sync(st)
    return (m.cpu().numpy().view(np.uint32).reshape(-1, max_matches, 2)[:B * window],
            c.cpu().numpy().view(np.uint32)[:B * window])


@pytest.mark.parametrize("algo,staged,threads", [(2, 1, 1024), (2, 1, 512), (2, 1, 256), (1, 1, 1024), (1, 0, 1024)],
                         ids=["split", "split-512", "split-256", "fused-staged", "fused-l1"])
@pytest.mark.parametrize("name,spec", cases.CASES, ids=[n for n, _ in cases.CASES])
def test_ref_layout_matches_reference_golden(ctx, golden, name, spec, algo, staged, threads):
    z, meta = golden
    data = cases.build(spec)
    n = data.size
    ctx.set_option("algo", algo)
    ctx.set_option("staged", staged)
    ctx.set_option("lzma_threads", threads)
    try:
        m, c = run_ref_layout(ctx, data, spec["window"], spec["lmax"], spec["ldepth"])
    finally:
        ctx.set_option("algo", 2)
        ctx.set_option("staged", 1)
        ctx.set_option("lzma_threads", 1024)
    assert int(c.max(initial=0)) <= 1
    assert not np.any(c[n:])
    assert not np.any(m[:, 1:, :])
    packed = np.where(c[:n] > 0, (m[:n, 0, 1] << 16) | m[:n, 0, 0], 0).astype(np.uint32)
    np.testing.assert_array_equal(packed, z[f"{name}/lzma_packed"])
    # slots of positions without a match are left untouched (zero here)
    assert not np.any(m[:n][c[:n] == 0])


@pytest.mark.parametrize("name,spec", [c for c in cases.CASES if c[1]["window"] == 65536],
                         ids=[n for n, s in cases.CASES if s["window"] == 65536])
def test_packed_host_api_matches_oracle(ctx, name, spec):
    data = cases.build(spec)
    packed, has = ctx.lzma2_match_find(data, spec["ldepth"])
    o = orc.lzma_packed(data, spec["ldepth"])
    np.testing.assert_array_equal(packed, o)
    np.testing.assert_array_equal(has, orc.has_matches(o, data.size))


def test_gpu_find_matches_layout(ctx):
    """GpuMatchData arrays (compress_lzma2_custom.rs:539-549) equal the oracle's
    reference layout, de-interleaved and zero-filled."""
    import gcz

    data = gcz.gen_synthetic(7, 300000, 128 << 20)
    md = gcz.gpu_find_matches(data, 0)
    m, c = orc.lzma_ref_layout(data, 8, 32)
    np.testing.assert_array_equal(md.match_counts, c)
    np.testing.assert_array_equal(md.match_distances.reshape(-1, 8), m[:, :, 0])
    np.testing.assert_array_equal(md.match_lengths.reshape(-1, 8), m[:, :, 1])
    assert md.num_sub_blocks == gcz.num_windows(data.size) and md.sub_block_size == 65536 and md.max_matches == 8


def test_against_reference_ptx(ctx):
    from oracle import ref_kernels

    if not ref_kernels.available():
        pytest.skip("oracle/_ref not built")
    import gcz

    rk = ref_kernels.RefKernels(0)
    data = gcz.gen_synthetic(3, 8 << 20, 128 << 20)
    rm, rc = rk.lzma(data, 8, 32)
    gm, gc = run_ref_layout(ctx, data, 65536, 8, 32)
    np.testing.assert_array_equal(gc, rc)
    np.testing.assert_array_equal(gm, rm)


def test_against_reference_ptx_one_pipeline_chunk(ctx):
    """One reference LZMA2 pipeline chunk (128 MiB, --dict-size 128,
    pipeline_lzma2.rs:116-190): the reference kernel's 8.5 GiB of slots and
    counts are reduced on the GPU to the per-position form (first slot,
    len << 16 | dist, 0 when the count is 0; the reference records at most one
    match per position) and compared with this library's packed matches
    there, so nothing large crosses PCIe."""
    from oracle import ref_kernels

    if not ref_kernels.available():
        pytest.skip("oracle/_ref not built")
    import torch as t
    import gcz

    n = 128 << 20
    data = gcz.gen_synthetic(3, n, 128 << 20)
    rk = ref_kernels.RefKernels(0)
    d_in = rk.to_device(data)
    bufs = rk.lzma_alloc(n)
    rk.lzma_launch(d_in, n, bufs)
    t.cuda.synchronize()
    m, c = bufs
    counts = c[:n]
    assert int(counts.max().item()) <= 1
    slots = m.view(-1, 8, 2)[:n, 0, :]
    ref_packed = t.where(counts > 0, (slots[:, 1] << 16) | slots[:, 0], t.zeros_like(counts))
    del bufs, m, slots
    t.cuda.empty_cache()
    B = gcz.num_windows(n)
    d_packed = t.empty(n, dtype=t.int32, device="cuda")
    d_has = t.empty(B, dtype=t.uint8, device="cuda")
    st = t.cuda.current_stream().cuda_stream
    ctx.lzma2_match_find_device(d_in.data_ptr(), n, 32, d_packed.data_ptr(), d_has.data_ptr(), st)
    ctx.sync(st)
    assert t.equal(d_packed, ref_packed)
    ref_has = (counts.view(B, 65536) > 0).any(dim=1).to(t.uint8)
    assert t.equal(d_has, ref_has)


def test_full_size_1gib_vs_oracle(ctx):
    """LZMA2 L1 workload (1 GiB, seed 3, copy offsets to 128 MiB)."""
    import torch as t
    import gcz

    n = 1 << 30
    data = gcz.gen_synthetic(3, n, 128 << 20)
    d_in = t.from_numpy(data).cuda()
    B = gcz.num_windows(n)
    d_packed = t.empty(n, dtype=t.int32, device="cuda")
    d_has = t.empty(B, dtype=t.uint8, device="cuda")
    st = t.cuda.current_stream().cuda_stream
    ctx.lzma2_match_find_device(d_in.data_ptr(), n, 32, d_packed.data_ptr(), d_has.data_ptr(), st)
    ctx.sync(st)
    packed = d_packed.cpu().numpy().view(np.uint32)
    o = orc.lzma_packed(data, 32, threads=32)
    np.testing.assert_array_equal(packed, o)
    np.testing.assert_array_equal(d_has.cpu().numpy(), orc.has_matches(o, n))
    rng = np.random.default_rng(1)
    lo = int(rng.integers(0, n - 200000))
    check_lzma_packed(data[lo - lo % 65536:lo - lo % 65536 + 131072], packed[lo - lo % 65536:lo - lo % 65536 + 131072])


def test_triage_returns_has_matches_only(ctx):
    """packed == NULL: only the per-window has-match bytes come back, equal to
    the full call's (and to the oracle's) on windows with and without matches."""
    import gcz

    data = np.concatenate([gcz.gen_synthetic(81, 5 * 65536 + 9, 128 << 20),
                           np.arange(65536, dtype=np.uint32).view(np.uint8)[:65536],
                           np.zeros(3, np.uint8)])
    has = ctx.lzma2_triage(data)
    p, h = ctx.lzma2_match_find(data)
    np.testing.assert_array_equal(has, h)
    np.testing.assert_array_equal(has, orc.has_matches(orc.lzma_packed(data, 32), data.size))
