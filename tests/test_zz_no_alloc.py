"""gcz_zstd_match_find_device_noalloc: the Zstd match-find step for callers
that cannot allocate device memory when they call in (their device memory is
owned by another allocator's reserved pool, or cudaMalloc / cudaFree would
stall a latency-bound loop, or they cannot hold a gcz_ctx because gcz_create
allocates).  Its scratch is a static device array in the library, shared by
every call, so the test checks that two calls in a row -- a full 8 MiB input,
then a smaller ragged one over the leftovers of the first -- each give exactly
the sequences and offsets of the allocating entry point
gcz_zstd_match_find_device (integer output: the tolerance is zero).

This file is named to be collected last.  It creates its own context and
buffers, so it also passes when run alone in a fresh process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stream_handle(torch):
    return torch.cuda.current_stream().cuda_stream  # 0 = default stream = NULL for the C ABI


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch
    import gcz

    torch.cuda.set_device(0)
    ctx = gcz.Context(0)
    st = _stream_handle(torch)
    for call, (seed, n) in enumerate(((41, gcz._lib.NOALLOC_MAX_INPUT), (42, 3 * 65536 + 4321))):
        data = gcz.gen_synthetic(seed, n, 8 << 20)
        d_in = torch.from_numpy(data).cuda()
        B = gcz.num_windows(n)
        cap = int(gcz.L.gcz_zstd_max_sequences(n))

        want_seqs = torch.zeros((cap, 4), dtype=torch.int32, device="cuda")
        want_off = torch.zeros(B + 1, dtype=torch.int64, device="cuda")
        ctx.zstd_match_find_device(d_in.data_ptr(), n, 16, want_seqs.data_ptr(), cap, want_off.data_ptr(), st)
        ctx.sync(st)

        got_seqs = torch.full((cap, 4), -1, dtype=torch.int32, device="cuda")
        got_off = torch.full((B + 1,), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = gcz.L.gcz_zstd_match_find_device_noalloc(0, d_in.data_ptr(), n, 16, got_seqs.data_ptr(), cap,
                                                      got_off.data_ptr(), st or None)
        assert rc == gcz._lib.GCZ_OK
        if call == 1:  # after the first call has set the device up, a call takes no device memory
            assert free_before - torch.cuda.mem_get_info()[0] < (2 << 20)

        w_off = want_off.cpu().numpy()
        np.testing.assert_array_equal(got_off.cpu().numpy(), w_off)
        total = int(w_off[-1])
        assert total > 0
        np.testing.assert_array_equal(got_seqs[:total].cpu().numpy(), want_seqs[:total].cpu().numpy())
        if call == 1:  # and, directly, the oracle (the CPU restatement pinned to the reference kernels)
            from oracle import oracle as orc

            o_seqs, o_off = orc.zstd_sequences(data, 16)
            np.testing.assert_array_equal(got_off.cpu().numpy().astype(np.uint64), o_off)
            np.testing.assert_array_equal(got_seqs[:total].cpu().numpy().view(np.uint32), o_seqs)
        del want_seqs, got_seqs
    ctx.close()


@pytest.mark.parametrize("depth", [1, 16], ids=["greedy", "lazy"])
@pytest.mark.parametrize("n", [1, 7, 15, 65536, 65536 + 17], ids=["1B", "7B", "15B", "one-window", "window+17"])
def test_noalloc_matches_allocating_entry_point_small_and_greedy(depth, n):
    """Inputs shorter than one 16-byte bulk copy (read with plain loads),
    exactly one window and one window plus a ragged tail, each with the greedy
    parse (depth 1) and the lazy one (depth 16)."""
    import torch
    import gcz

    torch.cuda.set_device(0)
    ctx = gcz.Context(0)
    st = _stream_handle(torch)
    data = gcz.gen_synthetic(50 + n, n, 8 << 20)
    d_in = torch.from_numpy(data).cuda()
    B = gcz.num_windows(n)
    cap = max(int(gcz.L.gcz_zstd_max_sequences(n)), 1)
    want_seqs = torch.zeros((cap, 4), dtype=torch.int32, device="cuda")
    want_off = torch.zeros(B + 1, dtype=torch.int64, device="cuda")
    ctx.zstd_match_find_device(d_in.data_ptr(), n, depth, want_seqs.data_ptr(), cap, want_off.data_ptr(), st)
    ctx.sync(st)
    got_seqs = torch.full((cap, 4), -1, dtype=torch.int32, device="cuda")
    got_off = torch.full((B + 1,), -1, dtype=torch.int64, device="cuda")
    rc = gcz.L.gcz_zstd_match_find_device_noalloc(0, d_in.data_ptr(), n, depth, got_seqs.data_ptr(), cap,
                                                  got_off.data_ptr(), st or None)
    assert rc == gcz._lib.GCZ_OK
    w_off = want_off.cpu().numpy()
    np.testing.assert_array_equal(got_off.cpu().numpy(), w_off)
    total = int(w_off[-1])
    np.testing.assert_array_equal(got_seqs[:total].cpu().numpy(), want_seqs[:total].cpu().numpy())
    ctx.close()


def test_noalloc_rejects_oversized_input_and_bad_arguments():
    import torch
    import gcz

    L = gcz.L
    buf = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    out = torch.zeros(4096, dtype=torch.int64, device="cuda")
    too_big = gcz._lib.NOALLOC_MAX_INPUT + 1
    assert L.gcz_zstd_match_find_device_noalloc(0, buf.data_ptr(), too_big, 16, out.data_ptr(), 10, out.data_ptr(),
                                                None) == gcz._lib.GCZ_ETOOLARGE
    assert L.gcz_zstd_match_find_device_noalloc(0, buf.data_ptr() + 1, 100, 16, out.data_ptr(), 10, out.data_ptr(),
                                                None) == gcz._lib.GCZ_EINVAL
    assert L.gcz_zstd_match_find_device_noalloc(-1, buf.data_ptr(), 100, 16, out.data_ptr(), 10, out.data_ptr(),
                                                None) == gcz._lib.GCZ_EINVAL


def test_noalloc_reports_small_output_capacity():
    import torch
    import gcz

    n = 1 << 20
    data = gcz.gen_synthetic(43, n, 8 << 20)
    d_in = torch.from_numpy(data).cuda()
    seqs = torch.zeros((8, 4), dtype=torch.int32, device="cuda")
    off = torch.zeros(gcz.num_windows(n) + 1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = gcz.L.gcz_zstd_match_find_device_noalloc(0, d_in.data_ptr(), n, 16, seqs.data_ptr(), 8, off.data_ptr(), None)
    assert rc == gcz._lib.GCZ_ECAPACITY
