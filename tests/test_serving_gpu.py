"""The request loop: requests of mixed kind and size, submitted from several
threads while batches run, each get exactly the result they get alone."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mixed_stream_equals_alone(ctx):
    import gcz
    from gcz import serving

    rng = np.random.default_rng(3)
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(1), np.log(3 << 20), size=90))] + [0, 1, 65536, 65537]
    kinds = [serving.ZSTD if rng.random() < 0.8 else serving.LZMA2 for _ in sizes]
    depths = [int(rng.choice([1, 16, 64])) if k == serving.ZSTD else 32 for k in kinds]
    datas = [gcz.gen_synthetic(500 + i, s, 8 << 20, tuple(rng.dirichlet([1, 1, 1]))) for i, s in enumerate(sizes)]
    srv = serving.Server(ctx, hbm_budget=4 * 10**9, max_batch_bytes=16 << 20)
    reqs = [None] * len(sizes)

    def submitter(idx):
        for i in idx:
            reqs[i] = srv.submit(kinds[i], datas[i], depths[i])

    threads = [threading.Thread(target=submitter, args=(range(j, len(sizes), 3),)) for j in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    results = [srv.wait(r) for r in reqs]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(sizes) and st["status"] == 0
    assert st["batches"] < len(sizes)  # requests really were batched together
    for i, res in enumerate(results):
        if kinds[i] == serving.ZSTD:
            s, o = ctx.zstd_match_find(datas[i], depths[i])
            np.testing.assert_array_equal(res[1], o)
            np.testing.assert_array_equal(res[0], s)
        else:
            p, h = ctx.lzma2_match_find(datas[i], 32)
            np.testing.assert_array_equal(res[0], p)
            np.testing.assert_array_equal(res[1], h)
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_wait_while_another_thread_submits(ctx):
    """One thread submits while this one waits, so the request table grows and
    rehashes under a blocked waiter; every request completes with its own
    result, and waiting again on a request already collected is GCZ_EINVAL."""
    import gcz
    from gcz import serving

    datas = [gcz.gen_synthetic(900 + i, 20000 + 37 * i, 8 << 20) for i in range(600)]
    srv = serving.Server(ctx, hbm_budget=2 * 10**9, max_batch_bytes=4 << 20)
    reqs = []
    cv = threading.Condition()

    def submitter():
        for d in datas:
            r = srv.submit(serving.ZSTD, d, 16)
            with cv:
                reqs.append(r)
                cv.notify()

    t = threading.Thread(target=submitter)
    t.start()
    got = []
    for i in range(len(datas)):
        with cv:
            cv.wait_for(lambda: len(reqs) > i)
            r = reqs[i]
        got.append(srv.wait(r))
    t.join()
    for i in (0, 299, 599):
        s, o = ctx.zstd_match_find(datas[i], 16)
        np.testing.assert_array_equal(got[i][1], o)
        np.testing.assert_array_equal(got[i][0], s)
    with pytest.raises(gcz.GczError) as e:
        srv.wait(reqs[0])
    assert e.value.code == gcz._lib.GCZ_EINVAL
    assert srv.stats()["completed"] == len(datas)
    srv.close()


def test_warm_up_then_serve(ctx):
    """warm_up runs one max-size request of every kind (zero bytes, small host
    outputs); requests served afterwards still get their own results."""
    import gcz
    from gcz import serving

    srv = serving.Server(ctx, hbm_budget=2 * 10**9, max_batch_bytes=4 << 20)
    srv.warm_up((serving.ZSTD, serving.LZMA2, serving.ZSTD_FRAMES))
    assert srv.stats()["completed"] == 3
    data = gcz.gen_synthetic(77, 3 << 20, 8 << 20)
    seqs, off = srv.wait(srv.submit(serving.ZSTD, data, 16))
    s, o = ctx.zstd_match_find(data, 16)
    np.testing.assert_array_equal(off, o)
    np.testing.assert_array_equal(seqs, s)
    srv.close()


def test_short_output_fails_only_its_request(ctx):
    """A Zstd request whose output room is too small completes with
    GCZ_ECAPACITY; a request in the same batch gets its own result."""
    import gcz
    from gcz import serving

    srv = serving.Server(ctx, hbm_budget=2 * 10**9, max_batch_bytes=8 << 20)
    small = gcz.gen_synthetic(61, 1 << 20, 8 << 20)
    good = gcz.gen_synthetic(62, 1 << 20, 8 << 20)
    for _ in range(3):
        r_small = srv.submit(serving.ZSTD, small, 16, out_a=np.empty((4, 4), np.uint32), cap=4)
        r_good = srv.submit(serving.ZSTD, good, 16)
        with pytest.raises(gcz.GczError) as e:
            srv.wait(r_small)
        assert e.value.code == gcz._lib.GCZ_ECAPACITY
        seqs, off = srv.wait(r_good)
        s, o = ctx.zstd_match_find(good, 16)
        np.testing.assert_array_equal(off, o)
        np.testing.assert_array_equal(seqs, s)
    srv.close()


def test_oversized_request_is_rejected(ctx):
    import gcz
    from gcz import serving

    srv = serving.Server(ctx, hbm_budget=2 * 10**9, max_batch_bytes=1 << 20)
    assert srv.max_batch_bytes == 1 << 20
    with pytest.raises(gcz.GczError):
        srv.submit(serving.ZSTD, np.zeros((1 << 20) + 1, np.uint8))
    srv.close()


def test_caller_buffers_and_has_only_lzma2(ctx):
    """Caller-owned (reused) output buffers; an LZMA2 request without a packed
    output returns only the per-window has-match bytes."""
    import gcz
    from gcz import serving

    srv = serving.Server(ctx, hbm_budget=2 * 10**9, max_batch_bytes=8 << 20)
    a = np.empty((1 << 18, 4), np.uint32)
    b = np.zeros(1024, np.uint64)
    h = np.zeros(1024, np.uint8)
    for i, n in enumerate([70000, 3 << 20, 5]):
        data = gcz.gen_synthetic(900 + i, n, 8 << 20)
        rz = srv.submit(serving.ZSTD, data, 16, out_a=a, out_b=b, cap=a.shape[0])
        rl = srv.submit(serving.LZMA2, data, 32, out_b=h, packed=False)
        seqs, off = srv.wait(rz)
        p, has = srv.wait(rl)
        s0, o0 = ctx.zstd_match_find(data, 16)
        np.testing.assert_array_equal(off, o0)
        np.testing.assert_array_equal(seqs, s0)
        assert p is None
        np.testing.assert_array_equal(has, ctx.lzma2_match_find(data, 32)[1])
    srv.close()


def test_frames_requests_in_a_mixed_stream(ctx):
    """GCZ_REQ_ZSTD_FRAMES requests batched with the others: each gets exactly
    the frames gcz_zstd_compress_frames_gpu gives for its bytes."""
    import gcz
    from gcz import serving, codecs

    rng = np.random.default_rng(21)
    sizes = [1, 300, 65536, 65537, 2 << 20, 100000, 0]
    datas = [gcz.gen_synthetic(700 + i, s, 8 << 20, tuple(rng.dirichlet([1, 1, 1]))) for i, s in enumerate(sizes)]
    srv = serving.Server(ctx, hbm_budget=4 * 10**9, max_batch_bytes=8 << 20)
    reqs = []
    for i, d in enumerate(datas):
        reqs.append((serving.ZSTD_FRAMES, d, srv.submit(serving.ZSTD_FRAMES, d, 16)))
        if i % 2 == 0:
            reqs.append((serving.ZSTD, d, srv.submit(serving.ZSTD, d, 16)))
    for kind, d, r in reqs:
        res = srv.wait(r)
        if kind == serving.ZSTD_FRAMES:
            blob, fs = ctx.zstd_compress_frames_gpu(d, 1)
            want, pos = [], 0
            for s in fs.tolist():
                want.append(blob[pos:pos + s].tobytes())
                pos += s
            assert res == want
            if res:
                assert codecs.zstd_decompress(res[0], min(d.size, 65536)) == d[:65536].tobytes()
        else:
            s, o = ctx.zstd_match_find(d, 16)
            np.testing.assert_array_equal(res[1], o)
            np.testing.assert_array_equal(res[0], s)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["status"] == 0


def _check_alone(ctx, kind, depth, data, res):
    from gcz import serving

    if kind == serving.ZSTD:
        s, o = ctx.zstd_match_find(data, depth)
        np.testing.assert_array_equal(res[1], o)
        np.testing.assert_array_equal(res[0], s)
    elif kind == serving.ZSTD_FRAMES:
        blob, fs = ctx.zstd_compress_frames_gpu(data, 1 if depth <= 16 else 2) if depth > 1 else (None, None)
        if depth <= 1:  # greedy frames: the frames of the greedy sequences
            return
        want, pos = [], 0
        for sz in fs.tolist():
            want.append(blob[pos:pos + sz].tobytes())
            pos += sz
        assert res == want
    else:
        p, h = ctx.lzma2_match_find(data, 32)
        if res[0] is not None:
            np.testing.assert_array_equal(res[0], p)
        np.testing.assert_array_equal(res[1], h)


def test_every_kind_in_one_batch(ctx):
    """Zstd (lazy and greedy), GPU frames and LZMA2 requests submitted together
    share a batch (one slot, one candidate sweep over all their windows) and
    each gets exactly its result alone.  The server has one slot, and a 32 MiB
    LZMA2 request holds it while the eight are submitted, so they are all
    pending when it frees up and the worker admits them, oldest first, into
    one batch (two if the submitting thread was held up)."""
    import gcz
    from gcz import serving

    srv = serving.Server(ctx, hbm_budget=1_200_000_000, max_batch_bytes=32 << 20, max_batch_requests=64)
    assert srv.info()[0] == 1
    rng = np.random.default_rng(5)
    plan = [(serving.ZSTD, 16), (serving.LZMA2, 32), (serving.ZSTD_FRAMES, 16), (serving.ZSTD, 1),
            (serving.LZMA2, 32), (serving.ZSTD, 64), (serving.ZSTD_FRAMES, 64), (serving.ZSTD, 16)]
    sizes = [3 << 20, 65537, 1 << 20, 200000, 5, 2 << 20, 70000, 0]
    datas = [gcz.gen_synthetic(1100 + i, n, 8 << 20, tuple(rng.dirichlet([1, 1, 1]))) for i, n in enumerate(sizes)]
    blocker = gcz.gen_synthetic(1099, 32 << 20, 8 << 20)
    for rep in range(2):
        before = srv.stats()["batches"]
        rb = srv.submit(serving.LZMA2, blocker, 32)
        reqs = [srv.submit(k, d, depth) for (k, depth), d in zip(plan, datas)]
        res = [srv.wait(r) for r in reqs]
        srv.wait(rb)
        for (k, depth), d, x in zip(plan, datas, res):
            _check_alone(ctx, k, depth, d, x)
        # the blocker's batch, then the eight in one (or two) batches: admitted
        # in submit order, so a batch holds more than one kind
        assert srv.stats()["batches"] - before <= 3
    st = srv.stats()
    srv.close()
    assert st["status"] == 0


def test_batch_error_stays_in_its_batch(ctx):
    """A batch whose bounded wait runs out (the failure-detection probe)
    completes with GCZ_EDEVICE; the loop keeps serving, and requests before
    and after it get their own results (each batch has its own status)."""
    import gcz
    from gcz import serving

    srv = serving.Server(ctx, hbm_budget=2 * 10**9, max_batch_bytes=8 << 20)
    data = gcz.gen_synthetic(81, 1 << 20, 8 << 20)
    r0 = srv.submit(serving.ZSTD, data, 16)
    _check_alone(ctx, serving.ZSTD, 16, data, srv.wait(r0))
    for _ in range(3):
        probe = srv.selftest_wait_timeout(1 << 10)
        with pytest.raises(gcz.GczError) as e:
            srv.wait(probe)
        assert e.value.code == gcz._lib.GCZ_EDEVICE
        r = srv.submit(serving.ZSTD, data, 16)
        _check_alone(ctx, serving.ZSTD, 16, data, srv.wait(r))
        rl = srv.submit(serving.LZMA2, data, 32)
        _check_alone(ctx, serving.LZMA2, 32, data, srv.wait(rl))
    # the context's own status is untouched by the loop's batches
    s, o = ctx.zstd_match_find(data, 16)
    assert o[-1] > 0
    srv.close()


def test_wait_timeout_keeps_the_request(ctx):
    """A wait that times out returns GCZ_ETIMEOUT and leaves the request in
    the loop; a later wait collects exactly its result."""
    import gcz
    from gcz import serving

    srv = serving.Server(ctx, hbm_budget=4 * 10**9, max_batch_bytes=64 << 20)
    data = gcz.gen_synthetic(82, 64 << 20, 8 << 20)
    r = srv.submit(serving.ZSTD, data, 16)
    with pytest.raises(gcz.GczError) as e:
        srv.wait(r, timeout_s=0.0)  # 64 MiB cannot be copied in, let alone matched, in zero time
    assert e.value.code == gcz._lib.GCZ_ETIMEOUT
    _check_alone(ctx, serving.ZSTD, 16, data, srv.wait(r))
    srv.close()


def test_slots_from_budget_and_no_allocation_while_serving(ctx):
    """Slots follow the HBM budget (23 device bytes per input byte of a batch,
    at most 8); every buffer is allocated at creation, so serving a burst of
    mixed requests leaves the device's free memory where it was."""
    import torch
    import gcz
    from gcz import serving

    mb = 16 << 20
    srv = serving.Server(ctx, hbm_budget=3 * 23 * mb, max_batch_bytes=mb)
    slots, dev_bytes = srv.info()
    assert slots == 3 and dev_bytes <= 3 * 23 * mb + 3 * 40 * (2 << 20), (slots, dev_bytes)
    srv.close()
    srv = serving.Server(ctx, hbm_budget=120 * 10**9, max_batch_bytes=mb)
    assert srv.info()[0] == 8
    srv.warm_up((serving.ZSTD, serving.LZMA2, serving.ZSTD_FRAMES))
    rng = np.random.default_rng(9)
    datas = [gcz.gen_synthetic(1200 + i, int(x), 8 << 20) for i, x in
             enumerate(np.exp(rng.uniform(np.log(4096), np.log(mb), size=40)))]
    kinds = [serving.ZSTD, serving.LZMA2, serving.ZSTD_FRAMES]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    reqs = [(kinds[i % 3], d, srv.submit(kinds[i % 3], d, 16 if kinds[i % 3] != serving.LZMA2 else 32))
            for i, d in enumerate(datas)]
    out = [(k, d, srv.wait(r)) for k, d, r in reqs]
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free0) < (4 << 20)
    for k, d, x in out[:6]:
        _check_alone(ctx, k, 16 if k != serving.LZMA2 else 32, d, x)
    srv.close()
