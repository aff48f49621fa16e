"""Several ranks, each owning a contiguous window range (gcz.shards): the
partition, the host-side gather and the timing reductions, run as two and
three `gloo` ranks on the CPU.  The per-rank match finder is the oracle here
(the GPU one is covered by the gpu tests); the gathered result of the ranks
must equal one oracle pass over the whole input."""
import datetime
import multiprocessing as mp
import socket
import traceback

import numpy as np
import pytest

import cases


def test_window_range_partitions_exactly():
    from gcz import shards

    for nb in [0, 1, 2, 3, 7, 16, 17, 1000, 16385]:
        for world in [1, 2, 3, 4, 8]:
            ranges = [shards.window_range(nb, world, r) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == nb
            for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
                assert a1 == b0
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        shards.window_range(4, 2, 2)


def test_byte_range_is_window_aligned():
    from gcz import shards

    n = 5 * 65536 + 123
    got = [shards.byte_range(n, 4, r) for r in range(4)]
    assert got == [(0, 2 * 65536), (2 * 65536, 4 * 65536), (4 * 65536, 5 * 65536), (5 * 65536, n)]
    assert [shards.byte_range(100, 3, r) for r in range(3)] == [(0, 100), (100, 100), (100, 100)]


def test_shard_table_slices_batch_windows():
    import gcz
    from gcz import shards

    _, wins, _ = gcz.batch_layout([70000, 1, 0, 200000, 65536])
    parts = [shards.shard_table(wins, 3, r) for r in range(3)]
    assert sum(len(p) for p in parts) == len(wins)
    np.testing.assert_array_equal(np.concatenate(parts), wins)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, inputs, out_q):
    try:
        import torch.distributed as dist

        from gcz import shards
        from oracle import oracle as orc

        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        res = {}
        for name, data in inputs.items():
            z_all = shards.zstd_match_find_sharded(
                data, 16, find=lambda b, d: orc.zstd_sequences(b, d, threads=2))
            z_root = shards.zstd_match_find_sharded(
                data, 16, root=0, find=lambda b, d: orc.zstd_sequences(b, d, threads=2))
            l_all = shards.lzma2_match_find_sharded(
                data, 32, find=lambda b, d: (lambda p: (p, orc.has_matches(p, b.size)))(orc.lzma_packed(b, d, threads=2)))
            res[name] = (z_all, z_root, l_all)
        mx = shards.max_over_ranks(1.5 * rank)
        sm = shards.sum_over_ranks(rank + 1)
        dist.barrier()
        dist.destroy_process_group()
        out_q.put((rank, res, mx, sm, None))
    except Exception:  # reported to the parent, which fails the test
        out_q.put((rank, None, None, None, traceback.format_exc()))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_match_find_equals_whole_input(world):
    from oracle import oracle as orc

    inputs = {
        "ragged": cases.build({"kind": "synthetic", "n": 5 * 65536 + 777, "seed": 61}),
        "text": cases.build({"kind": "text", "n": 3 * 65536, "seed": 62}),
        "tiny": cases.build({"kind": "synthetic", "n": 100, "seed": 63}),  # fewer windows than ranks
        "empty": np.zeros(0, np.uint8),
    }
    ctxm = mp.get_context("spawn")
    q = ctxm.Queue()
    port = _free_port()
    procs = [ctxm.Process(target=_rank_main, args=(r, world, port, inputs, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(world):
            rank, res, mx, sm, err = q.get(timeout=240)
            assert err is None, f"rank {rank}:\n{err}"
            got[rank] = (res, mx, sm)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for name, data in inputs.items():
        want_s, want_o = orc.zstd_sequences(data, 16, threads=4)
        want_p = orc.lzma_packed(data, 32, threads=4)
        want_h = orc.has_matches(want_p, data.size)
        for rank in range(world):
            (zs, zo), z_root, (lp, lh) = got[rank][0][name]
            np.testing.assert_array_equal(zo, want_o)
            np.testing.assert_array_equal(zs, want_s.reshape(-1, 4))
            np.testing.assert_array_equal(lp, want_p)
            np.testing.assert_array_equal(lh, want_h)
            if rank == 0:
                np.testing.assert_array_equal(z_root[0], zs)
                np.testing.assert_array_equal(z_root[1], zo)
            else:
                assert z_root is None
    for rank in range(world):
        assert got[rank][1] == 1.5 * (world - 1)
        assert got[rank][2] == world * (world + 1) / 2
