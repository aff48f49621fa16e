"""Failure detection on the GPU without a fault: a kernel wait that runs out
is reported as an error status, and the context keeps working afterwards.
Host-side failures (bad arguments, capacity, bad sequences, a rank that
raises) are covered in the other test files."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_is_reported(ctx):
    import gcz

    rc = gcz.L.gcz_selftest_wait_timeout(ctx.handle, 2000)
    assert rc == -5  # GCZ_EDEVICE
    assert b"bounded wait" in gcz.L.gcz_last_error(ctx.handle)
    # The status word was cleared when it was read, and the device still works.
    ctx.sync()
    data = gcz.gen_synthetic(77, 2 * 65536 + 100, 8 << 20)
    seqs, off = ctx.zstd_match_find(data, 16)
    o_s, o_o = orc.zstd_sequences(data, 16)
    np.testing.assert_array_equal(off, o_o)
    np.testing.assert_array_equal(seqs, o_s)


def test_error_status_does_not_leak_into_the_next_call(ctx):
    import gcz

    assert gcz.L.gcz_selftest_wait_timeout(ctx.handle, 100) == -5
    data = gcz.gen_synthetic(78, 65536, 8 << 20)
    packed, has = ctx.lzma2_match_find(data, 32)
    np.testing.assert_array_equal(packed, orc.lzma_packed(data, 32))
