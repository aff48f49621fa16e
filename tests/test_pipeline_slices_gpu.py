"""The host-buffer pipelines cut their input into slices and rotate the slices
over four slots (streams, device buffers, events), finishing each slice three
iterations after queueing it.  Whatever the slice size -- one window per slice,
so that every slot is reused many times, an odd size, or the whole input in one
slice -- every host call returns the same results, equal to the oracle's."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

SLICES = (1, 3, 16, 1 << 20)  # windows per slice; the last is one slice


@pytest.fixture()
def sliced_ctx():
    import gcz

    c = gcz.Context(0)
    yield c
    c.close()


def test_zstd_host_pipeline_any_slice_size(sliced_ctx):
    import gcz

    n = 12 * (1 << 20) + 4097
    data = gcz.gen_synthetic(41, n, 8 << 20)
    o_seqs, o_off = orc.zstd_sequences(data, 64, threads=16)
    for sw in SLICES:
        sliced_ctx.set_option("slice_windows", sw)
        seqs, off = sliced_ctx.zstd_match_find(data, 64)
        np.testing.assert_array_equal(off, o_off, err_msg=f"slice_windows={sw}")
        np.testing.assert_array_equal(seqs, o_seqs, err_msg=f"slice_windows={sw}")


def test_lzma2_host_pipelines_any_slice_size(sliced_ctx):
    import gcz

    n = 6 * (1 << 20) + 333
    data = gcz.gen_synthetic(42, n, 128 << 20)
    o_packed = orc.lzma_packed(data, 32, threads=16)
    o_has = orc.has_matches(o_packed, n)
    small = data[:40 * 65536 + 77]  # the reference layout is 64 bytes per input byte
    o_m, o_c = orc.lzma_ref_layout(small, 8, 32, threads=16)
    for sw in SLICES:
        sliced_ctx.set_option("slice_windows", sw)
        packed, has = sliced_ctx.lzma2_match_find(data)
        np.testing.assert_array_equal(packed, o_packed, err_msg=f"slice_windows={sw}")
        np.testing.assert_array_equal(has, o_has, err_msg=f"slice_windows={sw}")
        np.testing.assert_array_equal(sliced_ctx.lzma2_triage(data), o_has, err_msg=f"slice_windows={sw}")
        d, ln, c = sliced_ctx.lzma2_find_matches(small, 8)
        np.testing.assert_array_equal(c, o_c, err_msg=f"slice_windows={sw}")
        np.testing.assert_array_equal(d.reshape(-1, 8), o_m[:, :, 0], err_msg=f"slice_windows={sw}")
        np.testing.assert_array_equal(ln.reshape(-1, 8), o_m[:, :, 1], err_msg=f"slice_windows={sw}")
