"""Several GPUs: one process per GPU, each owning a disjoint, contiguous range
of 64 KiB windows.

Every window is independent -- the hash table is reset per window and no
candidate or match crosses a window edge (zstd_compress.cu:179-355,
lzma2_match_find.cu:54-194) -- so a rank's results for its windows equal the
single-GPU results for those windows and the data path has no exchange step.
The reference's own multi-GPU mode is host threads feeding separate devices
with disjoint sub-chunk ranges (pipeline_dual.rs:121, pipeline_lzma2.rs:176-221);
here each device has its own process, and the per-window results are gathered
to the host once the match finding is done.

The process group only carries the host-side gather and the timing reductions
(`max_over_ranks`); on "nccl" the reductions run on a device tensor, on "gloo"
on a host tensor.
"""
import numpy as np

from ._lib import WINDOW

__all__ = ["window_range", "byte_range", "shard_table", "zstd_match_find_sharded", "lzma2_match_find_sharded",
           "max_over_ranks", "sum_over_ranks", "world_rank"]


def world_rank(group=None):
    """(world size, rank) of `group`, or (1, 0) without an initialised process group."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def window_range(num_windows, world, rank):
    """[w0, w1) of the windows rank `rank` owns: contiguous, sizes differ by at
    most one window, lower ranks take the extra ones."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(int(num_windows), world)
    w0 = rank * base + min(rank, extra)
    return w0, w0 + base + (1 if rank < extra else 0)


def byte_range(n, world, rank, window=WINDOW):
    """[lo, hi) of the input bytes rank `rank` owns (window-aligned; the last
    rank with windows ends at n)."""
    nb = (int(n) + window - 1) // window
    w0, w1 = window_range(nb, world, rank)
    return min(w0 * window, n), min(w1 * window, n)


def shard_table(windows, world, rank):
    """The part of a batch window table (gcz.WINDOW_DTYPE rows) rank `rank`
    owns, as a contiguous slice; window i of the batch stays window i - w0 of the
    rank, with its slab offset, size and file index unchanged."""
    w0, w1 = window_range(len(windows), world, rank)
    return windows[w0:w1]


def _device_of(group):
    import torch
    import torch.distributed as dist

    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _reduce(value, op, group):
    import torch
    import torch.distributed as dist

    world, _ = world_rank(group)
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_of(group))
    dist.all_reduce(t, op=op, group=group)
    return float(t.item())


def max_over_ranks(value, group=None):
    """The largest `value` of all ranks (timings are reported as this max)."""
    import torch.distributed as dist

    return _reduce(value, dist.ReduceOp.MAX if dist.is_available() else None, group)


def sum_over_ranks(value, group=None):
    import torch.distributed as dist

    return _reduce(value, dist.ReduceOp.SUM if dist.is_available() else None, group)


def _gather(part, group, root):
    import torch.distributed as dist

    world, rank = world_rank(group)
    if world == 1:
        return [part]
    if root is None:
        parts = [None] * world
        dist.all_gather_object(parts, part, group=group)
        return parts
    parts = [None] * world if rank == root else None
    dist.gather_object(part, parts, dst=root, group=group)
    return parts


def zstd_match_find_sharded(data, search_depth=16, group=None, root=None, find=None):
    """Zstd sequences of the whole input, each rank matching only its windows.

    `find(bytes, depth) -> (seqs u32[N, 4], offsets u64[W+1])` is the per-rank
    match finder (default: this process's GPU context).  Returns the whole
    input's (seqs, offsets) on every rank, or on `root` only (None elsewhere)."""
    from . import _u8, context

    buf = _u8(data)
    world, rank = world_rank(group)
    lo, hi = byte_range(buf.size, world, rank)
    if find is None:
        import torch

        find = context(torch.cuda.current_device() if torch.cuda.is_available() else 0).zstd_match_find
    if hi > lo:
        seqs, off = find(buf[lo:hi], search_depth)
    else:
        seqs, off = np.empty((0, 4), np.uint32), np.zeros(1, np.uint64)
    parts = _gather((np.asarray(seqs), np.asarray(off, np.uint64)), group, root)
    if parts is None:
        return None
    # Sequence records are window-relative; only the offsets need rebasing.
    all_seqs = np.concatenate([p[0].reshape(-1, 4) for p in parts]).astype(np.uint32, copy=False)
    offs, base = [np.zeros(1, np.uint64)], np.uint64(0)
    for _, o in parts:
        offs.append(o[1:] + base)
        base += o[-1]
    return all_seqs, np.concatenate(offs)


def lzma2_match_find_sharded(data, search_depth=32, group=None, root=None, find=None):
    """LZMA2 packed matches (u32 per position) and per-window has-match bytes of
    the whole input, each rank matching only its windows; `find(bytes, depth)
    -> (packed, has)` as for zstd_match_find_sharded."""
    from . import _u8, context

    buf = _u8(data)
    world, rank = world_rank(group)
    lo, hi = byte_range(buf.size, world, rank)
    if find is None:
        import torch

        find = context(torch.cuda.current_device() if torch.cuda.is_available() else 0).lzma2_match_find
    if hi > lo:
        packed, has = find(buf[lo:hi], search_depth)
    else:
        packed, has = np.empty(0, np.uint32), np.empty(0, np.uint8)
    parts = _gather((np.asarray(packed, np.uint32), np.asarray(has, np.uint8)), group, root)
    if parts is None:
        return None
    return np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts])
