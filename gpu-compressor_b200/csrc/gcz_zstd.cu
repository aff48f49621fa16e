// Zstd L1/L2 match finder for sm_100a.
//
// Reproduces zstd_match_find (zstd_compress.cu:179-355) bit for bit: per 64 KiB
// window, a one-entry 14-bit hash table (empty == position 0), hash candidates
// verified on 3 bytes, the three repeat offsets {1,4,8} tried only when the hash
// candidate fails (first hit wins), one lazy step at pos+1 taken when
// len2 > len+1, and the table filled for every position of an emitted match.
//
// Why the parallel form is exact: every position p with p+3 < size is written
// into the table exactly once and in increasing order (visited positions at
// :235, the lazy position at :303, match interiors at :328-331), and every
// lookup at q (:232, and :280 with q = pos+1) happens after all p < q were
// written and before q is.  So the candidate the reference sees at q is
//     cand(q) = max{ p < q : hash(p) == hash(q) }, or 0 if there is none,
// a pure function of the input, independent of the parse.  One warp owns one
// window: it sweeps the positions 32 at a time computing cand(q) with
// __match_any_sync for in-step predecessors and the shared-memory table for
// earlier steps, then runs the parse one step behind the sweep (the lazy check
// at the last lane of a step needs the first candidate of the next step).  In
// literal runs the parse advances 32 positions per ballot; matches and lazy
// candidates are extended 128 bytes per warp iteration.
#include <type_traits>

#include "gcz_common.cuh"
#include "gcz_kernels.h"

namespace gcz {
namespace {

constexpr uint32_t kZstdMinMatch = 3;  // MIN_MATCH_LEN, zstd_compress.cu:28

// Length of the common run of window bytes at c and q, known to be >= len,
// bounded by lim (= size - q).  Warp-cooperative: each lane compares 4 bytes,
// 128 bytes per iteration.  All lanes return the same value.
template <class Win>
__device__ __forceinline__ uint32_t extend_warp(const Win &win, uint32_t c, uint32_t q, uint32_t len, uint32_t lim) {
    const uint32_t lane = lane_id();
    for (;;) {
        const uint32_t k = len + 4u * lane;
        uint32_t res = k;
        if (k < lim) {
            const uint32_t d = win.u32(q + k) ^ win.u32(c + k);
            const uint32_t fb = d ? (static_cast<uint32_t>(__ffs(d)) - 1u) >> 3 : 4u;
            const uint32_t rem = lim - k;
            res = k + (fb < rem ? fb : rem);
        }
        const uint32_t sb = __ballot_sync(kFull, res < k + 4u);
        if (sb) return __shfl_sync(kFull, res, __ffs(sb) - 1);
        len += 128u;
    }
}

// Sequence sinks.  Sequences are staged one per lane and flushed 32 at a time
// with coalesced stores.
struct PackedSink {  // uint2{ ll | (ml-3) << 16, off } at stride max_seqs
    uint2 *out;
    uint32_t a = 0, b = 0;
    __device__ __forceinline__ void put(uint32_t idx, uint32_t ll, uint32_t mlm3, uint32_t off) {
        if (lane_id() == (idx & 31u)) {
            a = ll | (mlm3 << 16);
            b = off;
        }
        if ((idx & 31u) == 31u) out[(idx & ~31u) + lane_id()] = make_uint2(a, b);
    }
    __device__ __forceinline__ void finish(uint32_t n) {
        if (lane_id() < (n & 31u)) out[(n & ~31u) + lane_id()] = make_uint2(a, b);
    }
};
struct RefSink {  // Sequence{literal_length, match_length-3, offset} (zstd_compress.cu:38-42)
    uint32_t *out;
    uint32_t a = 0, b = 0, c = 0;
    __device__ __forceinline__ void put(uint32_t idx, uint32_t ll, uint32_t mlm3, uint32_t off) {
        if (lane_id() == (idx & 31u)) {
            a = ll;
            b = mlm3;
            c = off;
        }
        if ((idx & 31u) == 31u) store((idx & ~31u) + lane_id());
    }
    __device__ __forceinline__ void store(uint32_t i) {
        out[3u * i + 0] = a;
        out[3u * i + 1] = b;
        out[3u * i + 2] = c;
    }
    __device__ __forceinline__ void finish(uint32_t n) {
        if (lane_id() < (n & 31u)) store((n & ~31u) + lane_id());
    }
};

// One window, one warp.  T: this warp's 16384-entry table in shared memory.
// Returns {sequence count, literal count}.
template <class Win, class Sink>
__device__ uint2 zstd_window(const Win &win, uint16_t *T, uint32_t size, bool lazy, uint32_t max_seqs, Sink &sink) {
    const uint32_t lane = lane_id();
    const uint32_t lt = lanemask_lt(), gt = lanemask_gt();
    {
        uint32_t *t32 = reinterpret_cast<uint32_t *>(T);
        for (uint32_t i = lane; i < kHashSize / 2; i += 32) t32[i] = 0u;  // empty == position 0 (:195-200)
    }
    __syncwarp();

    uint32_t p = 0, lit_start = 0, nseq = 0, covered = 0;
    uint32_t rep0 = 1, rep1 = 4, rep2 = 8;  // :225
    uint32_t px = 0, pc = 0, ph = 0;        // previous step: bytes, candidate, verified flag
    const uint32_t nsteps = (size + 31u) >> 5;

    for (uint32_t s = 0; s <= nsteps; ++s) {
        // ---- sweep step s: cand(q) and its 3-byte verification
        uint32_t cx = 0, cc = 0, ch = 0;
        if (s < nsteps) {
            const uint32_t q = (s << 5) + lane;
            const bool valid = q + 3u < size;
            cx = win.u32(q);
            const uint32_t h = hash4(cx);
            const uint32_t g = __match_any_sync(kFull, valid ? h : (0x80000000u | lane));
            const uint32_t lower = g & lt;
            const uint32_t tv = valid ? static_cast<uint32_t>(T[h]) : 0u;
            cc = lower ? ((s << 5) + 31u - static_cast<uint32_t>(__clz(lower))) : tv;
            __syncwarp();
            if (valid && !(g & gt)) T[h] = static_cast<uint16_t>(q);
            __syncwarp();
            ch = (valid && cc != q && ((cx ^ win.u32(cc)) & 0xFFFFFFu) == 0u) ? 1u : 0u;
        }
        // ---- parse positions of step s-1
        if (s > 0) {
            const uint32_t B = (s - 1u) << 5;
            const uint32_t q = B + lane;
            while (p < B + 32u && p + 3u < size) {
                const bool elig = q >= p && q + 3u < size;
                const uint32_t hb = __ballot_sync(kFull, elig && ph);
                const uint32_t pl = p - B;
                const uint32_t fh = hb ? static_cast<uint32_t>(__ffs(hb)) - 1u : 32u;
                uint32_t rb = 0, rsel = 0;
                if (fh > pl) {  // lanes in [pl, fh) have no hash match: try the repeat offsets (:259-275)
                    const bool need = elig && lane < fh;
                    const bool r0 = need && rep0 <= q && ((px ^ win.u32(rep0 <= q ? q - rep0 : 0u)) & 0xFFFFFFu) == 0u;
                    const bool r1 =
                        need && !r0 && rep1 <= q && ((px ^ win.u32(rep1 <= q ? q - rep1 : 0u)) & 0xFFFFFFu) == 0u;
                    const bool r2 = need && !r0 && !r1 && rep2 <= q &&
                                    ((px ^ win.u32(rep2 <= q ? q - rep2 : 0u)) & 0xFFFFFFu) == 0u;
                    rsel = r0 ? 0u : (r1 ? 1u : 2u);
                    rb = __ballot_sync(kFull, r0 || r1 || r2);
                }
                const uint32_t b = hb | rb;
                if (!b) {
                    p = B + 32u;
                    break;
                }
                const uint32_t f = static_cast<uint32_t>(__ffs(b)) - 1u;
                uint32_t pos = B + f, len, off;
                if ((hb >> f) & 1u) {
                    const uint32_t c = __shfl_sync(kFull, pc, f);
                    off = pos - c;
                    len = extend_warp(win, c, pos, kZstdMinMatch, size - pos);
                } else {
                    const uint32_t r = __shfl_sync(kFull, rsel, f);
                    off = r == 0u ? rep0 : (r == 1u ? rep1 : rep2);
                    len = extend_warp(win, pos - off, pos, kZstdMinMatch, size - pos);
                }
                // Lazy step (:278-307): the hash candidate of pos+1.
                const uint32_t h1a = __shfl_sync(kFull, ph, (f + 1u) & 31u);
                const uint32_t c1a = __shfl_sync(kFull, pc, (f + 1u) & 31u);
                const uint32_t h1b = __shfl_sync(kFull, ch, 0);
                const uint32_t c1b = __shfl_sync(kFull, cc, 0);
                if (lazy && pos + 4u < size) {
                    const uint32_t h1 = f < 31u ? h1a : h1b;
                    const uint32_t c1 = f < 31u ? c1a : c1b;
                    if (h1) {
                        const uint32_t len2 = extend_warp(win, c1, pos + 1u, kZstdMinMatch, size - pos - 1u);
                        if (len2 > len + 1u) {
                            pos += 1u;
                            len = len2;
                            off = pos - c1;
                        }
                    }
                }
                if (nseq < max_seqs) {  // :309-334
                    sink.put(nseq, pos - lit_start, len - kZstdMinMatch, off);
                    ++nseq;
                    rep2 = rep1;
                    rep1 = rep0;
                    rep0 = off;
                    covered += len;
                    p = pos + len;
                    lit_start = p;
                } else {
                    p = pos + 1u;
                }
            }
        }
        px = cx;
        pc = cc;
        ph = ch;
    }
    sink.finish(nseq);
    return make_uint2(nseq, size - covered);
}

struct ZstdArgs {
    const uint8_t *src;
    uint64_t n;             // total input bytes
    uint32_t window;        // window (chunk) size, multiple of 16, <= 65536
    uint32_t num_windows;
    uint32_t lazy;          // search_depth > 1
    uint32_t max_seqs;      // per-window capacity (stride of the outputs)
    uint2 *packed;          // PackedSink output (or null)
    uint32_t *ref_seqs;     // RefSink output (or null)
    uint32_t *seq_counts;
    uint32_t *lit_counts;   // may be null
    uint32_t *status;
};

constexpr uint32_t kSmemData = kMaxWindow + 64;                 // staged window + padding
constexpr uint32_t kSmemTable = kHashSize * sizeof(uint16_t);   // 32 KiB
constexpr uint32_t kSmemStaged = kSmemData + kSmemTable + 16;   // + mbarrier

// Persistent: one warp per CTA, windows strided over the grid.
template <bool kStaged, class Sink>
__global__ void __launch_bounds__(32) zstd_match_kernel(ZstdArgs a) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint16_t *T = reinterpret_cast<uint16_t *>(smem + (kStaged ? kSmemData : 0u));
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kSmemData + kSmemTable);
    uint32_t parity = 0;
    if (kStaged) {
        if (lane_id() == 0) {
            mbar_init(bar, 1);
            fence_mbar_init();
        }
        __syncwarp();
    }
    for (uint32_t w = blockIdx.x; w < a.num_windows; w += gridDim.x) {
        const uint64_t start = static_cast<uint64_t>(w) * a.window;
        const uint32_t size = static_cast<uint32_t>(a.n - start < a.window ? a.n - start : a.window);
        Sink sink;
        uint2 r;
        if constexpr (std::is_same<Sink, PackedSink>::value) {
            sink.out = a.packed + static_cast<uint64_t>(w) * a.max_seqs;
        } else {
            sink.out = a.ref_seqs + static_cast<uint64_t>(w) * a.max_seqs * 3u;
        }
        if constexpr (kStaged) {
            if (!stage_window(smem, a.src + start, size, bar, parity, a.status)) return;
            SmemWin win{reinterpret_cast<const uint32_t *>(smem)};
            r = zstd_window(win, T, size, a.lazy != 0, a.max_seqs, sink);
        } else {
            GlobalWin win{reinterpret_cast<const uint32_t *>(a.src + start), (size + 3u) >> 2};
            r = zstd_window(win, T, size, a.lazy != 0, a.max_seqs, sink);
        }
        if (lane_id() == 0) {
            a.seq_counts[w] = r.x;
            if (a.lit_counts) a.lit_counts[w] = r.y;
        }
    }
}

// Exclusive scan of per-window counts into 64-bit offsets (num+1 entries).
// One CTA of 1024 threads walks the array in tiles.
__global__ void __launch_bounds__(1024) scan_counts_kernel(const uint32_t *counts, uint32_t num, uint64_t *offsets) {
    __shared__ uint64_t warp_sums[32];
    __shared__ uint64_t carry_s;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
    if (tid == 0) carry_s = 0;
    __syncthreads();
    for (uint32_t base = 0; base < num; base += 1024u) {
        const uint32_t i = base + tid;
        const uint64_t v = i < num ? counts[i] : 0u;
        uint64_t x = v;
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint64_t y = __shfl_up_sync(kFull, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            uint64_t s = warp_sums[lane];
            for (uint32_t d = 1; d < 32; d <<= 1) {
                const uint64_t y = __shfl_up_sync(kFull, s, d);
                if (lane >= d) s += y;
            }
            warp_sums[lane] = s;  // inclusive over warps
        }
        __syncthreads();
        const uint64_t carry = carry_s;
        const uint64_t incl = x + (wid ? warp_sums[wid - 1] : 0u) + carry;
        if (i < num) offsets[i] = incl - v;
        __syncthreads();
        if (tid == 1023) carry_s = incl;
        __syncthreads();
    }
    if (tid == 0) offsets[num] = carry_s;
}

// Packed sequences at stride max_seqs -> compact ZSTD_Sequence records
// (offset, litLength, matchLength = ml-3+3, rep = 0), compress_zstd_custom.rs:140-153.
__global__ void __launch_bounds__(256) expand_seqs_kernel(const uint2 *packed, const uint32_t *counts,
                                                          const uint64_t *offsets, uint32_t num, uint32_t max_seqs,
                                                          uint4 *out, uint64_t capacity, uint32_t *status) {
    for (uint32_t w = blockIdx.x; w < num; w += gridDim.x) {
        const uint32_t cnt = counts[w];
        const uint64_t o = offsets[w];
        const uint2 *src = packed + static_cast<uint64_t>(w) * max_seqs;
        if (o + cnt > capacity) {
            if (threadIdx.x == 0) atomicOr(status, kErrCapacity);
            continue;
        }
        for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
            const uint2 v = src[i];
            out[o + i] = make_uint4(v.y, v.x & 0xFFFFu, (v.x >> 16) + kZstdMinMatch, 0u);
        }
    }
}

// The same records compacted as 8 bytes each: {litLength | (matchLength-3) << 16,
// offset} (a window's lengths and offsets are below 65536).
__global__ void __launch_bounds__(256) compact_seqs_kernel(const uint2 *packed, const uint32_t *counts,
                                                           const uint64_t *offsets, uint32_t num, uint32_t max_seqs,
                                                           uint2 *out, uint64_t capacity, uint32_t *status) {
    for (uint32_t w = blockIdx.x; w < num; w += gridDim.x) {
        const uint32_t cnt = counts[w];
        const uint64_t o = offsets[w];
        const uint2 *src = packed + static_cast<uint64_t>(w) * max_seqs;
        if (o + cnt > capacity) {
            if (threadIdx.x == 0) atomicOr(status, kErrCapacity);
            continue;
        }
        for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) out[o + i] = src[i];
    }
}

// Literal bytes in the reference layout (zstd_compress.cu:311-314,341-343):
// every byte not covered by a match, in order, at stride `window` per window.
// One warp per window walks its sequences.
__global__ void __launch_bounds__(32) zstd_literals_kernel(const uint8_t *src, uint64_t n, uint32_t window,
                                                           uint32_t num_windows, const uint32_t *ref_seqs,
                                                           const uint32_t *seq_counts, uint32_t max_seqs,
                                                           uint8_t *lits) {
    const uint32_t lane = lane_id();
    for (uint32_t w = blockIdx.x; w < num_windows; w += gridDim.x) {
        const uint64_t start = static_cast<uint64_t>(w) * window;
        const uint32_t size = static_cast<uint32_t>(n - start < window ? n - start : window);
        const uint8_t *s = src + start;
        uint8_t *d = lits + start;
        const uint32_t *sq = ref_seqs + static_cast<uint64_t>(w) * max_seqs * 3u;
        const uint32_t cnt = seq_counts[w];
        uint32_t pos = 0, nl = 0;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t ll = sq[3u * k], ml = sq[3u * k + 1] + kZstdMinMatch;
            for (uint32_t i = lane; i < ll; i += 32) d[nl + i] = s[pos + i];
            nl += ll;
            pos += ll + ml;
        }
        for (uint32_t i = lane; pos + i < size; i += 32) d[nl + i] = s[pos + i];
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers (host side)
// ---------------------------------------------------------------------------
static int zstd_grid(uint32_t num_windows, int num_sms, bool staged) {
    const int per_sm = staged ? 2 : 6;
    int g = num_sms * per_sm;
    if (static_cast<uint32_t>(g) > num_windows) g = static_cast<int>(num_windows);
    return g < 1 ? 1 : g;
}

cudaError_t launch_zstd_match(const ZstdLaunch &l, cudaStream_t st) {
    ZstdArgs a{};
    a.src = l.src;
    a.n = l.n;
    a.window = l.window;
    a.num_windows = l.num_windows;
    a.lazy = l.search_depth > 1 ? 1u : 0u;
    a.max_seqs = l.max_seqs;
    a.packed = reinterpret_cast<uint2 *>(l.packed);
    a.ref_seqs = l.ref_seqs;
    a.seq_counts = l.seq_counts;
    a.lit_counts = l.lit_counts;
    a.status = l.status;
    if (a.num_windows == 0) return cudaSuccess;
    const bool staged = l.staged != 0;
    const int grid = zstd_grid(a.num_windows, l.num_sms, staged);
    const uint32_t smem = staged ? kSmemStaged : kSmemTable;
    cudaError_t e;
    if (l.ref_seqs) {
        if (staged) {
            e = cudaFuncSetAttribute(zstd_match_kernel<true, RefSink>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
            zstd_match_kernel<true, RefSink><<<grid, 32, smem, st>>>(a);
        } else {
            e = cudaFuncSetAttribute(zstd_match_kernel<false, RefSink>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
            zstd_match_kernel<false, RefSink><<<grid, 32, smem, st>>>(a);
        }
    } else {
        if (staged) {
            e = cudaFuncSetAttribute(zstd_match_kernel<true, PackedSink>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
            zstd_match_kernel<true, PackedSink><<<grid, 32, smem, st>>>(a);
        } else {
            e = cudaFuncSetAttribute(zstd_match_kernel<false, PackedSink>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
            zstd_match_kernel<false, PackedSink><<<grid, 32, smem, st>>>(a);
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_scan_counts(const uint32_t *counts, uint32_t num, uint64_t *offsets, cudaStream_t st) {
    scan_counts_kernel<<<1, 1024, 0, st>>>(counts, num, offsets);
    return cudaGetLastError();
}

cudaError_t launch_expand_seqs(const void *packed, const uint32_t *counts, const uint64_t *offsets, uint32_t num,
                               uint32_t max_seqs, void *out, uint64_t capacity, uint32_t *status, int num_sms,
                               cudaStream_t st) {
    if (num == 0) return cudaSuccess;
    int grid = num_sms * 8;
    if (static_cast<uint32_t>(grid) > num) grid = static_cast<int>(num);
    expand_seqs_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const uint2 *>(packed), counts, offsets, num, max_seqs,
                                             reinterpret_cast<uint4 *>(out), capacity, status);
    return cudaGetLastError();
}

cudaError_t launch_compact_seqs(const void *packed, const uint32_t *counts, const uint64_t *offsets, uint32_t num,
                                uint32_t max_seqs, void *out, uint64_t capacity, uint32_t *status, int num_sms,
                                cudaStream_t st) {
    if (num == 0) return cudaSuccess;
    int grid = num_sms * 8;
    if (static_cast<uint32_t>(grid) > num) grid = static_cast<int>(num);
    compact_seqs_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const uint2 *>(packed), counts, offsets, num, max_seqs,
                                              reinterpret_cast<uint2 *>(out), capacity, status);
    return cudaGetLastError();
}

cudaError_t launch_zstd_literals(const uint8_t *src, uint64_t n, uint32_t window, uint32_t num_windows,
                                 const uint32_t *ref_seqs, const uint32_t *seq_counts, uint32_t max_seqs, uint8_t *lits,
                                 int num_sms, cudaStream_t st) {
    if (num_windows == 0) return cudaSuccess;
    int grid = num_sms * 16;
    if (static_cast<uint32_t>(grid) > num_windows) grid = static_cast<int>(num_windows);
    zstd_literals_kernel<<<grid, 32, 0, st>>>(src, n, window, num_windows, ref_seqs, seq_counts, max_seqs, lits);
    return cudaGetLastError();
}

}  // namespace gcz
