// LZMA2 L1+ match finder for sm_100a.
//
// Reproduces lzma2_match_find (lzma2_match_find.cu:54-194) bit for bit.  The
// reference walks each 64 KiB window with one thread: a one-entry 14-bit table
// (empty == 0xFFFF), the "chain" loop stops after its first candidate
// (:157-160), so every position gets at most one match:
//   - candidate = table entry for hash(q) (q+3 < size), verified on 4 bytes
//     (len 4, extended to <= min(size-q, 273)) or else on 2 bytes (len 2,
//     extended the same way, which stops at 3 at most);
//   - if there is none, a distance-1 run when src[q-1]==src[q]==src[q+1]
//     (:164-181).
// Every position with q+3 < size is inserted right after its own lookup, so
// the candidate at q is cand(q) = max{p < q : hash(p) == hash(q)} (or none):
// one warp per window computes it 32 positions per step (__match_any_sync for
// in-step predecessors, shared-memory table for earlier steps) and then every
// lane verifies and extends its own position independently.
#include <type_traits>

#include "gcz_common.cuh"
#include "gcz_kernels.h"

namespace gcz {
namespace {

constexpr uint32_t kLzmaMaxMatch = 273;  // MAX_MATCH_LEN, lzma2_match_find.cu:21
constexpr uint32_t kNone = 0xFFFFu;      // empty sentinel, :73

// First index in [len, lim) where the bytes at c+i and q+i differ, else lim.
template <class Win>
__device__ __forceinline__ uint32_t extend_lane(const Win &win, uint32_t c, uint32_t q, uint32_t len, uint32_t lim) {
    while (len < lim) {
        const uint32_t d = win.u32(q + len) ^ win.u32(c + len);
        if (d) {
            len += (static_cast<uint32_t>(__ffs(d)) - 1u) >> 3;
            return len < lim ? len : lim;
        }
        len += 4u;
    }
    return lim;
}

// First index in [len, lim) where byte q+i differs from `b`, else lim.
template <class Win>
__device__ __forceinline__ uint32_t run_lane(const Win &win, uint32_t q, uint32_t b, uint32_t len, uint32_t lim) {
    const uint32_t pat = b * 0x01010101u;
    while (len < lim) {
        const uint32_t d = win.u32(q + len) ^ pat;
        if (d) {
            len += (static_cast<uint32_t>(__ffs(d)) - 1u) >> 3;
            return len < lim ? len : lim;
        }
        len += 4u;
    }
    return lim;
}

struct LzmaArgs {
    const uint8_t *src;
    uint64_t n;
    uint32_t window;
    uint32_t num_windows;
    uint32_t search_depth;   // 0 disables the hash candidate (chain loop never runs)
    uint32_t max_matches;    // slot stride of the reference layout
    uint32_t *packed;        // compact: len<<16 | dist per position (or null)
    uint8_t *has_matches;    // per window (or null)
    uint32_t *ref_matches;   // reference layout LzmaMatch pairs (or null)
    uint32_t *ref_counts;    // reference layout counts (or null)
    uint32_t *status;
};

template <class Win>
__device__ void lzma_window(const Win &win, uint16_t *T, uint32_t size, const LzmaArgs &a, uint32_t w) {
    const uint32_t lane = lane_id();
    const uint32_t lt = lanemask_lt(), gt = lanemask_gt();
    {
        uint32_t *t32 = reinterpret_cast<uint32_t *>(T);
        for (uint32_t i = lane; i < kHashSize / 2; i += 32) t32[i] = 0xFFFFFFFFu;  // :72-74
    }
    __syncwarp();
    const uint64_t wbase = static_cast<uint64_t>(w) * a.window;
    uint32_t *packed = a.packed ? a.packed + wbase : nullptr;
    uint32_t *rc = a.ref_counts ? a.ref_counts + wbase : nullptr;
    uint32_t *rm = a.ref_matches ? a.ref_matches + wbase * a.max_matches * 2u : nullptr;
    uint32_t any = 0;
    const uint32_t nsteps = (size + 31u) >> 5;
    for (uint32_t s = 0; s < nsteps; ++s) {
        const uint32_t q = (s << 5) + lane;
        const bool valid4 = q + 3u < size;
        const uint32_t x = win.u32(q);
        const uint32_t h = hash4(x);
        const uint32_t g = __match_any_sync(kFull, valid4 ? h : (0x80000000u | lane));
        const uint32_t lower = g & lt;
        const uint32_t tv = valid4 ? static_cast<uint32_t>(T[h]) : kNone;
        const uint32_t cand = lower ? ((s << 5) + 31u - static_cast<uint32_t>(__clz(lower))) : tv;
        __syncwarp();
        if (valid4 && !(g & gt)) T[h] = static_cast<uint16_t>(q);  // :108
        __syncwarp();

        uint32_t dist = 0, len = 0;
        if (q + 1u < size) {
            if (valid4 && a.search_depth > 0 && cand != kNone) {
                const uint32_t lim = size - q < kLzmaMaxMatch ? size - q : kLzmaMaxMatch;
                const uint32_t y = win.u32(cand);
                uint32_t l = 0;
                if (y == x) {
                    l = extend_lane(win, cand, q, 4u, lim);             // :127-133
                } else if (((y ^ x) & 0xFFFFu) == 0u) {
                    l = ((y ^ x) & 0xFF0000u) == 0u ? 3u : 2u;          // :134-139 (byte 3 differs)
                }
                if (l >= 2u) {
                    dist = q - cand;
                    len = l;
                }
            }
            if (len == 0 && q > 0) {  // distance-1 run (:164-181)
                const uint32_t b0 = x & 0xFFu, b1 = (x >> 8) & 0xFFu;
                if (b1 == b0 && win.byte(q - 1u) == b0) {
                    const uint32_t lim = size - q < kLzmaMaxMatch ? size - q : kLzmaMaxMatch;
                    len = run_lane(win, q, b0, 2u, lim);
                    dist = 1;
                }
            }
        }
        if (q < size) {
            if (packed) packed[q] = len ? ((len << 16) | dist) : 0u;
            if (rc) rc[q] = len ? 1u : 0u;
            if (rm && len) {
                uint32_t *slot = rm + static_cast<uint64_t>(q) * a.max_matches * 2u;
                slot[0] = dist;
                slot[1] = len;
            }
        }
        any |= len;
    }
    if (rc)
        for (uint32_t q = size + lane; q < a.window; q += 32) rc[q] = 0u;  // :188-190
    any = __any_sync(kFull, any != 0);
    if (a.has_matches && lane == 0) a.has_matches[w] = any ? 1 : 0;
}

constexpr uint32_t kSmemData = kMaxWindow + 64;
constexpr uint32_t kSmemTable = kHashSize * sizeof(uint16_t);
constexpr uint32_t kSmemStaged = kSmemData + kSmemTable + 16;

template <bool kStaged>
__global__ void __launch_bounds__(32) lzma_match_kernel(LzmaArgs a) {
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
        if constexpr (kStaged) {
            if (!stage_window(smem, a.src + start, size, bar, parity, a.status)) return;
            SmemWin win{reinterpret_cast<const uint32_t *>(smem)};
            lzma_window(win, T, size, a, w);
        } else {
            GlobalWin win{reinterpret_cast<const uint32_t *>(a.src + start), (size + 3u) >> 2};
            lzma_window(win, T, size, a, w);
        }
    }
}

// Packed -> GpuMatchData layout (compress_lzma2_custom.rs:539-549): counts,
// and de-interleaved distance / length arrays with max_matches slots per
// position, unused slots zero (the reference allocates them with alloc_zeros).
__global__ void __launch_bounds__(256) lzma_unpack_kernel(const uint32_t *packed, uint64_t n, uint32_t window,
                                                          uint32_t num_windows, uint32_t max_matches,
                                                          uint32_t *dists, uint32_t *lens, uint32_t *counts) {
    const uint64_t total = static_cast<uint64_t>(num_windows) * window;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        // positions past n inside the last window have count 0
        const uint32_t v = i < n ? packed[i] : 0u;
        if (counts) counts[i] = v ? 1u : 0u;
        const uint64_t base = i * max_matches;
        for (uint32_t k = 0; k < max_matches; ++k) {
            if (dists) dists[base + k] = (k == 0) ? (v & 0xFFFFu) : 0u;
            if (lens) lens[base + k] = (k == 0) ? (v >> 16) : 0u;
        }
    }
}

// ---------------------------------------------------------------------------
// Second stage after the candidate sweep (gcz_sweep.cu): the window is staged
// into shared memory, cand(q) streams in from global memory, and every lane
// verifies its own position.  Lengths use the structure of match runs: when
// cand(q) == cand(q-1)+1 and both positions match on 4 bytes, the common run
// at q is the one at q-1 shortened by one, so only the first lane of each run
// (its head) extends, up to min(size-q, 273+31) bytes, and the other lanes of
// the run derive min(273, E_head - (q - head)) from it -- the same value the
// reference's per-position loop computes with its 273 cap.
constexpr uint32_t kL2Pre = 64;
constexpr uint32_t kL2DataBytes = kL2Pre + kMaxWindow + 64;

struct L2Smem {
    uint8_t data[kL2DataBytes];
    uint32_t any;
    uint32_t flags;
    alignas(8) uint64_t bar;
};

struct L2Args {
    const uint8_t *src;
    const uint16_t *cand;
    uint64_t n;
    uint32_t window;
    uint32_t num_windows;
    uint32_t search_depth;
    uint32_t max_matches;
    uint32_t *packed;
    uint8_t *has_matches;
    uint32_t *ref_matches;
    uint32_t *ref_counts;
    uint32_t *status;
    const WinDesc *wins;
};

// kL2Threads (256, 512 or 1024) is a schedule knob: the window's steps are
// split into kL2Threads / 32 contiguous ranges, one per warp.  Three CTAs
// share an SM (two of 1024 threads).  kRefOut: the reference layout's
// per-position counts and match slots are written too (the parity entry
// points); without it the step loop carries no code for them.
template <uint32_t kL2Threads, bool kRefOut>
__global__ void __launch_bounds__(kL2Threads, kL2Threads == 1024 ? 2 : 3) lzma_verify_kernel(L2Args a) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    L2Smem &S = *reinterpret_cast<L2Smem *>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t lt = lanemask_lt();
    uint32_t parity = 0;
    if (tid == 0) {
        mbar_init(&S.bar, 1);
        fence_mbar_init();
    }
    for (uint32_t i = tid; i < kL2Pre / 4; i += kL2Threads) reinterpret_cast<uint32_t *>(S.data)[i] = 0u;
    __syncthreads();
    SmemWin win{reinterpret_cast<const uint32_t *>(S.data + kL2Pre)};
    for (uint32_t wi = blockIdx.x; wi < a.num_windows; wi += gridDim.x) {
        const uint64_t start = a.wins ? a.wins[wi].offset : static_cast<uint64_t>(wi) * a.window;
        const uint32_t size =
            a.wins ? a.wins[wi].size : static_cast<uint32_t>(a.n - start < a.window ? a.n - start : a.window);
        __syncthreads();
        if (tid == 0) {
            S.any = 0;
            S.flags = 0;
        }
        __syncthreads();
        if (warp == 0) {
            if (!stage_window(S.data + kL2Pre, a.src + start, size, &S.bar, parity, a.status) && lane == 0)
                S.flags = 1u;
        }
        __syncthreads();
        if (S.flags) return;
        const uint16_t *cand = a.cand + start;
        uint32_t *packed = a.packed ? a.packed + start : nullptr;
        uint32_t *rc = kRefOut && a.ref_counts ? a.ref_counts + start : nullptr;
        uint32_t *rm = kRefOut && a.ref_matches ? a.ref_matches + start * a.max_matches * 2u : nullptr;
        uint32_t any = 0;
        const uint32_t nsteps = (size + 31u) >> 5;
        // Each warp takes a contiguous range of steps, so a run of matches
        // (cand(q) = cand(q-1) + 1) carries from one step's last lane into the
        // next step's first: lane 0 then derives its length instead of
        // extending again.  The carried length is exact when it is below 273
        // (an extension is cut only at 273 + 31 bytes or at the window's end).
        constexpr uint32_t kL2Warps = kL2Threads / 32;
        const uint32_t per = (nsteps + kL2Warps - 1u) / kL2Warps;
        const uint32_t s_begin = warp * per, s_end = min(nsteps, s_begin + per);
        uint32_t carry_c = kNone, carry_e = 0;  // last lane of the previous step: candidate, length (0: none)
        // The next step's candidates are loaded while this step is verified.
        uint32_t c_next = (s_begin < s_end && s_begin * 32u + lane + 3u < size) ? cand[s_begin * 32u + lane] : kNone;
        for (uint32_t st = s_begin; st < s_end; ++st) {
            const uint32_t q = st * 32u + lane;
            const bool inwin = q < size;
            const bool valid4 = q + 3u < size;
            const uint32_t x = win.u32(q);
            const uint32_t c = valid4 ? c_next : kNone;
            {
                const uint32_t st2 = st + 1u, q2 = st2 * 32u + lane;
                c_next = (st2 < s_end && q2 + 3u < size) ? static_cast<uint32_t>(cand[q2]) : kNone;
            }
            const bool has = valid4 && a.search_depth > 0 && c != kNone;
            const uint32_t y = has ? win.u32(c) : ~x;
            const bool eq4 = has && y == x;
            // run structure inside the step
            const uint32_t c_prev = __shfl_up_sync(kFull, c, 1);
            const uint32_t eq4_bits = __ballot_sync(kFull, eq4);
            const bool cont = lane > 0 && eq4 && ((eq4_bits >> (lane - 1)) & 1u) && c == c_prev + 1u;
            const uint32_t heads = __ballot_sync(kFull, !cont);
            const uint32_t head = 31u - static_cast<uint32_t>(__clz(heads & (lt | (1u << lane))));
            // Run heads compare 8 more bytes (bytes 4-11) with one unaligned
            // 8-byte read of each side, no loop; a head still matching after
            // that is finished by the whole warp (128 bytes per iteration), so
            // one long run does not leave 31 lanes idle.
            uint32_t ext = 0;
            const uint32_t bound = size - q < kLzmaMaxMatch + 31u ? size - q : kLzmaMaxMatch + 31u;
            bool pending = false;
            if (eq4 && !cont) {
                if (lane == 0 && carry_e > 4u && carry_e < kLzmaMaxMatch && c == carry_c + 1u) {
                    ext = carry_e - 1u;  // the previous step's last match, one byte on
                } else {
                    const uint32_t lim1 = bound < 12u ? bound : 12u;  // bound >= 4 (q + 3 < size)
                    uint32_t ql, qh, cl, ch;
                    win.u64(q + 4u, ql, qh);
                    win.u64(c + 4u, cl, ch);
                    const uint32_t dl = ql ^ cl, dh = qh ^ ch;
                    const uint32_t fb = dl ? (static_cast<uint32_t>(__ffs(dl)) - 1u) >> 3
                                           : (dh ? 4u + ((static_cast<uint32_t>(__ffs(dh)) - 1u) >> 3) : 8u);
                    ext = 4u + fb < lim1 ? 4u + fb : lim1;
                    pending = ext == lim1 && lim1 < bound;
                }
            }
            for (uint32_t pend = __ballot_sync(kFull, pending); pend; pend &= pend - 1u) {
                const uint32_t hl = static_cast<uint32_t>(__ffs(pend)) - 1u;
                const uint32_t hc = __shfl_sync(kFull, c, hl), hq = __shfl_sync(kFull, q, hl);
                const uint32_t hb = __shfl_sync(kFull, bound, hl);
                uint32_t len2 = __shfl_sync(kFull, ext, hl);
                for (;;) {
                    const uint32_t k = len2 + 4u * lane;
                    uint32_t res = k;
                    if (k < hb) {
                        const uint32_t d = win.u32(hq + k) ^ win.u32(hc + k);
                        const uint32_t fb = d ? (static_cast<uint32_t>(__ffs(d)) - 1u) >> 3 : 4u;
                        res = k + (fb < hb - k ? fb : hb - k);
                    }
                    const uint32_t sb = __ballot_sync(kFull, res < k + 4u);
                    if (sb) {
                        len2 = __shfl_sync(kFull, res, static_cast<uint32_t>(__ffs(sb)) - 1u);
                        break;
                    }
                    len2 += 128u;
                }
                if (lane == hl) ext = len2;
            }
            const uint32_t ext_head = __shfl_sync(kFull, ext, head);
            {
                const uint32_t e31 = eq4 ? ext_head - (lane - head) : 0u;
                carry_e = __shfl_sync(kFull, e31, 31);
                carry_c = __shfl_sync(kFull, c, 31);
            }
            uint32_t dist = 0, len = 0;
            if (inwin && q + 1u < size) {
                if (eq4) {
                    const uint32_t e = ext_head - (lane - head);
                    len = e < kLzmaMaxMatch ? e : kLzmaMaxMatch;
                    dist = q - c;
                } else if (has && ((y ^ x) & 0xFFFFu) == 0u) {
                    len = ((y ^ x) & 0xFF0000u) == 0u ? 3u : 2u;  // :134-139 (byte 3 differs)
                    dist = q - c;
                }
                if (len == 0 && q > 0) {  // distance-1 run (:164-181)
                    const uint32_t b0 = x & 0xFFu, b1 = (x >> 8) & 0xFFu;
                    if (b1 == b0 && win.byte(q - 1u) == b0) {
                        const uint32_t lim = size - q < kLzmaMaxMatch ? size - q : kLzmaMaxMatch;
                        len = run_lane(win, q, b0, 2u, lim);
                        dist = 1;
                    }
                }
            }
            if (inwin) {
                if (packed) packed[q] = len ? ((len << 16) | dist) : 0u;
                if (kRefOut && rc) rc[q] = len ? 1u : 0u;
                if (kRefOut && rm && len) {
                    uint32_t *slot = rm + static_cast<uint64_t>(q) * a.max_matches * 2u;
                    slot[0] = dist;
                    slot[1] = len;
                }
            }
            any |= len;
        }
        if (kRefOut && rc)
            for (uint32_t q = size + tid; q < a.window; q += kL2Threads) rc[q] = 0u;  // :188-190
        if (__any_sync(kFull, any != 0) && lane == 0) S.any = 1u;
        __syncthreads();
        if (tid == 0 && a.has_matches) a.has_matches[wi] = S.any ? 1 : 0;
    }
}

}  // namespace

cudaError_t launch_lzma_match(const LzmaLaunch &l, cudaStream_t st) {
    LzmaArgs a{};
    a.src = l.src;
    a.n = l.n;
    a.window = l.window;
    a.num_windows = l.num_windows;
    a.search_depth = l.search_depth;
    a.max_matches = l.max_matches;
    a.packed = l.packed;
    a.has_matches = l.has_matches;
    a.ref_matches = l.ref_matches;
    a.ref_counts = l.ref_counts;
    a.status = l.status;
    if (a.num_windows == 0) return cudaSuccess;
    const bool staged = l.staged != 0;
    int grid = l.num_sms * (staged ? 2 : 6);
    if (static_cast<uint32_t>(grid) > a.num_windows) grid = static_cast<int>(a.num_windows);
    const uint32_t smem = staged ? kSmemStaged : kSmemTable;
    cudaError_t e;
    if (staged) {
        { static SmemOnce smem_set_1{0}; e = set_smem_once(lzma_match_kernel<true>, smem, smem_set_1); }
        if (e != cudaSuccess) return e;
        lzma_match_kernel<true><<<grid, 32, smem, st>>>(a);
    } else {
        { static SmemOnce smem_set_2{0}; e = set_smem_once(lzma_match_kernel<false>, smem, smem_set_2); }
        if (e != cudaSuccess) return e;
        lzma_match_kernel<false><<<grid, 32, smem, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_lzma_unpack(const uint32_t *packed, uint64_t n, uint32_t window, uint32_t num_windows,
                               uint32_t max_matches, uint32_t *dists, uint32_t *lens, uint32_t *counts, int num_sms,
                               cudaStream_t st) {
    if (num_windows == 0) return cudaSuccess;
    lzma_unpack_kernel<<<num_sms * 8, 256, 0, st>>>(packed, n, window, num_windows, max_matches, dists, lens, counts);
    return cudaGetLastError();
}

namespace {
template <uint32_t kThreads, bool kRefOut>
cudaError_t launch_verify_variant(const L2Args &a, const LzmaLaunch &l, cudaStream_t st) {
    const uint32_t smem = sizeof(L2Smem);
    static SmemOnce smem_set{0};
    cudaError_t e = set_smem_once(lzma_verify_kernel<kThreads, kRefOut>, smem, smem_set);
    if (e != cudaSuccess) return e;
    // no more CTAs than fit on the SMs at once, so that no CTA waits for a second wave
    const int fit = kThreads == 1024 ? 2 : 3;
    int grid = l.num_sms * (l.ctas_per_sm > 0 && l.ctas_per_sm < fit ? l.ctas_per_sm : fit);
    if (static_cast<uint32_t>(grid) > l.num_windows) grid = static_cast<int>(l.num_windows);
    lzma_verify_kernel<kThreads, kRefOut><<<grid, kThreads, smem, st>>>(a);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_lzma_verify(const LzmaLaunch &l, const uint16_t *cand, cudaStream_t st) {
    if (l.num_windows == 0) return cudaSuccess;
    L2Args a{};
    a.src = l.src;
    a.cand = cand;
    a.n = l.n;
    a.window = l.window;
    a.num_windows = l.num_windows;
    a.search_depth = l.search_depth;
    a.max_matches = l.max_matches;
    a.packed = l.packed;
    a.has_matches = l.has_matches;
    a.ref_matches = l.ref_matches;
    a.ref_counts = l.ref_counts;
    a.status = l.status;
    a.wins = l.wins;
    if (a.ref_counts || a.ref_matches) {
        if (l.threads == 256) return launch_verify_variant<256, true>(a, l, st);
        if (l.threads == 512) return launch_verify_variant<512, true>(a, l, st);
        return launch_verify_variant<1024, true>(a, l, st);
    }
    if (l.threads == 256) return launch_verify_variant<256, false>(a, l, st);
    if (l.threads == 512) return launch_verify_variant<512, false>(a, l, st);
    return launch_verify_variant<1024, false>(a, l, st);
}

}  // namespace gcz
