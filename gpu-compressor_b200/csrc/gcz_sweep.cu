// Candidate sweep shared by the Zstd and LZMA2 match finders.
//
// Both reference kernels keep a one-entry 14-bit table per 64 KiB window and
// write every position p with p+3 < size into it exactly once, in increasing
// order, each lookup at q happening after all p < q were written
// (zstd_compress.cu:231-235,280,303,328-331; lzma2_match_find.cu:104-108).  The
// candidate either of them sees at q is therefore
//     cand(q) = max{ p < q : hash4(p) == hash4(q) }       (0xFFFF if none)
// which this kernel computes for every position of every window; the match
// finders then verify, extend and parse from it.
//
// One warp sweeps one window 32 positions per step.  Each lane reads its
// bucket (the last position of earlier steps), writes its own position and
// reads it back; when every lane reads back its own position no two lanes of
// the step share a bucket, the values read are the candidates and the table
// is up to date.  Otherwise (equal hashes inside a step) the table is restored
// from that step on, and in each step with equal hashes __match_any_sync
// groups the lanes: the in-step predecessor is the next lower lane of the
// group and the highest lane writes the bucket.  Only the table lives in
// shared memory (32 KiB), so seven windows are swept per SM; the input streams
// through coalesced 128-byte loads.
#include "gcz_common.cuh"
#include "gcz_kernels.h"

namespace gcz {
namespace {


struct SweepArgs {
    const uint8_t *src;
    uint64_t n;
    uint32_t window;
    uint32_t num_windows;
    uint16_t *cand;  // one entry per input byte, same offsets as src
    const WinDesc *wins;
};

// Lanes of this warp whose key equals this lane's (valid lanes only; an
// invalid lane matches only itself): kBits ballots, one per key bit, combined
// bit-sliced.  The ballots do not depend on each other, so their latency
// overlaps, unlike one __match_any_sync.
template <int kBits>
__device__ __forceinline__ uint32_t same_key_lanes(uint32_t key, bool valid) {
    uint32_t m = __ballot_sync(kFull, valid);
#pragma unroll
    for (int b = 0; b < kBits; ++b) {
        const bool bit = (key >> b) & 1u;
        const uint32_t bb = __ballot_sync(kFull, bit);
        m &= bit ? bb : ~bb;
    }
    return valid ? m : (1u << lane_id());
}

// The hashes of one 128-position block (independent of the table): step j,
// lane l is position blk * 128 + 32 j + l.  Lane l holds word l of the block
// (w0) and word l of the next block (w1; only lane 0's is used).
__device__ __forceinline__ void block_hashes(uint32_t blk, uint32_t size, uint32_t w0, uint32_t w1, uint32_t *h,
                                             bool *v) {
    const uint32_t lane = lane_id();
    const uint32_t up = __shfl_down_sync(kFull, w0, 1);
    const uint32_t n0 = __shfl_sync(kFull, w1, 0);
    const uint32_t w0n = lane == 31u ? n0 : up;  // word l+1
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t q = blk * 128u + j * 32u + lane;
        const uint32_t src_lane = j * 8u + (lane >> 2);
        const uint32_t lo = __shfl_sync(kFull, w0, src_lane);
        const uint32_t hi = __shfl_sync(kFull, w0n, src_lane);
        v[j] = q + 3u < size;
        h[j] = hash4(__funnelshift_r(lo, hi, (lane & 3u) * 8u));
    }
}

// The block's table work and candidates, from its hashes.
template <bool kBallotGroups>
__device__ __forceinline__ void block_table(uint16_t *T, uint16_t *out, uint32_t blk, uint32_t size,
                                            const uint32_t *h, const bool *v, uint32_t lt, uint32_t gt) {
    const uint32_t lane = lane_id();
    // Step by step: read the bucket, write this position,
    // read it back.  A lane that does not read back its own position
    // shares its bucket with another lane of the same step.
    uint32_t tv[4], dup = 0;
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t q = blk * 128u + j * 32u + lane;
        tv[j] = v[j] ? static_cast<uint32_t>(T[h[j]]) : 0xFFFFu;
        __syncwarp();
        if (v[j]) T[h[j]] = static_cast<uint16_t>(q);
        __syncwarp();
        if (v[j] && T[h[j]] != static_cast<uint16_t>(q)) dup |= 1u << j;
    }
    uint32_t g[4] = {1u << lane, 1u << lane, 1u << lane, 1u << lane};
    const uint32_t dsteps = __reduce_or_sync(kFull, dup);  // steps with equal hashes in two lanes
    if (dsteps) {
        // One block in two on compressible data.  Steps before the
        // first such step j0 wrote each bucket once and are exact.  Put
        // the table back as it was before j0 (latest steps first, so
        // each bucket ends with the value its earliest step from j0 on
        // read) and redo from j0, grouping the lanes of the steps that
        // share buckets.  Which lanes share a bucket depends only on
        // the hashes, so the other steps need no groups.
        const uint32_t j0 = static_cast<uint32_t>(__ffs(dsteps)) - 1u;
        __syncwarp();
#pragma unroll
        for (int j = 3; j >= 0; --j) {
            if (static_cast<uint32_t>(j) >= j0) {
                if (v[j]) T[h[j]] = static_cast<uint16_t>(tv[j]);
                __syncwarp();
            }
        }
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) {
            if (j < j0) continue;
            const uint32_t q = blk * 128u + j * 32u + lane;
            if ((dsteps >> j) & 1u) {
                if constexpr (kBallotGroups) g[j] = same_key_lanes<kHashLog>(h[j], v[j]);
                else g[j] = __match_any_sync(kFull, v[j] ? h[j] : (0x80000000u | lane));
            }
            tv[j] = v[j] ? static_cast<uint32_t>(T[h[j]]) : 0xFFFFu;
            __syncwarp();
            if (v[j] && !(g[j] & gt)) T[h[j]] = static_cast<uint16_t>(q);
            __syncwarp();
        }
    }
    // ... then the candidates.
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t q = blk * 128u + j * 32u + lane;
        const uint32_t lower = g[j] & lt;
        const uint32_t c = lower ? (q - lane + 31u - static_cast<uint32_t>(__clz(lower))) : tv[j];
        if (q < size) out[q] = static_cast<uint16_t>(c);
    }
}

// One 128-position block of a window's sweep: hashes, then table work.
template <bool kBallotGroups>
__device__ __forceinline__ void sweep_block(uint16_t *T, uint16_t *out, uint32_t blk, uint32_t size, uint32_t w0,
                                            uint32_t w1, uint32_t lt, uint32_t gt) {
    uint32_t h[4];
    bool v[4];
    block_hashes(blk, size, w0, w1, h, v);
    block_table<kBallotGroups>(T, out, blk, size, h, v, lt, gt);
}

// Word l of block b of a window (0 past its end).
__device__ __forceinline__ uint32_t block_word(const uint32_t *src32, uint32_t nwords, uint32_t b) {
    const uint32_t i = b * 32u + lane_id();
    return i < nwords ? __ldg(src32 + i) : 0u;
}

// kSweepWarpsPerCta windows per CTA, one 32 KiB table each (7 fill an SM's
// shared memory); a schedule knob, the candidates do not depend on it.  So is
// kBallotGroups: how the lanes of a step with equal hashes are grouped
// (__match_any_sync, or bit-sliced ballots), and kPf, how many 128-byte
// blocks ahead the input is prefetched into L2 (0: not at all; a compile-time
// distance, which measured 0.4 ms per GiB faster than the same distance read
// from the kernel's arguments).
template <int kSweepWarpsPerCta, bool kBallotGroups, uint32_t kPf>
__global__ void __launch_bounds__(32 * kSweepWarpsPerCta) cand_sweep_kernel(SweepArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint16_t *T = reinterpret_cast<uint16_t *>(smem) + warp * kHashSize;
    uint4 *T4 = reinterpret_cast<uint4 *>(T);
    const uint32_t lt = lanemask_lt(), gt = lanemask_gt();
    const uint32_t gwarps = gridDim.x * kSweepWarpsPerCta;
    for (uint32_t w = blockIdx.x * kSweepWarpsPerCta + warp; w < a.num_windows; w += gwarps) {
        const uint64_t start = a.wins ? a.wins[w].offset : static_cast<uint64_t>(w) * a.window;
        const uint32_t size =
            a.wins ? a.wins[w].size : static_cast<uint32_t>(a.n - start < a.window ? a.n - start : a.window);
        for (uint32_t i = lane; i < kHashSize * 2 / 16; i += 32) T4[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
        __syncwarp();
        const uint32_t *src32 = reinterpret_cast<const uint32_t *>(a.src + start);
        const uint32_t nwords = (size + 3u) >> 2;
        uint16_t *out = a.cand + start;
        const uint32_t nblk = (size + 127u) >> 7;
        // 128-byte blocks: lane l holds word l.  Each block's words are loaded
        // two blocks ahead of its sweep; with kPf > 0 lane 0 also prefetches
        // block b + kPf into L2 while block b is swept, so that those loads hit
        // L2 instead of waiting on DRAM.
        uint32_t w0 = block_word(src32, nwords, 0), w1 = block_word(src32, nwords, 1);
        for (uint32_t blk = 0; blk < nblk; ++blk) {
            if constexpr (kPf > 0) {
                const uint32_t pw = (blk + kPf) * 32u;
                if (lane == 0 && pw < nwords) asm volatile("prefetch.global.L2 [%0];" ::"l"(src32 + pw));
            }
            const uint32_t w2 = block_word(src32, nwords, blk + 2u);
            sweep_block<kBallotGroups>(T, out, blk, size, w0, w1, lt, gt);
            w0 = w1;
            w1 = w2;
        }
        __syncwarp();
    }
}

// The same candidates with each step's lanes grouped by hash one block
// ahead.  Which lanes of a step share a bucket depends only on the input
// bytes, so the groups of block b+1 are formed (by __match_any_sync or by
// bit-sliced ballots) while block b's table work runs, and their latency
// overlaps it.  With the groups known, each step is one read (every lane reads
// its bucket: the lowest lane of a group gets the table's candidate, the others
// take the next lower lane's position) and one write (the highest lane of each
// group), with no read-back and no redo.
template <bool kBallots>
__device__ __forceinline__ void block_hashes_groups(uint32_t blk, uint32_t size, uint32_t w0, uint32_t w1,
                                                    uint32_t *h, bool *v, uint32_t *g) {
    const uint32_t lane = lane_id();
    const uint32_t up = __shfl_down_sync(kFull, w0, 1);
    const uint32_t n0 = __shfl_sync(kFull, w1, 0);
    const uint32_t w0n = lane == 31u ? n0 : up;  // word l+1
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t q = blk * 128u + j * 32u + lane;
        const uint32_t src_lane = j * 8u + (lane >> 2);
        const uint32_t lo = __shfl_sync(kFull, w0, src_lane);
        const uint32_t hi = __shfl_sync(kFull, w0n, src_lane);
        v[j] = q + 3u < size;
        h[j] = hash4(__funnelshift_r(lo, hi, (lane & 3u) * 8u));
    }
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
        if constexpr (kBallots) g[j] = same_key_lanes<kHashLog>(h[j], v[j]);
        else g[j] = __match_any_sync(kFull, v[j] ? h[j] : (0x80000000u | lane));
    }
}

template <int kSweepWarpsPerCta, bool kBallots>
__global__ void __launch_bounds__(32 * kSweepWarpsPerCta) cand_sweep_ahead_kernel(SweepArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint16_t *T = reinterpret_cast<uint16_t *>(smem) + warp * kHashSize;
    uint4 *T4 = reinterpret_cast<uint4 *>(T);
    const uint32_t lt = lanemask_lt(), gt = lanemask_gt();
    const uint32_t gwarps = gridDim.x * kSweepWarpsPerCta;
    for (uint32_t w = blockIdx.x * kSweepWarpsPerCta + warp; w < a.num_windows; w += gwarps) {
        const uint64_t start = a.wins ? a.wins[w].offset : static_cast<uint64_t>(w) * a.window;
        const uint32_t size =
            a.wins ? a.wins[w].size : static_cast<uint32_t>(a.n - start < a.window ? a.n - start : a.window);
        for (uint32_t i = lane; i < kHashSize * 2 / 16; i += 32) T4[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
        __syncwarp();
        const uint32_t *src32 = reinterpret_cast<const uint32_t *>(a.src + start);
        const uint32_t nwords = (size + 3u) >> 2;
        uint16_t *out = a.cand + start;
        uint32_t w0 = lane < nwords ? __ldg(src32 + lane) : 0u;
        uint32_t w1 = 32u + lane < nwords ? __ldg(src32 + 32u + lane) : 0u;
        uint32_t h[4], g[4];
        bool v[4];
        block_hashes_groups<kBallots>(0u, size, w0, w1, h, v, g);
        for (uint32_t blk = 0; blk * 128u < size; ++blk) {
            const uint32_t nw = (blk + 2u) * 32u + lane;
            const uint32_t w2 = nw < nwords ? __ldg(src32 + nw) : 0u;
            // the next block's hashes and groups: no dependence on the table
            uint32_t hn[4], gn[4];
            bool vn[4];
            block_hashes_groups<kBallots>(blk + 1u, size, w1, w2, hn, vn, gn);
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j) {
                const uint32_t q = blk * 128u + j * 32u + lane;
                const uint32_t tv = v[j] ? static_cast<uint32_t>(T[h[j]]) : 0xFFFFu;
                __syncwarp();
                if (v[j] && !(g[j] & gt)) T[h[j]] = static_cast<uint16_t>(q);
                __syncwarp();
                const uint32_t lower = g[j] & lt;
                const uint32_t c = lower ? (q - lane + 31u - static_cast<uint32_t>(__clz(lower))) : tv;
                if (q < size) out[q] = static_cast<uint16_t>(c);
            }
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j) {
                h[j] = hn[j];
                v[j] = vn[j];
                g[j] = gn[j];
            }
            w0 = w1;
            w1 = w2;
        }
        __syncwarp();
    }
}

}  // namespace

namespace {
template <int kWarps, int kMode, uint32_t kPf = 0>
cudaError_t launch_sweep_variant(const SweepArgs &a, int num_sms, cudaStream_t st) {
    constexpr bool kBallots = (kMode & 1) != 0, kAhead = kMode >= 2;
    const auto kernel =
        kAhead ? cand_sweep_ahead_kernel<kWarps, kBallots> : cand_sweep_kernel<kWarps, kBallots, kAhead ? 0u : kPf>;
    const uint32_t smem = kWarps * kHashSize * sizeof(uint16_t);
    static SmemOnce smem_set{0};
    cudaError_t e = set_smem_once(kernel, smem, smem_set);
    if (e != cudaSuccess) return e;
    // as many CTAs per SM as the tables allow (one for 5-7 warps, two for 4 or less)
    const uint32_t per_sm = (227u * 1024u) / (smem + 1024u);
    uint32_t ctas = (a.num_windows + kWarps - 1) / kWarps;
    const uint32_t cap = static_cast<uint32_t>(num_sms) * (per_sm ? per_sm : 1u);
    if (ctas > cap) ctas = cap;
    kernel<<<ctas, 32 * kWarps, smem, st>>>(a);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_cand_sweep(const uint8_t *src, uint64_t n, uint32_t window, uint32_t num_windows, uint16_t *cand,
                              int num_sms, cudaStream_t st, const WinDesc *wins, int sweep_warps, int sweep_groups,
                              int sweep_prefetch) {
    if (num_windows == 0) return cudaSuccess;
    SweepArgs a{src, n, window, num_windows, cand, wins};
    // sweep_groups: 0 / 1 group equal-hash lanes (__match_any_sync / ballots)
    // only in blocks that need it, after a read-back; 2 / 3 form every step's
    // groups one block ahead.  sweep_prefetch: the read-back modes' L2
    // prefetch distance of the input, 0, 4 or 8 128-byte blocks (other values
    // are rounded down to one of these).
    const int pf = sweep_groups >= 2 ? 0 : (sweep_prefetch >= 8 ? 2 : (sweep_prefetch >= 4 ? 1 : 0));
    switch ((pf * 4 + sweep_groups) * 8 + sweep_warps) {
#define GCZ_SWEEP_CASE(P, M, W) \
    case (P * 4 + M) * 8 + W: return launch_sweep_variant<W, M, P * 4u>(a, num_sms, st);
#define GCZ_SWEEP_MODE(P, M) \
    GCZ_SWEEP_CASE(P, M, 4) GCZ_SWEEP_CASE(P, M, 5) GCZ_SWEEP_CASE(P, M, 6) GCZ_SWEEP_CASE(P, M, 7)
        GCZ_SWEEP_MODE(0, 0) GCZ_SWEEP_MODE(0, 1) GCZ_SWEEP_MODE(0, 2) GCZ_SWEEP_MODE(0, 3)
        GCZ_SWEEP_MODE(1, 0) GCZ_SWEEP_MODE(1, 1) GCZ_SWEEP_MODE(2, 0) GCZ_SWEEP_MODE(2, 1)
#undef GCZ_SWEEP_MODE
#undef GCZ_SWEEP_CASE
    default: return launch_sweep_variant<7, 0, 8u>(a, num_sms, st);
    }
}

}  // namespace gcz
