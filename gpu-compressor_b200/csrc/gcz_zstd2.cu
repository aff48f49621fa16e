// Zstd L1/L2 match finder, second stage: verification and parse.
//
// Input: the window bytes and cand(q) from the candidate sweep
// (gcz_sweep.cu).  Output: the exact sequence list of zstd_match_find
// (zstd_compress.cu:179-355) for every window.
//
// 1. The window is staged into shared memory with 1-D bulk copies.  Every
//    position's hash candidate (empty == position 0, :195-200) is verified on
//    3 bytes (:241-246) and the results form a bitmap.
// 2. Parse.  The reference parse is a deterministic state machine over
//    (pos, rep0, rep1, rep2): the next match and the next state depend on
//    nothing else.  The window is cut into 1 KiB segments, one lane each.
//    Every lane parses its segment from a guessed state (the segment start,
//    repeat offsets {1,4,8}); lane 0's guess is the true initial state.  Then
//    each lane keeps parsing past its segment end, and as soon as one of its
//    matches equals a match of a later lane's list -- same start, length and
//    offset, and the same repeat offsets afterwards -- both parses are in the
//    same state and stay identical, so that later list is exact from there on.
//    A chain walk from lane 0 then picks, in order: lane 0's list, its
//    continuation up to the meeting point, the met lane's list from there,
//    and so on.  Every lane on the chain is exact by induction.  Matches are
//    found per lane with the bitmap (hash matches) and word-wise byte
//    compares for the three repeat offsets (:259-275), so a lane skips up to
//    32 literal positions per step.
// 3. The chain is written as packed {ll | (ml-3) << 16, off} (or the
//    reference's {ll, ml-3, off} triples) at the per-window stride, capped at
//    max_seqs exactly like the reference's `num_seqs < max_sequences_per_chunk`
//    test (:309): the capped parse emits the first max_seqs matches of the
//    uncapped one and nothing after them.
// If a continuation does not meet a later list within kContCap matches the
// CTA falls back to an exact warp-wide parse of the whole window.
#include <type_traits>

#include "gcz_common.cuh"
#include "gcz_kernels.h"

namespace gcz {
namespace {

constexpr uint32_t kMinMatch = 3;                // MIN_MATCH_LEN, zstd_compress.cu:28
constexpr uint32_t kSeg = 1024;                  // bytes per speculative segment
constexpr uint32_t kLanes = kMaxWindow / kSeg;   // 64 segments per full window
constexpr uint32_t kThreads = 256;               // verification uses all 8 warps
// A segment's own parse starts matches in [seg_start, seg_end + 32) (the last
// step may look 31 positions ahead, the lazy step one more); matches are >= 3 bytes.
constexpr uint32_t kSpecCap = kSeg / 3 + 16;
constexpr uint32_t kContCap = 96;                // continuation matches before giving up
constexpr uint32_t kLaneCap = kSpecCap + kContCap;
constexpr uint32_t kNoLane = 0xFFFFu;

constexpr uint32_t kPre = 64;                           // zero bytes before the window
constexpr uint32_t kDataBytes = kPre + kMaxWindow + 64; // + zero pad after it
constexpr uint32_t kBmWords = kMaxWindow / 32 + 2;

struct SmemLayout {
    uint8_t data[kDataBytes];
    uint32_t bm[kBmWords];
    uint32_t spec_count[kLanes];
    uint32_t cont_count[kLanes];
    uint32_t sync_lane[kLanes];
    uint32_t sync_idx[kLanes];
    uint32_t chain_from[kLanes];
    uint32_t out_off[kLanes];
    uint32_t on_chain[kLanes];
    uint32_t ends[kThreads];
    uint32_t carry;
    uint32_t flags;
    uint32_t total;
    uint32_t covered;
    alignas(8) uint64_t bar;
};

struct Zstd2Args {
    const uint8_t *src;
    const uint16_t *cand;
    uint64_t n;
    uint32_t window;
    uint32_t num_windows;
    uint32_t lazy;
    uint32_t max_seqs;
    uint2 *seg;          // per window: kLanes * kLaneCap entries {start | (ml-3)<<16, off}
    uint2 *packed;       // packed output at stride max_seqs (or null)
    uint32_t *ref_seqs;  // reference triples at stride max_seqs (or null)
    uint32_t *seq_counts;
    uint32_t *lit_counts;
    uint32_t *status;
};

// ---------------------------------------------------------------- helpers
struct Win {
    const uint8_t *d;  // window byte 0 (kPre zero bytes before it in shared memory)
    __device__ __forceinline__ uint32_t u32(int q) const {
        const uint32_t *w = reinterpret_cast<const uint32_t *>(d - kPre);
        const uint32_t a = static_cast<uint32_t>(q + static_cast<int>(kPre));
        return __funnelshift_r(w[a >> 2], w[(a >> 2) + 1], (a & 3u) * 8u);
    }
};

// Aligned word stream over the staged window: next() returns the 4 bytes at
// the current position and advances by 4, with one shared-memory load and one
// funnel shift per call.
struct Stream {
    const uint32_t *w;
    uint32_t j, sh, cur;
    __device__ __forceinline__ Stream(const Win &win, int pos) {
        w = reinterpret_cast<const uint32_t *>(win.d - kPre);
        const uint32_t a = static_cast<uint32_t>(pos + static_cast<int>(kPre));
        j = a >> 2;
        sh = (a & 3u) * 8u;
        cur = w[j];
    }
    __device__ __forceinline__ uint32_t next() {
        const uint32_t nx = w[++j];
        const uint32_t v = __funnelshift_r(cur, nx, sh);
        cur = nx;
        return v;
    }
};

// First index in [0, lim) where bytes c+i and q+i differ, else lim.
__device__ __forceinline__ uint32_t extend(const Win &win, uint32_t c, uint32_t q, uint32_t lim) {
    Stream sc(win, static_cast<int>(c)), sq(win, static_cast<int>(q));
    uint32_t len = 0;
    while (len < lim) {
        const uint32_t d = sq.next() ^ sc.next();
        if (d) {
            len += (static_cast<uint32_t>(__ffs(d)) - 1u) >> 3;
            return len < lim ? len : lim;
        }
        len += 4u;
    }
    return lim;
}

__device__ __forceinline__ bool eq3(const Win &w, uint32_t a, uint32_t b) {
    return ((w.u32(static_cast<int>(a)) ^ w.u32(static_cast<int>(b))) & 0xFFFFFFu) == 0u;
}

// 0x80 in every byte of x that is zero.
__device__ __forceinline__ uint32_t zero_bytes(uint32_t x) {
    return ~(((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x) & 0x80808080u;
}

// Positions k+j (j < 4) of a 4-position chunk where offset d is usable
// (d <= p+k+j), as byte lanes: 0xFF per usable position.
__device__ __forceinline__ uint32_t usable(uint32_t d, uint32_t p, uint32_t k) {
    if (d <= p + k) return 0xFFFFFFFFu;
    const uint32_t v = d - p - k;  // first usable j
    return v >= 4u ? 0u : (0xFFFFFFFFu << (8u * v));
}

// Bit 8j+7: the 3 bytes at chunk position j are all zero in the xor stream
// whose zero-byte masks are z (this word) and y (next word).
__device__ __forceinline__ uint32_t three_equal(uint32_t z, uint32_t y) {
    return z & __funnelshift_r(z, y, 8) & __funnelshift_r(z, y, 16);
}

// First offset i in [0, n) (n <= 32) at which one of the repeat offsets d
// (d <= p+i) gives 3 equal bytes (src[p+i..p+i+2] == src[p+i-d..]), else n.
// Positions are examined 4 at a time and the search stops at the first hit.
__device__ __forceinline__ uint32_t rep_search(const Win &win, uint32_t p, uint32_t n, uint32_t r0, uint32_t r1,
                                               uint32_t r2) {
    if (n == 0) return 0;
    // offsets usable somewhere in [p, p+n), duplicates dropped
    const bool e0 = r0 < p + n;
    const bool e1 = r1 < p + n && r1 != r0;
    const bool e2 = r2 < p + n && r2 != r0 && r2 != r1;
    if (!(e0 || e1 || e2)) return n;
    Stream a(win, static_cast<int>(p));
    Stream b0(win, e0 ? static_cast<int>(p) - static_cast<int>(r0) : 0);
    Stream b1(win, e1 ? static_cast<int>(p) - static_cast<int>(r1) : 0);
    Stream b2(win, e2 ? static_cast<int>(p) - static_cast<int>(r2) : 0);
    const uint32_t A = a.next();
    uint32_t z0 = e0 ? zero_bytes(A ^ b0.next()) : 0u;
    uint32_t z1 = e1 ? zero_bytes(A ^ b1.next()) : 0u;
    uint32_t z2 = e2 ? zero_bytes(A ^ b2.next()) : 0u;
    uint32_t found = n;
    for (uint32_t k = 0; k < found; k += 4u) {
        const uint32_t A1 = a.next();
        uint32_t t = 0;
        if (e0) {
            const uint32_t y = zero_bytes(A1 ^ b0.next());
            t |= three_equal(z0, y) & usable(r0, p, k);
            z0 = y;
        }
        if (e1) {
            const uint32_t y = zero_bytes(A1 ^ b1.next());
            t |= three_equal(z1, y) & usable(r1, p, k);
            z1 = y;
        }
        if (e2) {
            const uint32_t y = zero_bytes(A1 ^ b2.next());
            t |= three_equal(z2, y) & usable(r2, p, k);
            z2 = y;
        }
        if (t) {
            const uint32_t i = k + ((static_cast<uint32_t>(__ffs(t)) - 1u) >> 3);
            if (i < found) found = i;
        }
    }
    return found;
}

struct PState {
    uint32_t p, r0, r1, r2;
};

struct Match {
    uint32_t start, len, off;
};

__device__ __forceinline__ uint32_t cand_at(const uint16_t *cand, uint32_t q) {
    const uint32_t c = cand[q];
    return c == 0xFFFFu ? 0u : c;  // empty table entry is position 0 in the Zstd kernel
}

__device__ __forceinline__ uint32_t bm_bit(const uint32_t *bm, uint32_t q) { return (bm[q >> 5] >> (q & 31u)) & 1u; }

// One step of the exact parse from state s (s.p + 3 < size): either finds the
// next match (returns true, s advanced past it, reps updated) or moves s.p
// over up to 32 literal positions (returns false).
__device__ __forceinline__ bool parse_step(const Win &w, const uint32_t *bm, const uint16_t *cand, uint32_t size,
                                           bool lazy, PState &s, Match &m) {
    const uint32_t p = s.p;
    const uint32_t lim = size - 3u - p;
    const uint32_t nscan = lim < 32u ? lim : 32u;
    uint32_t H = __funnelshift_r(bm[p >> 5], bm[(p >> 5) + 1], p & 31u);
    if (nscan < 32u) H &= (1u << nscan) - 1u;
    uint32_t f, off, len;
    bool hash;
    if (H & 1u) {
        f = p;
        hash = true;
    } else {
        const uint32_t n = H ? static_cast<uint32_t>(__ffs(H)) - 1u : nscan;  // positions without a hash match
        const uint32_t r = rep_search(w, p, n, s.r0, s.r1, s.r2);
        if (r < n) {
            f = p + r;
            hash = false;
        } else if (H) {
            f = p + n;
            hash = true;
        } else {
            s.p = p + nscan;
            return false;
        }
    }
    // Both candidates (f and f+1, for the lazy step) are loaded together.
    const uint32_t cf = cand_at(cand, f), cf1 = cand_at(cand, f + 1u);
    if (hash) {
        const uint32_t c = cf;
        off = f - c;
        len = extend(w, c + kMinMatch, f + kMinMatch, size - f - kMinMatch) + kMinMatch;
    } else {  // first repeat offset with 3 equal bytes wins (:259-275)
        if (s.r0 <= f && eq3(w, f, f - s.r0)) off = s.r0;
        else if (s.r1 <= f && eq3(w, f, f - s.r1)) off = s.r1;
        else off = s.r2;
        len = extend(w, f - off + kMinMatch, f + kMinMatch, size - f - kMinMatch) + kMinMatch;
    }
    if (lazy && f + 4u < size && bm_bit(bm, f + 1u)) {  // :278-307
        const uint32_t c1 = cf1;
        const uint32_t len2 =
            extend(w, c1 + kMinMatch, f + 1u + kMinMatch, size - f - 1u - kMinMatch) + kMinMatch;
        if (len2 > len + 1u) {
            f += 1u;
            len = len2;
            off = f - c1;
        }
    }
    m.start = f;
    m.len = len;
    m.off = off;
    s.r2 = s.r1;
    s.r1 = s.r0;
    s.r0 = off;
    s.p = f + len;
    return true;
}

__device__ __forceinline__ uint2 pack_entry(const Match &m) {
    return make_uint2(m.start | ((m.len - kMinMatch) << 16), m.off);
}

// Repeat offsets after entry j of a lane list whose parse started from {1,4,8}.
__device__ __forceinline__ void reps_after(const uint2 *list, uint32_t j, uint32_t &a, uint32_t &b, uint32_t &c) {
    a = list[j].y;
    b = j >= 1 ? list[j - 1].y : 1u;
    c = j >= 2 ? list[j - 2].y : (j == 1 ? 1u : 4u);
}

// ---------------------------------------------------------------- fallback
// Exact warp-wide parse of the whole window (warp 0): ballot over 32
// positions for literal runs, one match at a time.
template <class Emit>
__device__ void warp_parse(const Win &w, const uint32_t *bm, const uint16_t *cand, uint32_t size, bool lazy,
                           Emit emit) {
    const uint32_t lane = lane_id();
    uint32_t p = 0, r0 = 1, r1 = 4, r2 = 8, idx = 0;
    while (p + 3u < size) {
        const uint32_t B = p & ~31u;
        const uint32_t q = B + lane;
        const bool elig = q >= p && q + 3u < size;
        const uint32_t hb = __ballot_sync(kFull, elig && bm_bit(bm, q));
        const uint32_t fh = hb ? static_cast<uint32_t>(__ffs(hb)) - 1u : 32u;
        uint32_t rb = 0, rsel = 0;
        if (fh > p - B) {
            const bool need = elig && lane < fh;
            const bool a0 = need && r0 <= q && eq3(w, q, r0 <= q ? q - r0 : 0u);
            const bool a1 = need && !a0 && r1 <= q && eq3(w, q, r1 <= q ? q - r1 : 0u);
            const bool a2 = need && !a0 && !a1 && r2 <= q && eq3(w, q, r2 <= q ? q - r2 : 0u);
            rsel = a0 ? 0u : (a1 ? 1u : 2u);
            rb = __ballot_sync(kFull, a0 || a1 || a2);
        }
        const uint32_t b = hb | rb;
        if (!b) {
            p = B + 32u;
            continue;
        }
        const uint32_t f0 = static_cast<uint32_t>(__ffs(b)) - 1u;
        uint32_t f = B + f0, off, len;
        if ((hb >> f0) & 1u) {
            const uint32_t c = cand_at(cand, f);
            off = f - c;
            len = extend(w, c + kMinMatch, f + kMinMatch, size - f - kMinMatch) + kMinMatch;
        } else {
            const uint32_t r = __shfl_sync(kFull, rsel, f0);
            off = r == 0u ? r0 : (r == 1u ? r1 : r2);
            len = extend(w, f - off + kMinMatch, f + kMinMatch, size - f - kMinMatch) + kMinMatch;
        }
        if (lazy && f + 4u < size && bm_bit(bm, f + 1u)) {
            const uint32_t c1 = cand_at(cand, f + 1u);
            const uint32_t len2 =
                extend(w, c1 + kMinMatch, f + 1u + kMinMatch, size - f - 1u - kMinMatch) + kMinMatch;
            if (len2 > len + 1u) {
                f += 1u;
                len = len2;
                off = f - c1;
            }
        }
        if (lane == 0) emit(idx, f, len, off);
        ++idx;
        r2 = r1;
        r1 = r0;
        r0 = off;
        p = f + len;
    }
}

// ---------------------------------------------------------------- kernel
template <bool kRef>
__global__ void __launch_bounds__(kThreads) zstd_parse_kernel(Zstd2Args a) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    SmemLayout &S = *reinterpret_cast<SmemLayout *>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    uint32_t parity = 0;
    if (tid == 0) {
        mbar_init(&S.bar, 1);
        fence_mbar_init();
    }
    for (uint32_t i = tid; i < kPre / 4; i += kThreads) reinterpret_cast<uint32_t *>(S.data)[i] = 0u;
    __syncthreads();
    Win win{S.data + kPre};

    for (uint32_t wi = blockIdx.x; wi < a.num_windows; wi += gridDim.x) {
        const uint64_t start = static_cast<uint64_t>(wi) * a.window;
        const uint32_t size = static_cast<uint32_t>(a.n - start < a.window ? a.n - start : a.window);
        const uint16_t *cand = a.cand + start;
        uint2 *seg = a.seg + static_cast<uint64_t>(wi) * kLanes * kLaneCap;

        // ---- 1. stage the window (warp 0), verification bitmap (all warps)
        __syncthreads();  // previous window fully consumed
        if (tid == 0) {
            S.flags = 0;
            S.covered = 0;
        }
        __syncthreads();
        if (warp == 0) {
            if (!stage_window(S.data + kPre, a.src + start, size, &S.bar, parity, a.status) && lane == 0)
                S.flags = 2u;
        }
        __syncthreads();
        if (S.flags & 2u) return;  // bulk copy never completed: status already recorded, all threads leave
        const uint32_t nsteps = (size + 31u) >> 5;
        // Batches of kVB steps per warp: all kVB candidate loads are issued
        // before any is used, so one memory latency covers the batch.
        constexpr uint32_t kVB = 16;
        for (uint32_t b0 = warp * kVB; b0 < kBmWords; b0 += (kThreads / 32) * kVB) {
            uint32_t cv[kVB];
#pragma unroll
            for (uint32_t u = 0; u < kVB; ++u) {
                const uint32_t q = (b0 + u) * 32u + lane;
                cv[u] = (b0 + u < nsteps && q + 3u < size && q > 0u) ? static_cast<uint32_t>(cand[q]) : 0x10000u;
            }
#pragma unroll
            for (uint32_t u = 0; u < kVB; ++u) {
                const uint32_t st = b0 + u;
                const uint32_t q = st * 32u + lane;
                bool hm = false;
                if (cv[u] != 0x10000u) hm = eq3(win, q, cv[u] == 0xFFFFu ? 0u : cv[u]);
                const uint32_t bits = __ballot_sync(kFull, hm);
                if (lane == 0 && st < kBmWords) S.bm[st] = bits;
            }
        }
        __syncthreads();

        // ---- 2a. speculative parse of each segment
        const uint32_t nseg = (size + kSeg - 1u) / kSeg;
        const uint32_t lim_pos = size > 3u ? size - 3u : 0u;  // positions q < lim_pos can start a match
        uint2 *mine = seg + tid * kLaneCap;
        PState s{tid * kSeg, 1u, 4u, 8u};
        uint32_t nspec = 0;
        const bool active = tid < kLanes && tid < nseg && tid * kSeg < lim_pos;
        const uint32_t seg_end = (tid + 1u) * kSeg;
        const bool last_active = !((tid + 1u) < nseg && (tid + 1u) * kSeg < lim_pos);
        if (active) {
            const uint32_t stop = last_active ? size : seg_end;
            Match m;
            while (s.p < stop && s.p + 3u < size) {
                if (parse_step(win, S.bm, cand, size, a.lazy != 0, s, m)) {
                    mine[nspec++] = pack_entry(m);  // nspec <= kSpecCap: starts lie in one segment
                }
            }
        }
        if (tid < kLanes) {
            S.spec_count[tid] = nspec;
            S.cont_count[tid] = 0;
            S.sync_lane[tid] = kNoLane;
            S.sync_idx[tid] = 0;
        }
        __syncthreads();

        // ---- 2b. continue each lane's parse until it meets a later lane's list
        if (active && !last_active) {
            uint32_t t = kNoLane, j = 0, ncont = 0;
            bool synced = false;
            Match m;
            while (s.p + 3u < size) {
                if (!parse_step(win, S.bm, cand, size, a.lazy != 0, s, m)) continue;
                const uint32_t tl = m.start / kSeg;  // lane whose territory holds this match start
                if (tl != t) {
                    t = tl;
                    j = 0;
                }
                const uint32_t tcount = t < kLanes ? S.spec_count[t] : 0u;
                const uint2 *tl_list = seg + t * kLaneCap;
                while (j < tcount && (tl_list[j].x & 0xFFFFu) < m.start) ++j;
                if (j < tcount && tl_list[j].x == pack_entry(m).x && tl_list[j].y == m.off) {
                    uint32_t e0, e1, e2;
                    reps_after(tl_list, j, e0, e1, e2);
                    if (e0 == s.r0 && e1 == s.r1 && e2 == s.r2) {
                        S.sync_lane[tid] = t;
                        S.sync_idx[tid] = j;
                        synced = true;
                        break;
                    }
                }
                if (ncont == kContCap) {
                    atomicOr(&S.flags, 1u);  // give up: exact fallback below
                    break;
                }
                mine[kSpecCap + ncont++] = pack_entry(m);
            }
            S.cont_count[tid] = ncont;
            (void)synced;
        }
        __syncthreads();

        const bool fallback = (S.flags & 1u) != 0;
        uint32_t total = 0;
        if (!fallback) {
            // ---- 3. chain walk (one thread), then copy in chain order
            if (tid == 0) {
                for (uint32_t i = 0; i < kLanes; ++i) S.on_chain[i] = 0;
                uint32_t cur = 0, from = 0, acc = 0;
                if (nseg > 0 && lim_pos > 0) {
                    for (;;) {
                        S.on_chain[cur] = 1;
                        S.chain_from[cur] = from;
                        S.out_off[cur] = acc;
                        acc += (S.spec_count[cur] - from) + S.cont_count[cur];
                        const uint32_t nx = S.sync_lane[cur];
                        if (nx == kNoLane) break;
                        from = S.sync_idx[cur];
                        cur = nx;
                    }
                }
                S.total = acc;
            }
            __syncthreads();
            total = S.total;
            const uint32_t keep = total < a.max_seqs ? total : a.max_seqs;
            // Write {start, ml-3, off} in order; ll is filled in the next pass.
            if (tid < kLanes && S.on_chain[tid]) {
                uint32_t o = S.out_off[tid];
                const uint32_t from = S.chain_from[tid], ns = S.spec_count[tid], nc = S.cont_count[tid];
                uint32_t cov = 0;
                for (uint32_t i = from; i < ns + nc; ++i, ++o) {
                    const uint2 e = mine[i < ns ? i : kSpecCap + (i - ns)];
                    if (o < keep) {
                        cov += (e.x >> 16) + kMinMatch;
                        if constexpr (kRef) {
                            uint32_t *r = a.ref_seqs + (static_cast<uint64_t>(wi) * a.max_seqs + o) * 3u;
                            r[0] = e.x & 0xFFFFu;  // start for now
                            r[1] = e.x >> 16;
                            r[2] = e.y;
                        } else {
                            a.packed[static_cast<uint64_t>(wi) * a.max_seqs + o] = e;
                        }
                    }
                }
                if (cov) atomicAdd(&S.covered, cov);
            }
            __syncthreads();
            // start -> literal length: ll(o) = start(o) - end(o-1), chunk by chunk;
            // every entry is read (and its end shared) before any is rewritten.
            if (tid == 0) S.carry = 0;
            for (uint32_t base = 0; base < keep; base += kThreads) {
                const uint32_t o = base + tid;
                uint32_t st0 = 0, mlm3 = 0, off = 0;
                if (o < keep) {
                    if constexpr (kRef) {
                        const uint32_t *r = a.ref_seqs + (static_cast<uint64_t>(wi) * a.max_seqs + o) * 3u;
                        st0 = r[0];
                        mlm3 = r[1];
                        off = r[2];
                    } else {
                        const uint2 e = a.packed[static_cast<uint64_t>(wi) * a.max_seqs + o];
                        st0 = e.x & 0xFFFFu;
                        mlm3 = e.x >> 16;
                        off = e.y;
                    }
                }
                S.ends[tid] = st0 + mlm3 + kMinMatch;
                __syncthreads();
                const uint32_t prev_end = tid ? S.ends[tid - 1] : S.carry;
                const uint32_t last = (keep - base < kThreads ? keep - base : kThreads) - 1u;
                const uint32_t next_carry = S.ends[last];
                if (o < keep) {
                    const uint32_t ll = st0 - prev_end;
                    if constexpr (kRef) {
                        uint32_t *r = a.ref_seqs + (static_cast<uint64_t>(wi) * a.max_seqs + o) * 3u;
                        r[0] = ll;
                        r[1] = mlm3;
                        r[2] = off;
                    } else {
                        a.packed[static_cast<uint64_t>(wi) * a.max_seqs + o] = make_uint2(ll | (mlm3 << 16), off);
                    }
                }
                __syncthreads();
                if (tid == 0) S.carry = next_carry;
            }
            if (tid == 0) {
                a.seq_counts[wi] = keep;
                if (a.lit_counts) a.lit_counts[wi] = size - S.covered;
            }
        } else {
            // ---- exact warp-wide parse of the whole window
            if (warp == 0) {
                const uint32_t cap = a.max_seqs;
                uint32_t cov = 0, cnt = 0, prev_end = 0;
                auto emit = [&](uint32_t idx, uint32_t f, uint32_t len, uint32_t off) {
                    if (idx < cap) {
                        const uint32_t ll = f - prev_end;
                        if constexpr (kRef) {
                            uint32_t *r = a.ref_seqs + (static_cast<uint64_t>(wi) * a.max_seqs + idx) * 3u;
                            r[0] = ll;
                            r[1] = len - kMinMatch;
                            r[2] = off;
                        } else {
                            a.packed[static_cast<uint64_t>(wi) * a.max_seqs + idx] =
                                make_uint2(ll | ((len - kMinMatch) << 16), off);
                        }
                        cov += len;
                        cnt = idx + 1u;
                    }
                    prev_end = f + len;
                };
                warp_parse(win, S.bm, cand, size, a.lazy != 0, emit);
                if (lane == 0) {
                    a.seq_counts[wi] = cnt;
                    if (a.lit_counts) a.lit_counts[wi] = size - cov;
                    atomicAdd(a.status + 1, 1u);  // fallback counter (diagnostics)
                }
            }
        }
    }
}

}  // namespace

size_t zstd2_seg_scratch_entries(uint32_t num_windows) {
    return static_cast<size_t>(num_windows) * kLanes * kLaneCap;
}

cudaError_t launch_zstd_parse(const Zstd2Launch &l, cudaStream_t st) {
    if (l.num_windows == 0) return cudaSuccess;
    Zstd2Args a{};
    a.src = l.src;
    a.cand = l.cand;
    a.n = l.n;
    a.window = l.window;
    a.num_windows = l.num_windows;
    a.lazy = l.search_depth > 1 ? 1u : 0u;
    a.max_seqs = l.max_seqs;
    a.seg = reinterpret_cast<uint2 *>(l.seg);
    a.packed = reinterpret_cast<uint2 *>(l.packed);
    a.ref_seqs = l.ref_seqs;
    a.seq_counts = l.seq_counts;
    a.lit_counts = l.lit_counts;
    a.status = l.status;
    const uint32_t smem = sizeof(SmemLayout);
    int grid = l.num_sms * l.ctas_per_sm;
    if (static_cast<uint32_t>(grid) > l.num_windows) grid = static_cast<int>(l.num_windows);
    cudaError_t e;
    if (l.ref_seqs) {
        e = cudaFuncSetAttribute(zstd_parse_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        zstd_parse_kernel<true><<<grid, kThreads, smem, st>>>(a);
    } else {
        e = cudaFuncSetAttribute(zstd_parse_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        zstd_parse_kernel<false><<<grid, kThreads, smem, st>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace gcz
