// Zstd L1/L2 match finder, second stage: verification and parse.
//
// Input: the window bytes and cand(q) from the candidate sweep
// (gcz_sweep.cu).  Output: the exact sequence list of zstd_match_find
// (zstd_compress.cu:179-355) for every window.
//
// 1. The window is staged into shared memory with 1-D bulk copies.  Every
//    position's hash candidate (empty == position 0, :195-200) is verified on
//    3 bytes (:241-246); the results form a bitmap.
// 2. Parse.  The reference parse is a deterministic state machine over
//    (pos, rep0, rep1, rep2): the next match and the next state depend on
//    nothing else.  The window is cut into 4 KiB segments, one warp each.
//    Every warp parses its segment from a guessed state (the segment start,
//    repeat offsets {1,4,8}); warp 0's guess is the true initial state.  Then
//    each warp keeps parsing past its segment end, and as soon as one of its
//    matches equals a match of a later warp's list -- same start, length and
//    offset, and the same repeat offsets afterwards -- both parses are in the
//    same state and stay identical, so that later list is exact from there on.
//    A chain walk from warp 0 then picks, in order: warp 0's list, its
//    continuation up to the meeting point, the met warp's list from there, and
//    so on; every list on the chain is exact by induction.  (On the synthetic
//    workload a guessed parse meets the true one after ~180 bytes, three
//    matches, so the overlap costs ~4% extra parse work.)
//    Each warp parses like the reference, one match at a time, but with all
//    32 lanes: the hash-match bits of the next positions come from the
//    bitmap, the lanes test the three repeat offsets (:259-275) on the
//    positions before the first hash match -- one (position, offset) pair per
//    lane when there are at most 10 of them, one position per lane up to 32,
//    and four positions per lane (8-byte compares) over up to 128 positions
//    that hold no hash match -- a ballot finds the first event, matches are
//    extended 128 bytes per warp iteration, and one lazy step (:278-307)
//    follows.
// 3. The chain is written in one pass as packed {ll | (ml-3) << 16, off} (or
//    the reference's {ll, ml-3, off} triples) at the per-window stride, each
//    literal length taken from the entry before it, capped at
//    max_seqs exactly like the reference's `num_seqs < max_sequences_per_chunk`
//    test (:309): the capped parse emits the first max_seqs matches of the
//    uncapped one and nothing after them.
// In the 8- and 4-lane group layouts, once only one group of a warp is still
// continuing, the whole warp finishes that continuation with warp-wide steps.
// If a continuation does not meet a later list within kContCap matches the
// CTA falls back to an exact warp-wide parse of the whole window.
#include <type_traits>

#include "gcz_common.cuh"
#include "gcz_kernels.h"

namespace gcz {
namespace {

constexpr uint32_t kMinMatch = 3;                 // MIN_MATCH_LEN, zstd_compress.cu:28
// Speculative segment width is a schedule knob: 2, 4 or 8 KiB parsed by one
// warp each (32, 16 or 8 warps per window), 1 KiB parsed by an 8-lane group
// (four segments per warp, 64 per window), or 512 bytes parsed by a 4-lane
// group (eight segments per warp, 128 per window).  It never changes the
// sequences.
template <uint32_t SegW, uint32_t GL = 32>
struct SegCfg {
    static constexpr uint32_t kSegW = SegW;
    static constexpr uint32_t kSegs = kMaxWindow / SegW;
    static constexpr uint32_t kThreads = kSegs * GL;
    static constexpr uint32_t kWarps = kThreads / 32;
    // A segment's own parse ends with a step that starts before seg_end and
    // looks at most kLook positions ahead (a warp's wide scan 128, a group's
    // scan 32), the lazy step one more; matches do not overlap and are >= 3
    // bytes, so a list holds at most (SegW + kLook) / 3 + 1 entries; lists are
    // written in 32-entry blocks.
    static constexpr uint32_t kLook = GL == 32 ? 128 : 32;
    static constexpr uint32_t kSpecCap = ((SegW + kLook) / 3 + 1 + 31) / 32 * 32;
    // continuation matches before giving up (a guessed parse meets the true
    // one after ~3 matches; the cap keeps every layout's lists within the
    // 1 KiB layout's 32768 entries per window)
    static constexpr uint32_t kContCap = GL == 32 ? 256 : (GL == 8 ? 128 : 64);
    static constexpr uint32_t kLaneCap = kSpecCap + kContCap;
    static constexpr uint32_t kMinBlocks = kThreads >= 1024 ? 1 : 3;
};
constexpr uint32_t kNoWarp = 0xFFFFu;
constexpr uint32_t kNoEntry = 0xFFFFu;

constexpr uint32_t kPre = 64;                           // zero bytes before the window
constexpr uint32_t kDataBytes = kPre + kMaxWindow + 64; // + zero pad after it
constexpr uint32_t kBmWords = kMaxWindow / 32 + 8;  // the wide scan reads up to 4 words past a step's first

template <uint32_t kSegs>
struct SmemLayout {
    uint8_t data[kDataBytes];
    uint32_t bm[kBmWords];
    // Per segment, 16 bits each (list lengths, indices and output offsets of
    // a window are below 2^15; segment indices below 2^7), so that 128
    // segments fit beside the window at three CTAs per SM.
    uint16_t spec_count[kSegs];
    uint16_t cont_count[kSegs];
    uint16_t sync_warp[kSegs];
    uint16_t sync_idx[kSegs];
    uint16_t chain_from[kSegs];
    uint16_t out_off[kSegs];
    uint16_t on_chain[kSegs];
    uint16_t prev_last[kSegs];  // seg index of the entry before a chain segment's first copied one (kNoEntry: none)
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
    uint2 *seg;          // per window: kSegs * kLaneCap entries {start | (ml-3)<<16, off} (the widest layout's stride)
    uint2 *packed;       // packed output at stride max_seqs (or null)
    uint32_t *ref_seqs;  // reference triples at stride max_seqs (or null)
    uint32_t *seq_counts;
    uint32_t *lit_counts;
    uint32_t *status;
    const WinDesc *wins;
    uint32_t seg_stride;  // seg entries per window
};

// ---------------------------------------------------------------- helpers
struct Win {
    const uint8_t *d;  // window byte 0 (kPre zero bytes before it in shared memory)
    __device__ __forceinline__ uint32_t u32(int q) const {
        const uint32_t *w = reinterpret_cast<const uint32_t *>(d - kPre);
        const uint32_t a = static_cast<uint32_t>(q + static_cast<int>(kPre));
        return __funnelshift_r(w[a >> 2], w[(a >> 2) + 1], (a & 3u) * 8u);
    }
    // The 4 bytes at q, q a multiple of 4.
    __device__ __forceinline__ uint32_t w32(uint32_t q) const { return reinterpret_cast<const uint32_t *>(d)[q >> 2]; }
    // The 8 bytes at q: three aligned words, two funnel shifts.
    __device__ __forceinline__ void u64(int q, uint32_t &lo, uint32_t &hi) const {
        const uint32_t *w = reinterpret_cast<const uint32_t *>(d - kPre);
        const uint32_t a = static_cast<uint32_t>(q + static_cast<int>(kPre));
        const uint32_t i = a >> 2, sh = (a & 3u) * 8u;
        const uint32_t w1 = w[i + 1];
        lo = __funnelshift_r(w[i], w1, sh);
        hi = __funnelshift_r(w1, w[i + 2], sh);
    }
};

// First index in [0, lim) where bytes c+i and q+i differ, else lim.
// Warp-cooperative (all lanes call it with the same arguments): each lane
// compares 4 bytes, 128 bytes per iteration.
__device__ __forceinline__ uint32_t extend_warp(const Win &w, uint32_t c, uint32_t q, uint32_t lim) {
    const uint32_t lane = lane_id();
    uint32_t len = 0;
    for (;;) {
        const uint32_t k = len + 4u * lane;
        uint32_t res = k;
        if (k < lim) {
            const uint32_t d = w.u32(static_cast<int>(q + k)) ^ w.u32(static_cast<int>(c + k));
            const uint32_t fb = d ? (static_cast<uint32_t>(__ffs(d)) - 1u) >> 3 : 4u;
            const uint32_t rem = lim - k;
            res = k + (fb < rem ? fb : rem);
        }
        const uint32_t sb = __ballot_sync(kFull, res < k + 4u);
        if (sb) return __shfl_sync(kFull, res, __ffs(sb) - 1);
        len += 128u;
    }
}

// Two extensions at once: lanes 0-15 extend (ca, qa) up to la, lanes 16-31
// extend (cb, qb) up to lb, 64 bytes per half per iteration.
__device__ __forceinline__ void extend_pair(const Win &w, uint32_t ca, uint32_t qa, uint32_t la, uint32_t cb,
                                            uint32_t qb, uint32_t lb, uint32_t &ra, uint32_t &rb) {
    const uint32_t lane = lane_id(), half = lane >> 4, hl = lane & 15u;
    const uint32_t c = half ? cb : ca, q = half ? qb : qa, lim = half ? lb : la;
    bool da = false, db = false;
    ra = 0;
    rb = 0;
    for (uint32_t len = 0;; len += 64u) {
        const uint32_t k = len + 4u * hl;
        uint32_t res = k;
        if (k < lim) {
            const uint32_t d = w.u32(static_cast<int>(q + k)) ^ w.u32(static_cast<int>(c + k));
            const uint32_t fb = d ? (static_cast<uint32_t>(__ffs(d)) - 1u) >> 3 : 4u;
            const uint32_t rem = lim - k;
            res = k + (fb < rem ? fb : rem);
        }
        const uint32_t sb = __ballot_sync(kFull, res < k + 4u);
        const uint32_t sa = sb & 0xFFFFu, sbb = sb >> 16;
        const uint32_t va = __shfl_sync(kFull, res, sa ? __ffs(sa) - 1 : 0);
        const uint32_t vb = __shfl_sync(kFull, res, sbb ? 16 + __ffs(sbb) - 1 : 16);
        if (!da && sa) {
            ra = va;
            da = true;
        }
        if (!db && sbb) {
            rb = vb;
            db = true;
        }
        if (da && db) return;
    }
}

// Rolling register buffer of candidates for one warp: lane l holds
// cand[base + l], cand[base + 32 + l] and cand[base + 64 + l] (the third block
// is a prefetch), base 32-aligned.
struct CandBuf {
    const uint16_t *cand;
    uint32_t size, base, c0, c1, c2;
    __device__ __forceinline__ uint32_t ld(uint32_t pos) const {
        return pos < size ? static_cast<uint32_t>(cand[pos]) : 0u;
    }
    __device__ __forceinline__ void init(uint32_t p) {
        const uint32_t lane = lane_id();
        base = p & ~31u;
        c0 = ld(base + lane);
        c1 = ld(base + 32u + lane);
        c2 = ld(base + 64u + lane);
    }
    // Make positions [p, p+33) available (p uniform).
    __device__ __forceinline__ void advance(uint32_t p) {
        const uint32_t nb = p & ~31u, lane = lane_id();
        if (nb == base) return;
        if (nb == base + 32u) {
            c0 = c1;
            c1 = c2;
            c2 = ld(nb + 64u + lane);
        } else if (nb == base + 64u) {
            c0 = c2;
            c1 = ld(nb + 32u + lane);
            c2 = ld(nb + 64u + lane);
        } else {
            init(p);
            return;
        }
        base = nb;
    }
    // cand[pos] for pos in [base, base+96) (pos uniform).
    __device__ __forceinline__ uint32_t get(uint32_t pos) const {
        const uint32_t k = pos - base;
        const uint32_t r = k < 32u ? c0 : (k < 64u ? c1 : c2);
        return __shfl_sync(kFull, r, k & 31u);
    }
};

__device__ __forceinline__ bool eq3(const Win &w, uint32_t a, uint32_t b) {
    return ((w.u32(static_cast<int>(a)) ^ w.u32(static_cast<int>(b))) & 0xFFFFFFu) == 0u;
}

__device__ __forceinline__ uint32_t bm_bit(const uint32_t *bm, uint32_t q) { return (bm[q >> 5] >> (q & 31u)) & 1u; }

__device__ __forceinline__ uint32_t zmap(uint32_t c) { return c == 0xFFFFu ? 0u : c; }  // empty entry = position 0

struct PState {
    uint32_t p, r0, r1, r2;
};

struct Match {
    uint32_t start, len, off;
};

// One warp-uniform step of the exact parse from state s (s.p + 3 < size):
// either finds the next match (returns true, s advanced past it, repeat
// offsets updated) or moves s.p over up to 32 literal positions.
__device__ __forceinline__ bool warp_step(const Win &w, const uint32_t *bm, CandBuf &cb, uint32_t size, bool lazy,
                                          PState &s, Match &m) {
    const uint32_t lane = lane_id();
    const uint32_t p = s.p;
    const uint32_t lim = size - 3u - p;
    const uint32_t nscan = lim < 32u ? lim : 32u;
    uint32_t H = __funnelshift_r(bm[p >> 5], bm[(p >> 5) + 1], p & 31u);
    if (nscan < 32u) H &= (1u << nscan) - 1u;
    const uint32_t q = p + lane;
    cb.advance(p);  // candidates of p .. p+32 (and the next block in flight)
    uint32_t f, r = 0;  // event position; for a repeat-offset match, which repeat offset (0-2)
    bool hash;
    if (H & 1u) {
        f = p;
        hash = true;
    } else {
        // Repeat offsets are tried only at positions without a hash match, in
        // order r0, r1, r2, and the first position with a hit wins
        // (zstd_compress.cu:259-275).  How the lanes share the tests depends
        // on how many positions come before the first hash match.
        const uint32_t n = H ? static_cast<uint32_t>(__ffs(H)) - 1u : nscan;  // positions without a hash match
        if (n <= 10u) {
            // Few positions: one (position, repeat offset) pair per lane, in
            // position-major order, so the first set ballot bit is the event.
            const uint32_t i = lane / 3u, k = lane - 3u * i;
            const uint32_t rv = k == 0u ? s.r0 : (k == 1u ? s.r1 : s.r2);
            const uint32_t qq = p + i;
            const bool hit = i < n && rv <= qq && eq3(w, qq, rv <= qq ? qq - rv : qq);
            const uint32_t rb = __ballot_sync(kFull, hit);
            if (rb) {
                const uint32_t l = static_cast<uint32_t>(__ffs(rb)) - 1u;
                f = p + l / 3u;
                r = l % 3u;
                hash = false;
            } else if (H) {
                f = p + n;
                hash = true;
            } else {
                s.p = p + nscan;
                return false;
            }
        } else if (H == 0u && lim > 32u) {
            // No hash match in 32 positions: scan up to 128, four positions
            // per lane, each repeat offset tested on 8-byte words.
            const uint32_t n4s = lim < 128u ? lim : 128u;
            const uint32_t wi = p >> 5, sh = p & 31u;
            uint32_t n4 = n4s;
#pragma unroll
            for (uint32_t k = 3; k >= 1; --k) {
                const uint32_t hk = __funnelshift_r(bm[wi + k], bm[wi + k + 1u], sh);
                if (hk) n4 = 32u * k + static_cast<uint32_t>(__ffs(hk)) - 1u;
            }
            if (n4 > n4s) n4 = n4s;
            const uint32_t j0 = 4u * lane;  // this lane's first position index
            const uint32_t q0 = j0 < n4 ? p + j0 : p;
            const uint32_t vlim = j0 < n4 ? (n4 - j0 < 4u ? n4 - j0 : 4u) : 0u;  // positions of this lane to test
            const uint32_t xlo = w.u32(static_cast<int>(q0)), xhi = w.u32(static_cast<int>(q0 + 4u));
            uint32_t mk[3];
#pragma unroll
            for (uint32_t k = 0; k < 3; ++k) {
                const uint32_t rv = k == 0u ? s.r0 : (k == 1u ? s.r1 : s.r2);
                // positions q0 + t with t < vlim and q0 + t >= rv; their source bytes start at q0 - rv + t >= 0
                const uint32_t tmin = rv > q0 ? rv - q0 : 0u;
                uint32_t valid = tmin < vlim ? ((1u << vlim) - 1u) & ~((1u << tmin) - 1u) : 0u;
                const int yb = valid ? static_cast<int>(q0) - static_cast<int>(rv) : static_cast<int>(q0);
                const uint32_t dlo = xlo ^ w.u32(yb), dhi = xhi ^ w.u32(yb + 4);
                const uint32_t e = ((dlo & 0xFFFFFFu) == 0u ? 1u : 0u) | ((dlo >> 8) == 0u ? 2u : 0u) |
                                   ((__funnelshift_r(dlo, dhi, 16) & 0xFFFFFFu) == 0u ? 4u : 0u) |
                                   ((__funnelshift_r(dlo, dhi, 24) & 0xFFFFFFu) == 0u ? 8u : 0u);
                mk[k] = e & valid;
            }
            const uint32_t any = mk[0] | mk[1] | mk[2];
            const uint32_t rb = __ballot_sync(kFull, any != 0u);
            if (rb) {
                const uint32_t l = static_cast<uint32_t>(__ffs(rb)) - 1u;
                const uint32_t al = __shfl_sync(kFull, any, l), m0 = __shfl_sync(kFull, mk[0], l),
                               m1 = __shfl_sync(kFull, mk[1], l);
                const uint32_t t = static_cast<uint32_t>(__ffs(al)) - 1u;
                f = p + 4u * l + t;
                r = (m0 >> t) & 1u ? 0u : ((m1 >> t) & 1u ? 1u : 2u);
                hash = false;
            } else if (n4 < n4s) {
                f = p + n4;
                hash = true;
            } else {
                s.p = p + n4s;
                return false;
            }
        } else {
            const bool need = lane < n;
            const uint32_t x = w.u32(static_cast<int>(q));
            const bool a0 =
                need && s.r0 <= q && ((x ^ w.u32(static_cast<int>(s.r0 <= q ? q - s.r0 : 0u))) & 0xFFFFFFu) == 0u;
            const bool a1 = need && !a0 && s.r1 <= q &&
                            ((x ^ w.u32(static_cast<int>(s.r1 <= q ? q - s.r1 : 0u))) & 0xFFFFFFu) == 0u;
            const bool a2 = need && !a0 && !a1 && s.r2 <= q &&
                            ((x ^ w.u32(static_cast<int>(s.r2 <= q ? q - s.r2 : 0u))) & 0xFFFFFFu) == 0u;
            const uint32_t rsel = a0 ? 0u : (a1 ? 1u : 2u);
            const uint32_t rb = __ballot_sync(kFull, a0 || a1 || a2);
            if (rb) {
                const uint32_t l = static_cast<uint32_t>(__ffs(rb)) - 1u;
                f = p + l;
                r = __shfl_sync(kFull, rsel, l);
                hash = false;
            } else if (H) {
                f = p + n;
                hash = true;
            } else {
                s.p = p + nscan;
                return false;
            }
        }
    }
    cb.advance(f);  // a wide scan's event can lie past the buffer
    const uint32_t cf = zmap(cb.get(f));
    const uint32_t cf1 = zmap(cb.get(f + 1u));
    uint32_t off, c0;
    if (hash) {
        off = f - cf;
        c0 = cf;
    } else {  // first repeat offset with 3 equal bytes wins
        off = r == 0u ? s.r0 : (r == 1u ? s.r1 : s.r2);
        c0 = f - off;
    }
    uint32_t len;
    // The lazy candidate at f+1 (zstd_compress.cu:278-307) is taken only when
    // len2 > len + 1.  When it is the same match one byte on (cand(f+1) ==
    // c0 + 1) it is exactly one byte shorter -- its 3 verified bytes include
    // byte f+3 == c0+3, so the main match extends past 3 -- and is never taken.
    if (lazy && f + 4u < size && bm_bit(bm, f + 1u) && cf1 != c0 + 1u) {  // main match and lazy candidate together
        uint32_t l1, l2;
        extend_pair(w, c0 + kMinMatch, f + kMinMatch, size - f - kMinMatch, cf1 + kMinMatch, f + 1u + kMinMatch,
                    size - f - 1u - kMinMatch, l1, l2);
        len = l1 + kMinMatch;
        const uint32_t len2 = l2 + kMinMatch;
        if (len2 > len + 1u) {
            f += 1u;
            len = len2;
            off = f - cf1;
        }
    } else {
        len = extend_warp(w, c0 + kMinMatch, f + kMinMatch, size - f - kMinMatch) + kMinMatch;
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

// Group-wide extension: the lanes of each GL-lane group compare 4 bytes each
// (4 * GL per iteration) of their group's own (c, q, lim) and get the first
// index in [0, lim) where bytes c+i and q+i differ, else lim; groups with
// act == false get 0.  All 32 lanes call it (the loop runs while any group
// is still extending).
template <uint32_t GL>
__device__ __forceinline__ uint32_t extend_group(const Win &w, uint32_t c, uint32_t q, uint32_t lim, bool act) {
    const uint32_t lane = lane_id(), gl = lane & (GL - 1u), gb = lane & ~(GL - 1u);
    uint32_t len = 0, out = 0;
    bool done = !act;
    while (__any_sync(kFull, !done)) {
        const uint32_t k = len + 8u * gl;  // 8 bytes per lane
        uint32_t res = k;
        if (!done && k < lim) {
            uint32_t ql, qh, cl, ch;
            w.u64(static_cast<int>(q + k), ql, qh);
            w.u64(static_cast<int>(c + k), cl, ch);
            const uint32_t dl = ql ^ cl, dh = qh ^ ch;
            const uint32_t fb = dl ? (static_cast<uint32_t>(__ffs(dl)) - 1u) >> 3
                                   : (dh ? 4u + ((static_cast<uint32_t>(__ffs(dh)) - 1u) >> 3) : 8u);
            const uint32_t rem = lim - k;
            res = k + (fb < rem ? fb : rem);
        }
        const uint32_t sb = (__ballot_sync(kFull, !done && res < k + 8u) >> gb) & ((1u << GL) - 1u);
        const uint32_t v = __shfl_sync(kFull, res, gb + (sb ? static_cast<uint32_t>(__ffs(sb)) - 1u : 0u));
        if (!done && sb) {
            out = v;
            done = true;
        }
        len += 8u * GL;
    }
    return out;
}

// Bit t (t < 16) set when bytes q+t .. q+t+2 equal bytes q-r+t .. q-r+t+2
// (zstd_compress.cu:259-275 tests one position at a time).  Both 18-byte
// ranges are read as aligned words; a byte of x ^ y is zero exactly when its
// 0x80 flag survives ~(((d & 0x7F..) + 0x7F..) | d | 0x7F..), three flags in
// a row mark a 3-byte match, and a multiply gathers each word's four flags.
__device__ __forceinline__ uint32_t rep3_scan16(const Win &w, uint32_t q, uint32_t r) {
    const uint32_t *wd = reinterpret_cast<const uint32_t *>(w.d - kPre);
    const uint32_t ax = q + kPre, ay = q - r + kPre;
    const uint32_t *px = wd + (ax >> 2), *py = wd + (ay >> 2);
    const uint32_t sx = (ax & 3u) * 8u, sy = (ay & 3u) * 8u;
    uint32_t z[5];
    uint32_t xp = px[0], yp = py[0];
#pragma unroll
    for (uint32_t j = 0; j < 5; ++j) {
        const uint32_t xn = px[j + 1], yn = py[j + 1];
        const uint32_t d = __funnelshift_r(xp, xn, sx) ^ __funnelshift_r(yp, yn, sy);
        z[j] = ~(((d & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | d | 0x7F7F7F7Fu);
        xp = xn;
        yp = yn;
    }
    uint32_t m = 0;
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t e = z[j] & __funnelshift_r(z[j], z[j + 1], 8) & __funnelshift_r(z[j], z[j + 1], 16);
        m |= ((e * 0x00204081u) >> 28) << (4u * j);
    }
    return m;
}

// Bit t (t < 32) set when bytes q+t .. q+t+2 equal bytes q-r+t .. q-r+t+2:
// rep3_scan16 over 32 positions (34-byte ranges, ten aligned words each).
__device__ __forceinline__ uint32_t rep3_scan32(const Win &w, uint32_t q, uint32_t r) {
    const uint32_t *wd = reinterpret_cast<const uint32_t *>(w.d - kPre);
    const uint32_t ax = q + kPre, ay = q - r + kPre;
    const uint32_t *px = wd + (ax >> 2), *py = wd + (ay >> 2);
    const uint32_t sx = (ax & 3u) * 8u, sy = (ay & 3u) * 8u;
    uint32_t z[9];
    uint32_t xp = px[0], yp = py[0];
#pragma unroll
    for (uint32_t j = 0; j < 9; ++j) {
        const uint32_t xn = px[j + 1], yn = py[j + 1];
        const uint32_t d = __funnelshift_r(xp, xn, sx) ^ __funnelshift_r(yp, yn, sy);
        z[j] = ~(((d & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | d | 0x7F7F7F7Fu);
        xp = xn;
        yp = yn;
    }
    uint32_t m = 0;
#pragma unroll
    for (uint32_t j = 0; j < 8; ++j) {
        const uint32_t e = z[j] & __funnelshift_r(z[j], z[j + 1], 8) & __funnelshift_r(z[j], z[j + 1], 16);
        m |= ((e * 0x00204081u) >> 28) << (4u * j);
    }
    return m;
}

// One step of the exact parse for every GL-lane group of the warp at once
// (GL = 8 or 4), each from its own state s (group-uniform); groups with
// run == false keep theirs.  A group looks at the 32 positions from s.p: the
// hash-match bits come from the bitmap, and the lanes test the three repeat
// offsets among the positions before the first hash match
// (zstd_compress.cu:259-275) -- six lanes of 16 positions each (GL = 8) or
// three of 32 (GL = 4).  The first event is the match, extended 8 * GL bytes
// per group iteration, with the lazy step (:278-307) at f+1; with no event
// the group moves over the 32 positions.  Returns whether the group found a
// match (m set, s advanced past it, repeat offsets updated).
template <uint32_t GL>
__device__ __forceinline__ bool group_step(const Win &w, const uint32_t *bm, const uint16_t *cand, uint32_t size,
                                           bool lazy, bool run, PState &s, Match &m) {
    static_assert(GL == 8 || GL == 4, "8- or 4-lane groups");
    const uint32_t lane = lane_id(), gl = lane & (GL - 1u), gb = lane & ~(GL - 1u);
    const uint32_t p = run ? s.p : 0u;
    const uint32_t lim = run ? size - 3u - p : 0u;
    const uint32_t n32 = lim < 32u ? lim : 32u;
    uint32_t H = __funnelshift_r(bm[p >> 5], bm[(p >> 5) + 1], p & 31u);
    if (n32 < 32u) H &= (1u << n32) - 1u;
    const uint32_t nh = H ? static_cast<uint32_t>(__ffs(H)) - 1u : n32;  // positions without a hash match
    // The candidates at the first hash match and the position after it are
    // loaded before the repeat-offset test, so that their latency overlaps
    // it: the event is that hash match unless a repeat offset hits earlier
    // (a few times per window), and only then is cand(f+1) loaded again.
    const uint32_t fh = nh < n32 ? p + nh : 0u;
    const uint32_t ch0 = cand[fh], ch1 = cand[fh + 1u];
    uint32_t m0, m1, m2;  // per repeat offset: hits among the 32 positions
    if constexpr (GL == 8) {
        // Lane 2k+h (k < 3) tests repeat offset k on the 16 positions from
        // p + 16h that come before the first hash match and whose source lies
        // in the window; lanes 6 and 7 test nothing.
        const uint32_t rk = gl >> 1, hh = gl & 1u;
        const uint32_t q0 = p + 16u * hh;
        const uint32_t rv = rk == 0u ? s.r0 : (rk == 1u ? s.r1 : s.r2);
        const uint32_t lo = rv > q0 ? (rv - q0 < 16u ? rv - q0 : 16u) : 0u;
        const uint32_t hi = (rk < 3u && nh > 16u * hh) ? (nh - 16u * hh < 16u ? nh - 16u * hh : 16u) : 0u;
        const uint32_t vm = ((1u << hi) - 1u) & ~((1u << lo) - 1u);
        const uint32_t mk = rep3_scan16(w, q0, rv <= q0 + 16u ? rv : 0u) & vm;
        const uint32_t mo = __shfl_xor_sync(kFull, mk, 1);
        const uint32_t mf = hh ? (mo | (mk << 16)) : (mk | (mo << 16));  // offset rk over all 32 positions
        m0 = __shfl_sync(kFull, mf, gb);
        m1 = __shfl_sync(kFull, mf, gb + 2u);
        m2 = __shfl_sync(kFull, mf, gb + 4u);
    } else {
        // Lane k (k < 3) tests repeat offset k on the 32 positions from p
        // that come before the first hash match and whose source lies in the
        // window; lane 3 tests nothing.
        const uint32_t rv = gl == 0u ? s.r0 : (gl == 1u ? s.r1 : s.r2);
        const uint32_t lo = rv > p ? (rv - p < 32u ? rv - p : 32u) : 0u;
        const uint32_t hi = gl < 3u ? nh : 0u;  // nh <= 32
        const uint32_t vm = (hi >= 32u ? ~0u : (1u << hi) - 1u) & (lo >= 32u ? 0u : ~((1u << lo) - 1u));
        const uint32_t mk = rep3_scan32(w, p, rv <= p + 32u ? rv : 0u) & vm;
        m0 = __shfl_sync(kFull, mk, gb);
        m1 = __shfl_sync(kFull, mk, gb + 1u);
        m2 = __shfl_sync(kFull, mk, gb + 2u);
    }
    const uint32_t al = m0 | m1 | m2;
    const bool rep = al != 0u;
    const bool ev = run && (rep || nh < n32);
    uint32_t f = p + nh, r = 0;
    if (rep) {
        const uint32_t t = static_cast<uint32_t>(__ffs(al)) - 1u;
        f = p + t;
        r = (m0 >> t) & 1u ? 0u : ((m1 >> t) & 1u ? 1u : 2u);
    }
    const uint32_t fc = ev ? f : 0u;
    const uint32_t cf = zmap(ch0);
    uint32_t cf1 = zmap(ch1);
    if (rep) cf1 = zmap(cand[fc + 1u]);
    uint32_t off, c0;
    if (!rep) {
        off = fc - cf;
        c0 = cf;
    } else {  // first repeat offset with 3 equal bytes wins
        off = r == 0u ? s.r0 : (r == 1u ? s.r1 : s.r2);
        c0 = fc - off;
    }
    // The lazy candidate at f+1 is skipped when it is the same match one byte on
    // (cand(f+1) == c0 + 1): it is exactly one byte shorter, never taken.
    const bool ltry = ev && lazy && fc + 4u < size && bm_bit(bm, fc + 1u) && cf1 != c0 + 1u;
    const uint32_t e1 = extend_group<GL>(w, c0 + kMinMatch, fc + kMinMatch, ev ? size - fc - kMinMatch : 0u, ev);
    const uint32_t e2 =
        extend_group<GL>(w, cf1 + kMinMatch, fc + 1u + kMinMatch, ltry ? size - fc - 1u - kMinMatch : 0u, ltry);
    uint32_t len = e1 + kMinMatch;
    f = fc;
    if (ltry && e2 + kMinMatch > len + 1u) {
        f = fc + 1u;
        len = e2 + kMinMatch;
        off = f - cf1;
    }
    if (ev) {
        m.start = f;
        m.len = len;
        m.off = off;
        s.r2 = s.r1;
        s.r1 = s.r0;
        s.r0 = off;
        s.p = f + len;
    } else if (run) {
        s.p = p + n32;
    }
    return ev;
}

__device__ __forceinline__ uint2 pack_entry(const Match &m) {
    return make_uint2(m.start | ((m.len - kMinMatch) << 16), m.off);
}

// Repeat offsets after entry j of a list whose parse started from {1,4,8}.
__device__ __forceinline__ void reps_after(const uint2 *list, uint32_t j, uint32_t &a, uint32_t &b, uint32_t &c) {
    a = list[j].y;
    b = j >= 1 ? list[j - 1].y : 1u;
    c = j >= 2 ? list[j - 2].y : (j == 1 ? 1u : 4u);
}

// Warp-buffered list writer: entry i is held by lane i%32 until 32 are ready.
struct ListWriter {
    uint2 *out;
    uint32_t n;
    uint2 v;
    __device__ __forceinline__ explicit ListWriter(uint2 *o) : out(o), n(0), v(make_uint2(0u, 0u)) {}
    __device__ __forceinline__ void put(const uint2 &e) {
        if (lane_id() == (n & 31u)) v = e;
        if ((n & 31u) == 31u) out[(n & ~31u) + lane_id()] = v;
        ++n;
    }
    __device__ __forceinline__ void flush() {
        if (lane_id() < (n & 31u)) out[(n & ~31u) + lane_id()] = v;
    }
};

// ---------------------------------------------------------------- kernel
template <bool kRef, uint32_t SegW, uint32_t GL>
__global__ void __launch_bounds__(SegCfg<SegW, GL>::kThreads, SegCfg<SegW, GL>::kMinBlocks)
    zstd_parse_kernel(Zstd2Args a) {
    using C = SegCfg<SegW, GL>;
    constexpr uint32_t kSegW = C::kSegW, kWarps = C::kWarps, kThreads = C::kThreads, kSegs = C::kSegs;
    constexpr uint32_t kSpecCap = C::kSpecCap, kLaneCap = C::kLaneCap, kContCap = C::kContCap;
    extern __shared__ __align__(128) uint8_t smem_raw[];
    SmemLayout<kSegs> &S = *reinterpret_cast<SmemLayout<kSegs> *>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    uint32_t parity = 0;
    if (tid == 0) {
        mbar_init(&S.bar, 1);
        fence_mbar_init();
    }
    for (uint32_t i = tid; i < kPre / 4; i += kThreads) reinterpret_cast<uint32_t *>(S.data)[i] = 0u;
    __syncthreads();
    Win win{S.data + kPre};
    const bool lazy = a.lazy != 0;

    for (uint32_t wi = blockIdx.x; wi < a.num_windows; wi += gridDim.x) {
        const uint64_t start = a.wins ? a.wins[wi].offset : static_cast<uint64_t>(wi) * a.window;
        const uint32_t size =
            a.wins ? a.wins[wi].size : static_cast<uint32_t>(a.n - start < a.window ? a.n - start : a.window);
        const uint16_t *cand = a.cand + start;
        uint2 *seg = a.seg + static_cast<uint64_t>(wi) * a.seg_stride;

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
        // Lane l covers positions 4l .. 4l+3 of a 128-position chunk: one
        // 8-byte load brings its four candidates (2-byte loads where the
        // window's candidates are not 8-byte aligned or the chunk ends the
        // window), one aligned 8-byte read its own bytes, and the 8 lanes of
        // each bitmap word gather their four bits with three shuffles.  kVC
        // chunks per batch: their candidate loads are all issued first.
        constexpr uint32_t kChunks = kBmWords / 4u, kVC = 4;
        static_assert(kBmWords % 4u == 0u, "bitmap words come in 128-position chunks");
        const bool al8 = (reinterpret_cast<uintptr_t>(cand) & 7u) == 0u;
        for (uint32_t c0 = warp * kVC; c0 < kChunks; c0 += kWarps * kVC) {
            uint2 cv[kVC];
#pragma unroll
            for (uint32_t u = 0; u < kVC; ++u) {
                const uint32_t q = (c0 + u) * 128u + 4u * lane;
                if (al8 && q + 4u <= size) {
                    cv[u] = *reinterpret_cast<const uint2 *>(cand + q);
                } else {
                    uint32_t e[4];
#pragma unroll
                    for (uint32_t k = 0; k < 4; ++k) e[k] = q + k < size ? static_cast<uint32_t>(cand[q + k]) : 0u;
                    cv[u] = make_uint2(e[0] | (e[1] << 16), e[2] | (e[3] << 16));
                }
            }
#pragma unroll
            for (uint32_t u = 0; u < kVC; ++u) {
                const uint32_t ch = c0 + u;
                const uint32_t q = ch * 128u + 4u * lane;
                uint32_t nib = 0;
                if (q < size) {
                    const uint32_t x0 = win.w32(q), x1 = win.w32(q + 4u);
#pragma unroll
                    for (uint32_t k = 0; k < 4; ++k) {
                        const uint32_t cw = k < 2u ? cv[u].x : cv[u].y;
                        const uint32_t c = zmap((k & 1u) ? cw >> 16 : cw & 0xFFFFu);
                        const uint32_t xk = k ? __funnelshift_r(x0, x1, 8u * k) : x0;
                        const uint32_t qk = q + k;
                        const bool hm = qk + 3u < size && qk > 0u && ((xk ^ win.u32(static_cast<int>(c))) & 0xFFFFFFu) == 0u;
                        nib |= static_cast<uint32_t>(hm) << k;
                    }
                }
                uint32_t v = nib << (4u * (lane & 7u));
                v |= __shfl_xor_sync(kFull, v, 1);
                v |= __shfl_xor_sync(kFull, v, 2);
                v |= __shfl_xor_sync(kFull, v, 4);
                if ((lane & 7u) == 0u && ch < kChunks) S.bm[ch * 4u + (lane >> 3)] = v;
            }
        }
        __syncthreads();

        const uint32_t lim_pos = size > 3u ? size - 3u : 0u;  // positions q < lim_pos can start a match
        if constexpr (GL == 32) {
            // ---- 2a. speculative parse of each segment (one warp each)
            const uint32_t seg_start = warp * kSegW, seg_end = seg_start + kSegW;
            const bool active = seg_start < lim_pos;
            const bool last_active = !(seg_end < lim_pos);
            ListWriter lw(seg + warp * kLaneCap);
            PState s{seg_start, 1u, 4u, 8u};
            CandBuf cb{cand, size, 0u, 0u, 0u, 0u};
            if (active) cb.init(seg_start);
            if (active) {
                const uint32_t stop = last_active ? size : seg_end;
                Match m;
                while (s.p < stop && s.p + 3u < size) {
                    if (warp_step(win, S.bm, cb, size, lazy, s, m)) lw.put(pack_entry(m));
                }
                lw.flush();
            }
            if (lane == 0) {
                S.spec_count[warp] = lw.n;
                S.cont_count[warp] = 0;
                S.sync_warp[warp] = kNoWarp;
                S.sync_idx[warp] = 0;
            }
            __syncthreads();

            // ---- 2b. continue each warp's parse until it meets a later warp's list
            if (active && !last_active) {
                ListWriter cw(seg + warp * kLaneCap + kSpecCap);
                uint32_t t = kNoWarp, j = 0;
                Match m;
                while (s.p + 3u < size) {
                    if (!warp_step(win, S.bm, cb, size, lazy, s, m)) continue;
                    const uint32_t tw = m.start / kSegW;  // warp whose segment holds this match start
                    if (tw != t) {
                        t = tw;
                        j = 0;
                    }
                    const uint32_t tcount = S.spec_count[t];
                    const uint2 *tl = seg + t * kLaneCap;
                    // first entry of t's list with start >= m.start (lists are sorted by start)
                    for (;;) {
                        const uint32_t idx = j + lane;
                        const bool ge = idx >= tcount || (tl[idx].x & 0xFFFFu) >= m.start;
                        const uint32_t b = __ballot_sync(kFull, ge);
                        if (b) {
                            j += static_cast<uint32_t>(__ffs(b)) - 1u;
                            break;
                        }
                        j += 32u;
                    }
                    bool met = false;
                    if (j < tcount) {
                        const uint2 e = tl[j];
                        if (e.x == pack_entry(m).x && e.y == m.off) {
                            uint32_t e0, e1, e2;
                            reps_after(tl, j, e0, e1, e2);
                            met = e0 == s.r0 && e1 == s.r1 && e2 == s.r2;
                        }
                    }
                    if (met) {
                        if (lane == 0) {
                            S.sync_warp[warp] = t;
                            S.sync_idx[warp] = j;
                        }
                        break;
                    }
                    if (cw.n == kContCap) {
                        if (lane == 0) atomicOr(&S.flags, 1u);  // give up: exact fallback below
                        break;
                    }
                    cw.put(pack_entry(m));
                }
                cw.flush();
                if (lane == 0) S.cont_count[warp] = cw.n;
            }
            __syncthreads();
        } else {
            // ---- 2a. speculative parse of each segment (one 8-lane group each)
            const uint32_t sg = tid / GL, gl = lane & (GL - 1u), gb = lane & ~(GL - 1u);
            const uint32_t seg_start = sg * kSegW, seg_end = seg_start + kSegW;
            const bool active = seg_start < lim_pos;
            const bool last_active = !(seg_end < lim_pos);
            const uint32_t stop = last_active ? size : seg_end;
            uint2 *lst = seg + sg * kLaneCap;
            PState s{seg_start, 1u, 4u, 8u};
            uint32_t n = 0;
            for (;;) {
                const bool run = active && s.p < stop && s.p + 3u < size;
                if (!__any_sync(kFull, run)) break;
                Match m;
                if (group_step<GL>(win, S.bm, cand, size, lazy, run, s, m)) {
                    if (gl == 0) lst[n] = pack_entry(m);
                    ++n;
                }
            }
            if (gl == 0) {
                S.spec_count[sg] = n;
                S.cont_count[sg] = 0;
                S.sync_warp[sg] = kNoWarp;
                S.sync_idx[sg] = 0;
            }
            __syncthreads();

            // ---- 2b. continue each group's parse until it meets a later segment's list
            bool crun = active && !last_active;
            uint32_t t = kNoWarp, j = 0, cn = 0;
            uint2 *cl = lst + kSpecCap;
            for (;;) {
                const bool run = crun && s.p + 3u < size;
                const uint32_t runners = __ballot_sync(kFull, run && gl == 0u);
                if (!runners) break;
                if ((runners & (runners - 1u)) == 0u) {
                    // Only one group of the warp still runs (the slow tail of the
                    // phase): the whole warp takes over its parse with warp-wide
                    // steps (up to 128 positions scanned, 128 bytes extended per
                    // iteration), same meeting test, then the loop ends.
                    const uint32_t L = static_cast<uint32_t>(__ffs(runners)) - 1u;
                    PState ws{__shfl_sync(kFull, s.p, L), __shfl_sync(kFull, s.r0, L), __shfl_sync(kFull, s.r1, L),
                              __shfl_sync(kFull, s.r2, L)};
                    const uint32_t wsg = __shfl_sync(kFull, sg, L);
                    uint32_t wt = __shfl_sync(kFull, t, L), wj = __shfl_sync(kFull, j, L),
                             wcn = __shfl_sync(kFull, cn, L);
                    uint2 *wcl = seg + wsg * kLaneCap + kSpecCap;
                    CandBuf wcb{cand, size, 0u, 0u, 0u, 0u};
                    wcb.init(ws.p);
                    while (ws.p + 3u < size) {
                        Match m;
                        if (!warp_step(win, S.bm, wcb, size, lazy, ws, m)) continue;
                        const uint32_t tw = m.start / kSegW;  // segment that holds this match start
                        if (tw != wt) {
                            wt = tw;
                            wj = 0;
                        }
                        const uint32_t tcount = S.spec_count[wt];
                        const uint2 *tl = seg + wt * kLaneCap;
                        // first entry of wt's list with start >= m.start, 32 per step
                        for (;;) {
                            const uint32_t idx = wj + lane;
                            const bool ge = idx >= tcount || (tl[idx].x & 0xFFFFu) >= m.start;
                            const uint32_t b = __ballot_sync(kFull, ge);
                            if (b) {
                                wj += static_cast<uint32_t>(__ffs(b)) - 1u;
                                break;
                            }
                            wj += 32u;
                        }
                        bool met = false;
                        if (wj < tcount) {
                            const uint2 e = tl[wj];
                            if (e.x == pack_entry(m).x && e.y == m.off) {
                                uint32_t e0, e1, e2;
                                reps_after(tl, wj, e0, e1, e2);
                                met = e0 == ws.r0 && e1 == ws.r1 && e2 == ws.r2;
                            }
                        }
                        if (met) {
                            if (lane == 0) {
                                S.sync_warp[wsg] = wt;
                                S.sync_idx[wsg] = wj;
                            }
                            break;
                        }
                        if (wcn == kContCap) {
                            if (lane == 0) atomicOr(&S.flags, 1u);  // give up: exact fallback below
                            break;
                        }
                        if (lane == 0) wcl[wcn] = pack_entry(m);
                        ++wcn;
                    }
                    if (lane >= L && lane < L + GL) {
                        cn = wcn;
                        crun = false;
                    }
                    break;
                }
                Match m;
                const bool ev = group_step<GL>(win, S.bm, cand, size, lazy, run, s, m);
                uint32_t tcount = 0;
                const uint2 *tl = seg;
                if (ev) {
                    const uint32_t tw = m.start / kSegW;  // segment that holds this match start
                    if (tw != t) {
                        t = tw;
                        j = 0;
                    }
                    tcount = S.spec_count[t];
                    tl = seg + t * kLaneCap;
                }
                // first entry of t's list with start >= m.start (lists are sorted by start), 8 per step
                bool found = !ev;
                while (__any_sync(kFull, !found)) {
                    const uint32_t idx = j + gl;
                    const bool ge = !found && (idx >= tcount || (tl[idx].x & 0xFFFFu) >= m.start);
                    const uint32_t b = (__ballot_sync(kFull, ge) >> gb) & ((1u << GL) - 1u);
                    if (!found) {
                        if (b) {
                            j += static_cast<uint32_t>(__ffs(b)) - 1u;
                            found = true;
                        } else {
                            j += GL;
                        }
                    }
                }
                if (!ev) {
                    if (!run) crun = false;
                    continue;
                }
                bool met = false;
                if (j < tcount) {
                    const uint2 e = tl[j];
                    if (e.x == pack_entry(m).x && e.y == m.off) {
                        uint32_t e0, e1, e2;
                        reps_after(tl, j, e0, e1, e2);
                        met = e0 == s.r0 && e1 == s.r1 && e2 == s.r2;
                    }
                }
                if (met) {
                    if (gl == 0) {
                        S.sync_warp[sg] = t;
                        S.sync_idx[sg] = j;
                    }
                    crun = false;
                } else if (cn == kContCap) {
                    if (gl == 0) atomicOr(&S.flags, 1u);  // give up: exact fallback below
                    crun = false;
                } else {
                    if (gl == 0) cl[cn] = pack_entry(m);
                    ++cn;
                }
            }
            if (gl == 0) S.cont_count[sg] = cn;
            __syncthreads();
        }

        if (!(S.flags & 1u)) {
            // ---- 3. chain walk, then copy in chain order.  Nearly always every
            // continuation meets the next segment's list, so the chain is
            // segments 0..K in order (K: the first segment with no link): warp
            // 0 then sets it up at once -- output offsets by a scan of the
            // segments' contributions, each segment's preceding entry by a max
            // scan (entry indices grow with the segment).  Otherwise one
            // thread walks the links.
            bool chained = false;
            if (warp == 0 && lim_pos > 0) {
                constexpr uint32_t kPer = (kSegs + 31u) / 32u;  // segments per lane, contiguous
                uint32_t kf = kSegs;
                bool gap = false;
#pragma unroll
                for (uint32_t u = 0; u < kPer; ++u) {
                    const uint32_t i = lane * kPer + u;
                    if (i < kSegs && S.sync_warp[i] == kNoWarp && i < kf) kf = i;
                }
                const uint32_t K = __reduce_min_sync(kFull, kf);  // segment 0 always parses, so K < kSegs
#pragma unroll
                for (uint32_t u = 0; u < kPer; ++u) {
                    const uint32_t i = lane * kPer + u;
                    if (i < K && S.sync_warp[i] != i + 1u) gap = true;
                }
                chained = !__any_sync(kFull, gap);
                if (chained) {
                    uint32_t con[kPer], lst1[kPer], sum = 0, lmax = 0;
#pragma unroll
                    for (uint32_t u = 0; u < kPer; ++u) {
                        const uint32_t i = lane * kPer + u;
                        con[u] = 0;
                        lst1[u] = 0;
                        if (i <= K) {
                            const uint32_t from = i ? static_cast<uint32_t>(S.sync_idx[i - 1u]) : 0u;
                            const uint32_t ns = S.spec_count[i], nc = S.cont_count[i];
                            con[u] = ns - from + nc;
                            if (con[u]) lst1[u] = 1u + i * kLaneCap + (nc ? kSpecCap + nc - 1u : ns - 1u);
                        }
                        sum += con[u];
                        lmax = lst1[u] > lmax ? lst1[u] : lmax;
                    }
                    // exclusive scans over the lanes: sum of contributions, max of last entries (+1)
                    uint32_t incl = sum, mx = lmax;
#pragma unroll
                    for (uint32_t d = 1; d < 32u; d <<= 1) {
                        const uint32_t o = __shfl_up_sync(kFull, incl, d), om = __shfl_up_sync(kFull, mx, d);
                        if (lane >= d) {
                            incl += o;
                            mx = om > mx ? om : mx;
                        }
                    }
                    uint32_t acc = incl - sum, last1 = __shfl_up_sync(kFull, mx, 1);
                    if (lane == 0) last1 = 0;
#pragma unroll
                    for (uint32_t u = 0; u < kPer; ++u) {
                        const uint32_t i = lane * kPer + u;
                        if (i >= kSegs) continue;
                        const bool on = i <= K;
                        S.on_chain[i] = on ? 1u : 0u;
                        if (on) {
                            S.chain_from[i] = i ? S.sync_idx[i - 1u] : 0u;
                            S.out_off[i] = acc;
                            S.prev_last[i] = last1 ? last1 - 1u : kNoEntry;
                        }
                        acc += con[u];
                        last1 = lst1[u] > last1 ? lst1[u] : last1;
                    }
                    if (lane == 31u) S.total = incl;
                }
            }
            chained = __syncthreads_or(chained);
            if (tid == 0 && !chained) {
                for (uint32_t i = 0; i < kSegs; ++i) S.on_chain[i] = 0;
                uint32_t cur = 0, from = 0, acc = 0, last = kNoEntry;
                if (lim_pos > 0) {
                    for (;;) {
                        S.on_chain[cur] = 1;
                        S.chain_from[cur] = from;
                        S.out_off[cur] = acc;
                        S.prev_last[cur] = last;
                        const uint32_t ns = S.spec_count[cur], nc = S.cont_count[cur];
                        acc += (ns - from) + nc;
                        if (ns + nc > from) last = cur * kLaneCap + (nc ? kSpecCap + nc - 1u : ns - 1u);
                        const uint32_t nx = S.sync_warp[cur];
                        if (nx == kNoWarp) break;
                        from = S.sync_idx[cur];
                        cur = nx;
                    }
                }
                S.total = acc;
            }
            __syncthreads();
            const uint32_t total = S.total;
            const uint32_t keep = total < a.max_seqs ? total : a.max_seqs;
            // Write {ll, ml-3, off} in chain order: an entry's literal length is
            // its start minus the end of the entry before it -- the previous
            // entry of the same list, or for a segment's first copied entry the
            // last entry contributed before it, which the chain walk located.
            const uint32_t csg = tid / GL, csl = tid % GL;  // segment whose list this thread copies
            if (S.on_chain[csg]) {
                const uint32_t from = S.chain_from[csg], ns = S.spec_count[csg], nc = S.cont_count[csg];
                const uint32_t base = S.out_off[csg];
                const uint2 *mine = seg + csg * kLaneCap;
                uint32_t cov = 0;
                for (uint32_t i = from + csl; i < ns + nc; i += GL) {
                    const uint32_t o = base + (i - from);
                    if (o >= keep) break;
                    const uint2 e = mine[i < ns ? i : kSpecCap + (i - ns)];
                    const uint32_t pi =
                        i > from ? csg * kLaneCap + (i - 1u < ns ? i - 1u : kSpecCap + (i - 1u - ns)) : S.prev_last[csg];
                    uint32_t pe = 0;
                    if (pi != kNoEntry) {
                        const uint32_t px = seg[pi].x;
                        pe = (px & 0xFFFFu) + (px >> 16) + kMinMatch;
                    }
                    const uint32_t st0 = e.x & 0xFFFFu, mlm3 = e.x >> 16;
                    const uint32_t ll = st0 - pe;
                    cov += mlm3 + kMinMatch;
                    if constexpr (kRef) {
                        uint32_t *r = a.ref_seqs + (static_cast<uint64_t>(wi) * a.max_seqs + o) * 3u;
                        r[0] = ll;
                        r[1] = mlm3;
                        r[2] = e.y;
                    } else {
                        a.packed[static_cast<uint64_t>(wi) * a.max_seqs + o] = make_uint2(ll | (mlm3 << 16), e.y);
                    }
                }
                if (cov) atomicAdd(&S.covered, cov);
            }
            __syncthreads();
            if (tid == 0) {
                a.seq_counts[wi] = keep;
                if (a.lit_counts) a.lit_counts[wi] = size - S.covered;
            }
        } else if (warp == 0) {
            // ---- exact warp-wide parse of the whole window
            PState fs{0u, 1u, 4u, 8u};
            CandBuf fcb{cand, size, 0u, 0u, 0u, 0u};
            fcb.init(0u);
            uint32_t idx = 0, cov = 0, prev_end = 0;
            Match m;
            while (fs.p + 3u < size) {
                if (!warp_step(win, S.bm, fcb, size, lazy, fs, m)) continue;
                if (idx < a.max_seqs && lane == 0) {
                    const uint32_t ll = m.start - prev_end;
                    if constexpr (kRef) {
                        uint32_t *r = a.ref_seqs + (static_cast<uint64_t>(wi) * a.max_seqs + idx) * 3u;
                        r[0] = ll;
                        r[1] = m.len - kMinMatch;
                        r[2] = m.off;
                    } else {
                        a.packed[static_cast<uint64_t>(wi) * a.max_seqs + idx] =
                            make_uint2(ll | ((m.len - kMinMatch) << 16), m.off);
                    }
                }
                if (idx < a.max_seqs) cov += m.len;
                ++idx;
                prev_end = m.start + m.len;
            }
            if (lane == 0) {
                a.seq_counts[wi] = idx < a.max_seqs ? idx : a.max_seqs;
                if (a.lit_counts) a.lit_counts[wi] = size - cov;
                atomicAdd(a.status + 1, 1u);  // fallback counter (diagnostics)
            }
        }
    }
}

}  // namespace

// Seg entries per window: the largest of the layouts, so that a buffer sized
// once serves every segment width.
template <uint32_t SegW, uint32_t GL = 32>
constexpr uint32_t seg_entries() { return SegCfg<SegW, GL>::kSegs * SegCfg<SegW, GL>::kLaneCap; }
constexpr uint32_t kSegStride = []() constexpr {
    uint32_t m = seg_entries<2048>();
    if (seg_entries<4096>() > m) m = seg_entries<4096>();
    if (seg_entries<8192>() > m) m = seg_entries<8192>();
    if (seg_entries<1024, 8>() > m) m = seg_entries<1024, 8>();
    if (seg_entries<512, 4>() > m) m = seg_entries<512, 4>();
    return m;
}();

size_t zstd2_seg_scratch_entries(uint32_t num_windows) { return static_cast<size_t>(num_windows) * kSegStride; }

namespace {
template <bool kRef, uint32_t SegW, uint32_t GL>
cudaError_t launch_parse_variant(const Zstd2Args &a, int num_sms, int ctas_per_sm, cudaStream_t st) {
    using C = SegCfg<SegW, GL>;
    const uint32_t smem = sizeof(SmemLayout<C::kSegs>);
    static_assert(sizeof(SmemLayout<C::kSegs>) + 1024 <= 233472 / 3, "three CTAs per SM must fit");
    static SmemOnce smem_set{0};
    cudaError_t e = set_smem_once(zstd_parse_kernel<kRef, SegW, GL>, smem, smem_set);
    if (e != cudaSuccess) return e;
    int grid = num_sms * ctas_per_sm;
    if (static_cast<uint32_t>(grid) > a.num_windows) grid = static_cast<int>(a.num_windows);
    zstd_parse_kernel<kRef, SegW, GL><<<grid, C::kThreads, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool kRef>
cudaError_t launch_parse_ref(const Zstd2Args &a, uint32_t seg_width, int num_sms, int ctas_per_sm, cudaStream_t st) {
    if (seg_width == 512) return launch_parse_variant<kRef, 512, 4>(a, num_sms, ctas_per_sm, st);
    if (seg_width == 1024) return launch_parse_variant<kRef, 1024, 8>(a, num_sms, ctas_per_sm, st);
    if (seg_width == 2048) return launch_parse_variant<kRef, 2048, 32>(a, num_sms, ctas_per_sm, st);
    if (seg_width == 8192) return launch_parse_variant<kRef, 8192, 32>(a, num_sms, ctas_per_sm, st);
    return launch_parse_variant<kRef, 4096, 32>(a, num_sms, ctas_per_sm, st);
}
}  // namespace

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
    a.wins = l.wins;
    a.seg_stride = kSegStride;
    return l.ref_seqs ? launch_parse_ref<true>(a, l.seg_width, l.num_sms, l.ctas_per_sm, st)
                      : launch_parse_ref<false>(a, l.seg_width, l.num_sms, l.ctas_per_sm, st);
}

}  // namespace gcz
