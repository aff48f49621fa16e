// Zstd entropy stage on the GPU: one Zstd frame per 64 KiB window, built from
// the window's ZSTD_Sequence records, decodable by any conforming decoder
// (stock libzstd).
//
// Frame layout (RFC 8878): magic, a single-segment frame header with the
// content size, and one block.  The block is a compressed block when that is
// smaller than the window, else a raw block.  A compressed block holds
//   - the window's literal bytes, in order, as the smallest of a raw, an RLE
//     or a Huffman-coded literals block;
//   - a sequences section in Predefined_Mode for literal lengths, offsets and
//     match lengths (the format's default distributions, so no table is
//     transmitted), whose bitstream is written by an FSE (tANS) encoder
//     derived from the decoder's state tables: for symbol s and the decoder
//     state D' that follows, the encoder picks the state D of s with
//     baseline(D) <= D' < baseline(D) + 2^nbBits(D) and writes D' - baseline(D).
// Offsets use the format's repeat codes whenever the actual offset equals one
// of the three repeat offsets the decoder holds at that point.
//
// Kernels, per window:
//   zenc_literals_kernel   (one CTA):    window staged by bulk copy, literal
//                                        gather, raw literal section, histogram
//   zenc_huf_plan_kernel   (one warp):   Huffman code and tree description
//   zenc_huf_write_kernel  (one CTA):    RLE or Huffman-coded literal section
//                                        where that is smaller
//   zenc_sequences_kernel  (one warp):   repeat-code pass, FSE chains, bitstream,
//                                        block header, frame size
//   zenc_compact_kernel    (one CTA):    frames back to back at scanned offsets
// Frames are built in per-window slots of kZencSlot bytes first, because a
// frame's size is known only once its bitstream is written.
#include "gcz_common.cuh"
#include "gcz_kernels.h"

namespace gcz {
namespace {

constexpr uint32_t kErrBadSequences = 4;  // status bit: sequences do not describe their window
constexpr uint32_t kLitThreads = 256;

// Predefined distributions (RFC 8878 3.1.1.3.2.2); -1 = "less than 1".
__constant__ int8_t kLLNorm[36] = {4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2,
                                   2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1};
__constant__ int8_t kMLNorm[53] = {1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                   1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                   1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1};
__constant__ int8_t kOFNorm[29] = {1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1,
                                   1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1};
constexpr uint32_t kLLLog = 6, kMLLog = 6, kOFLog = 5;
constexpr uint32_t kLLSyms = 36, kMLSyms = 53, kOFSyms = 29;

// Literal-length and match-length codes (RFC 8878 3.1.1.3.2.1.1): baseline and
// number of extra bits per code.
__constant__ uint32_t kLLBase[36] = {0,  1,  2,  3,  4,  5,   6,   7,   8,    9,    10,   11,
                                     12, 13, 14, 15, 16, 18,  20,  22,  24,   28,   32,   40,
                                     48, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536};
__constant__ uint8_t kLLBits[36] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1,
                                    1, 1, 2, 2, 3, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
__constant__ uint32_t kMLBase[53] = {3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13,  14,  15,   16,   17,   18,   19,   20,
                                     21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31,  32,  33,   34,   35,   37,   39,   41,
                                     43, 47, 51, 59, 67, 83, 99, 131, 259, 515, 1027, 2051, 4099, 8195, 16387, 32771, 65539};
__constant__ uint8_t kMLBits[53] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  0,  0,  0, 0, 0,
                                    0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 3, 3, 4, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};

__device__ __forceinline__ uint32_t highbit(uint32_t x) { return 31u - static_cast<uint32_t>(__clz(x)); }

// Largest code whose baseline is <= v (bases ascending).
__device__ __forceinline__ uint32_t code_of(const uint32_t *base, uint32_t ncodes, uint32_t v) {
    uint32_t lo = 0, hi = ncodes - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (base[mid] <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Code tables copied to shared memory (lanes of a warp look up different
// codes): baselines, extra bits, and codes of the small values; above those,
// codes follow the highest set bit.
struct CodeTables {
    uint32_t ll_base[kLLSyms];
    uint32_t ml_base[kMLSyms];
    uint8_t ll_bits[kLLSyms];
    uint8_t ml_bits[kMLSyms];
    uint8_t ll_lut[64];   // code of literal length v < 64
    uint8_t ml_lut[128];  // code of match length v + 3, v < 128
    __device__ void build() {
        for (uint32_t i = threadIdx.x; i < kLLSyms; i += blockDim.x) {
            ll_base[i] = kLLBase[i];
            ll_bits[i] = kLLBits[i];
        }
        for (uint32_t i = threadIdx.x; i < kMLSyms; i += blockDim.x) {
            ml_base[i] = kMLBase[i];
            ml_bits[i] = kMLBits[i];
        }
        for (uint32_t v = threadIdx.x; v < 64u; v += blockDim.x) ll_lut[v] = static_cast<uint8_t>(code_of(kLLBase, kLLSyms, v));
        for (uint32_t v = threadIdx.x; v < 128u; v += blockDim.x)
            ml_lut[v] = static_cast<uint8_t>(code_of(kMLBase, kMLSyms, v + 3u));
    }
    // Literal lengths >= 64 take code 19 + highbit (64 -> 25, ..., 65536 -> 35).
    __device__ __forceinline__ uint32_t ll_code(uint32_t ll) const { return ll < 64u ? ll_lut[ll] : highbit(ll) + 19u; }
    // Match lengths >= 131 take code 36 + highbit(ml - 3) (131 -> 43, ..., 65539 -> 52).
    __device__ __forceinline__ uint32_t ml_code(uint32_t ml) const {
        const uint32_t v = ml - 3u;
        return v < 128u ? ml_lut[v] : highbit(v) + 36u;
    }
};

// Forward bit writer (the decoder reads the stream backwards from its end
// marker).  Bytes go to global memory one at a time: frame positions have no
// alignment.
struct BitWriter {
    uint8_t *out;
    uint32_t pos;  // bytes written
    uint64_t acc;
    uint32_t nbits;
    __device__ __forceinline__ void add(uint32_t v, uint32_t nb) {
        acc |= static_cast<uint64_t>(v) << nbits;
        nbits += nb;
        if (nbits >= 32u) {
            const uint32_t w = static_cast<uint32_t>(acc);
            out[pos] = static_cast<uint8_t>(w);
            out[pos + 1] = static_cast<uint8_t>(w >> 8);
            out[pos + 2] = static_cast<uint8_t>(w >> 16);
            out[pos + 3] = static_cast<uint8_t>(w >> 24);
            pos += 4u;
            acc >>= 32;
            nbits -= 32u;
        }
    }
    __device__ __forceinline__ void close() {
        add(1u, 1u);  // end marker
        while (nbits > 0u) {
            out[pos++] = static_cast<uint8_t>(acc);
            acc >>= 8;
            nbits = nbits > 8u ? nbits - 8u : 0u;
        }
    }
};

struct ZencArgs {
    const uint8_t *src;
    uint64_t n;
    uint32_t window;
    uint32_t num_windows;
    const uint4 *seqs;         // ZSTD_Sequence records {offset, litLength, matchLength, rep}
    const uint64_t *seq_offsets;  // num_windows + 1
    uint8_t *slots;            // kZencSlot bytes per window
    uint32_t *ovs;             // kZencMaxSeqs per window
    uint32_t *sec_off;         // start of the sequences section in the slot (0 = raw frame)
    uint32_t *fsize;           // frame bytes
    uint8_t *raw;              // 1 = raw block
    uint32_t *hist;            // 256 literal-byte counts per window
    uint8_t *plan;             // kZencPlanBytes per window
    uint32_t *status;
    const WinDesc *wins;       // optional window table (null: windows at b * window)
};

__device__ __forceinline__ uint32_t win_size(const ZencArgs &a, uint32_t b) {
    if (a.wins) return a.wins[b].size;
    const uint64_t s = static_cast<uint64_t>(b) * a.window;
    return static_cast<uint32_t>(a.n - s < a.window ? a.n - s : a.window);
}
// First byte of window b: at b * window, or where the window table puts it.
__device__ __forceinline__ const uint8_t *win_src(const ZencArgs &a, uint32_t b) {
    return a.src + (a.wins ? a.wins[b].offset : static_cast<uint64_t>(b) * a.window);
}
__device__ __forceinline__ uint32_t frame_header_bytes(uint32_t w) { return 4u + 1u + (w < 256u ? 1u : 2u); }

__device__ void write_frame_header(uint8_t *p, uint32_t w) {
    p[0] = 0x28;
    p[1] = 0xB5;
    p[2] = 0x2F;
    p[3] = 0xFD;
    if (w < 256u) {
        p[4] = 0x20;  // Single_Segment, 1-byte Frame_Content_Size
        p[5] = static_cast<uint8_t>(w);
    } else {
        p[4] = 0x60;  // Single_Segment, 2-byte Frame_Content_Size (value - 256)
        p[5] = static_cast<uint8_t>(w - 256u);
        p[6] = static_cast<uint8_t>((w - 256u) >> 8);
    }
}

__device__ __forceinline__ void write_block_header(uint8_t *p, uint32_t type, uint32_t size) {
    const uint32_t h = 1u | (type << 1) | (size << 3);  // Last_Block set: one block per frame
    p[0] = static_cast<uint8_t>(h);
    p[1] = static_cast<uint8_t>(h >> 8);
    p[2] = static_cast<uint8_t>(h >> 16);
}

// 4 bytes at p (any alignment) from global memory: the aligned words that
// hold them, funnel-shifted; the second word is read only when p is unaligned,
// so no word without a wanted byte is touched.
__device__ __forceinline__ uint32_t load4(const uint8_t *p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~static_cast<uintptr_t>(3));
    const uint32_t sh = static_cast<uint32_t>(a & 3u) * 8u;
    const uint32_t lo = __ldg(w);
    return sh ? __funnelshift_r(lo, __ldg(w + 1), sh) : lo;
}

// The CTA copies n bytes from s to d (any alignments): aligned 32-bit stores
// for the whole words of d, byte stores at its two ends.
__device__ void cta_copy(uint8_t *d, const uint8_t *s, uint32_t n) {
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    const uint32_t head = min(n, (4u - static_cast<uint32_t>(reinterpret_cast<uintptr_t>(d) & 3u)) & 3u);
    for (uint32_t k = tid; k < head; k += nt) d[k] = s[k];
    const uint32_t nw = (n - head) >> 2;
    uint32_t *dw = reinterpret_cast<uint32_t *>(d + head);
    for (uint32_t k = tid; k < nw; k += nt) dw[k] = load4(s + head + 4u * k);
    for (uint32_t k = head + 4u * nw + tid; k < n; k += nt) d[k] = s[k];
}

// ---------------------------------------------------------------- literals
// The literal section is the smallest of: raw; RLE (one distinct byte);
// Huffman-coded (RFC 8878 4.2), one stream below 1024 literals, else four.
// The Huffman code: two-queue construction over the present bytes (leaves
// sorted by count, then byte value; a leaf wins ties), lengths limited to 11
// bits by moving pairs of leaves up the tree (which keeps the code complete),
// the longest codes to the least frequent bytes, canonical code values (the
// longest codes take the smallest values, ties by byte value).  Weights are
// sent directly when there are at most 128 of them, else FSE-compressed with
// accuracy 6: counts normalised by floor(c * 64 / N) (at least 1), the
// largest absorbing the remainder; two interleaved states; the state of the
// second-to-last weight is chosen with at least one update bit, so that the
// decoder's last update runs past the stream start and decoding ends there.
//
// Three kernels: zenc_literals_kernel gathers each window's literals, writes
// the raw literal section (the default) and the byte histogram;
// zenc_huf_plan_kernel builds the code of a window in one warp (many windows
// per SM, so the serial steps of one overlap the others');
// zenc_huf_write_kernel rewrites the section as RLE or Huffman-coded where
// that is smaller.
constexpr uint32_t kHufMaxBits = 11;

// Per-window record from the plan to the write kernel.
struct PlanRec {
    uint8_t len[256];
    uint16_t code[256];
    uint8_t tree[132];  // Huffman_Tree_Description
    uint32_t tree_bytes;
    uint32_t mode;  // 0: keep raw, 1: RLE, 2: Huffman candidate
    uint32_t nlit;
    uint32_t rle;
};
static_assert(sizeof(PlanRec) <= kZencPlanBytes, "plan record");

__device__ __forceinline__ uint32_t raw_lit_header_bytes(uint32_t nlit) {
    return nlit < 32u ? 1u : (nlit < 4096u ? 2u : 3u);
}
__device__ void write_raw_lit_header(uint8_t *h, uint32_t type, uint32_t nlit) {
    const uint32_t hb = raw_lit_header_bytes(nlit);
    if (hb == 1u) {
        h[0] = static_cast<uint8_t>(type | (nlit << 3));
    } else if (hb == 2u) {
        h[0] = static_cast<uint8_t>(type | (1u << 2) | ((nlit << 4) & 0xF0u));
        h[1] = static_cast<uint8_t>(nlit >> 4);
    } else {
        h[0] = static_cast<uint8_t>(type | (3u << 2) | ((nlit << 4) & 0xF0u));
        h[1] = static_cast<uint8_t>(nlit >> 4);
        h[2] = static_cast<uint8_t>(nlit >> 12);
    }
}

// Gathers the literals of each window into shared memory (one CTA per
// window), validates the sequences, writes frame header + raw literal
// section into the slot and the histogram of the literal bytes.  The window
// is staged into shared memory with 1-D bulk copies first, so the gather
// copies shared memory to shared memory.
constexpr uint32_t kGatherThreads = 512;

struct GatherSmem {
    uint8_t win[kMaxWindow + 64];  // staged window, zero padding after it
    uint8_t lit[kMaxWindow];
    // Byte counts: 4 copies per warp (by lane & 3), so the lanes that count
    // the same frequent byte at once are spread over copies; summed at the end.
    uint32_t hist[kGatherThreads / 32 * 4][256];
    uint32_t warp_ll[kGatherThreads / 32], warp_pos[kGatherThreads / 32];
    uint32_t bad, flags;
    alignas(8) uint64_t bar;
};

__global__ void __launch_bounds__(kGatherThreads) zenc_literals_kernel(ZencArgs a) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    GatherSmem &S = *reinterpret_cast<GatherSmem *>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
    uint32_t parity = 0;
    if (tid == 0) {
        mbar_init(&S.bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    for (uint32_t b = blockIdx.x; b < a.num_windows; b += gridDim.x) {
        const uint32_t w = win_size(a, b);
        const uint8_t *src = win_src(a, b);
        const uint64_t s0 = a.seq_offsets[b];
        const uint32_t ns = static_cast<uint32_t>(a.seq_offsets[b + 1] - s0);
        const uint4 *sq = a.seqs + s0;
        uint8_t *slot = a.slots + static_cast<uint64_t>(b) * kZencSlot;
        PlanRec *plan = reinterpret_cast<PlanRec *>(a.plan + static_cast<uint64_t>(b) * kZencPlanBytes);
        const uint32_t fh = frame_header_bytes(w);
        if (tid == 0) {
            S.bad = ns > kZencMaxSeqs ? 1u : 0u;
            S.flags = 0u;
        }
        for (uint32_t k = tid; k < kGatherThreads / 32 * 4 * 256; k += kGatherThreads) (&S.hist[0][0])[k] = 0u;
        __syncthreads();
        if (ns == 0u) {  // no sequences: the raw block is smaller
            if (tid == 0) {
                write_frame_header(slot, w);
                a.sec_off[b] = 0u;
                plan->nlit = 0u;
            }
            __syncthreads();
            continue;
        }
        if (wid == 0 && !stage_window(S.win, src, w, &S.bar, parity, a.status) && lane == 0) S.flags = 1u;
        // Each warp owns a contiguous, equal share of the sequences and copies
        // every literal run of its share with all 32 lanes, so one long run
        // does not hold up the CTA.  First the warps' totals, then a scan over
        // the warps gives each share's first literal index and source position.
        constexpr uint32_t kW32 = kGatherThreads / 32;
        const uint32_t per = (ns + kW32 - 1) / kW32;
        const uint32_t i0 = min(wid * per, ns), i1 = min(i0 + per, ns);
        uint32_t sll = 0, spos = 0;
        for (uint32_t i = i0 + lane; i < i1; i += 32u) {
            const uint4 q = sq[i];
            // lengths bounded by the window, so the sums below cannot wrap
            if (q.x == 0u || q.y > kMaxWindow || q.z < 3u || q.z > kMaxWindow) S.bad = 1u;
            sll += q.y;
            spos += q.y + q.z;
        }
        for (uint32_t o = 16; o > 0; o >>= 1) {
            sll += __shfl_xor_sync(kFull, sll, o);
            spos += __shfl_xor_sync(kFull, spos, o);
        }
        if (lane == 0) {
            S.warp_ll[wid] = sll;
            S.warp_pos[wid] = spos;
        }
        __syncthreads();
        if (S.flags) return;  // the bulk copy never completed: status recorded, every thread leaves
        uint32_t d = 0, p = 0, TLL = 0, TP = 0;
        for (uint32_t k = 0; k < kW32; ++k) {
            if (k < wid) {
                d += S.warp_ll[k];
                p += S.warp_pos[k];
            }
            TLL += S.warp_ll[k];
            TP += S.warp_pos[k];
        }
        if (!(TP > w || S.bad)) {
            for (uint32_t ib = i0; ib < i1; ib += 32u) {
                const uint32_t i = ib + lane;
                uint4 q = make_uint4(0u, 0u, 0u, 0u);
                if (i < i1) q = sq[i];
                uint32_t xl = q.y, xp = q.y + q.z;  // inclusive scans over the batch
                for (uint32_t o = 1; o < 32; o <<= 1) {
                    const uint32_t yl = __shfl_up_sync(kFull, xl, o), yp = __shfl_up_sync(kFull, xp, o);
                    if (lane >= o) {
                        xl += yl;
                        xp += yp;
                    }
                }
                const uint32_t my_d = d + xl - q.y, my_p = p + xp - q.y - q.z;
                if (i < i1 && q.x > my_p + q.y) S.bad = 1u;  // match would reach before the window start
                const uint32_t cnt = min(32u, i1 - ib);
                for (uint32_t j = 0; j < cnt; ++j) {
                    const uint32_t rd = __shfl_sync(kFull, my_d, j), rp = __shfl_sync(kFull, my_p, j);
                    const uint32_t rl = __shfl_sync(kFull, q.y, j);
                    for (uint32_t k = lane; k < rl; k += 32u) S.lit[rd + k] = S.win[rp + k];
                }
                d += __shfl_sync(kFull, xl, 31);
                p += __shfl_sync(kFull, xp, 31);
            }
            for (uint32_t k = tid; k < w - TP; k += kGatherThreads) S.lit[TLL + k] = S.win[TP + k];
        }
        __syncthreads();
        if (S.bad) {
            if (tid == 0) {
                atomicOr(a.status, kErrBadSequences);
                write_frame_header(slot, w);
                a.sec_off[b] = 0;  // raw frame
                plan->nlit = 0u;
            }
            __syncthreads();
            continue;
        }
        const uint32_t nlit = TLL + (w - TP);
        const uint32_t rh = raw_lit_header_bytes(nlit);
        uint8_t *dst = slot + fh + 3u + rh;
        uint32_t *myhist = S.hist[wid * 4u + (lane & 3u)];
        for (uint32_t k = tid; k < nlit; k += kGatherThreads) {
            const uint32_t x = S.lit[k];
            dst[k] = static_cast<uint8_t>(x);
            atomicAdd(&myhist[x], 1u);
        }
        if (tid == 0) {
            write_frame_header(slot, w);
            write_raw_lit_header(slot + fh + 3u, 0u, nlit);
            a.sec_off[b] = fh + 3u + rh + nlit;
            plan->nlit = nlit;
        }
        __syncthreads();
        if (tid < 256u) {
            uint32_t c = 0;
            for (uint32_t h = 0; h < kGatherThreads / 32 * 4; ++h) c += S.hist[h][tid];
            a.hist[static_cast<uint64_t>(b) * 256u + tid] = c;
        }
        __syncthreads();
    }
}

// Bits into a byte buffer in shared memory, LSB first.
struct SmemBits {
    uint8_t *p;
    uint32_t cap, pos, nbits;
    uint64_t acc;
    bool ovf;
    __device__ void add(uint32_t v, uint32_t nb) {
        acc |= static_cast<uint64_t>(v) << nbits;
        nbits += nb;
        while (nbits >= 8u) {
            if (pos < cap) p[pos] = static_cast<uint8_t>(acc);
            else ovf = true;
            ++pos;
            acc >>= 8;
            nbits -= 8u;
        }
    }
    __device__ void flush() {  // pad the last partial byte with zeros
        if (nbits) add(0u, 8u - nbits);
    }
    __device__ void close() {  // end marker, then pad
        add(1u, 1u);
        flush();
    }
};

constexpr uint32_t kPlanWarps = 4;

struct PlanSmem {  // one per warp
    uint32_t count[256];
    uint32_t node[511];
    uint32_t bl[64];
    uint32_t start[16];
    uint32_t cw[12];
    uint32_t misc[4];  // [0] tree payload bytes (FSE), [1] ok
    uint16_t leaf[256];
    uint16_t anc[2][512];
    uint16_t code[256];
    uint8_t dep[2][512];
    uint8_t len[256];
    uint8_t tree[132];
    uint8_t wts[256];
    uint8_t st[256];
    uint8_t fsym[64], fnb[64], fbase[64];
    uint8_t fenc[12 * 64];
};

// FSE-compressed weights P.wts[0..N) into P.tree + 1 (lane 0, after the
// parallel steps the caller ran); returns its size, or 0.
__device__ uint32_t plan_fse_weights(PlanSmem &P, uint32_t N) {
    const uint32_t lane = lane_id();
    if (lane < 12u) P.cw[lane] = 0u;
    __syncwarp();
    for (uint32_t i = lane; i < N; i += 32u) atomicAdd(&P.cw[P.wts[i]], 1u);
    __syncwarp();
    int norm[12];
    uint32_t distinct = 0;
    int sum = 0, big = 0;
    for (uint32_t s2 = 0; s2 < 12; ++s2) {
        const uint32_t c = P.cw[s2];
        distinct += c ? 1u : 0u;
        norm[s2] = c ? max(1, static_cast<int>(c * 64u / N)) : 0;
        sum += norm[s2];
        if (norm[s2] > norm[big]) big = static_cast<int>(s2);
    }
    norm[big] += 64 - sum;
    if (distinct < 2u || norm[big] <= 0) return 0;  // warp-uniform
    if (lane == 0) {  // decoder table (no "less than 1" entries, so no high threshold)
        uint32_t pos = 0;
        for (uint32_t s2 = 0; s2 < 12; ++s2)
            for (int c = 0; c < norm[s2]; ++c) {
                P.fsym[pos] = static_cast<uint8_t>(s2);
                pos = (pos + 43u) & 63u;  // step (64 >> 1) + (64 >> 3) + 3
            }
        uint32_t nxt[12];
        for (uint32_t s2 = 0; s2 < 12; ++s2) nxt[s2] = static_cast<uint32_t>(norm[s2]);
        for (uint32_t u = 0; u < 64; ++u) {
            const uint32_t x = nxt[P.fsym[u]]++;
            const uint32_t nb = 6u - highbit(x);
            P.fnb[u] = static_cast<uint8_t>(nb);
            P.fbase[u] = static_cast<uint8_t>((x << nb) - 64u);
        }
    }
    __syncwarp();
    for (uint32_t u = lane; u < 64u; u += 32u) {
        const uint32_t b0 = P.fbase[u], e = b0 + (1u << P.fnb[u]);
        for (uint32_t v = b0; v < e; ++v) P.fenc[P.fsym[u] * 64u + v] = static_cast<uint8_t>(u);
    }
    __syncwarp();
    uint32_t size = 0;
    if (lane == 0) {
        // table description (RFC 8878 4.1.1)
        SmemBits wr{P.tree + 1, 127u, 0u, 0u, 0ull, false};
        wr.add(1u, 4u);  // accuracy 6
        int remaining = 65, threshold = 64;
        uint32_t nb = 7;
        int lastw = 11;
        while (norm[lastw] == 0) --lastw;
        for (int s2 = 0; s2 <= lastw; ++s2) {
            const int v = norm[s2] + 1, mx = (2 * threshold - 1) - remaining;
            if (v < mx) wr.add(static_cast<uint32_t>(v), nb - 1u);
            else if (v < threshold) wr.add(static_cast<uint32_t>(v), nb);
            else wr.add(static_cast<uint32_t>(v + mx), nb);
            remaining -= norm[s2];
            while (remaining < threshold) {
                --nb;
                threshold >>= 1;
            }
            if (norm[s2] == 0) {
                int z = 0;
                while (s2 + 1 + z < lastw && norm[s2 + 1 + z] == 0) ++z;
                s2 += z;
                for (; z >= 3; z -= 3) wr.add(3u, 2u);
                wr.add(static_cast<uint32_t>(z), 2u);
            }
        }
        wr.flush();
        // states: the last two weights pick theirs, the rest follow the chain
        const uint32_t w1 = P.wts[N - 1], w2 = P.wts[N - 2];
        uint32_t s_last = 64, s_prev = 64;
        for (uint32_t u = 0; u < 64; ++u) {
            if (s_last == 64 && P.fsym[u] == w1) s_last = u;
            if (s_prev == 64 && P.fsym[u] == w2 && P.fnb[u] >= 1u) s_prev = u;
        }
        if (s_prev != 64) {
            P.st[N - 1] = static_cast<uint8_t>(s_last);
            P.st[N - 2] = static_cast<uint8_t>(s_prev);
            for (int i = static_cast<int>(N) - 3; i >= 0; --i) P.st[i] = P.fenc[P.wts[i] * 64u + P.st[i + 2]];
            SmemBits bs{P.tree + 1 + wr.pos, 127u > wr.pos ? 127u - wr.pos : 0u, 0u, 0u, 0ull, false};
            for (int i = static_cast<int>(N) - 3; i >= 0; --i) {
                const uint32_t sti = P.st[i];
                bs.add(P.st[i + 2] - P.fbase[sti], P.fnb[sti]);
            }
            bs.add(P.st[1], 6u);
            bs.add(P.st[0], 6u);
            bs.close();
            if (!wr.ovf && !bs.ovf && wr.pos + bs.pos <= 127u) size = wr.pos + bs.pos;
        }
    }
    return __shfl_sync(kFull, size, 0);
}

// One warp per window: the Huffman code of the window's literals.
__global__ void __launch_bounds__(32 * kPlanWarps) zenc_huf_plan_kernel(ZencArgs a) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    PlanSmem &P = reinterpret_cast<PlanSmem *>(smem_raw)[wid];
    for (uint32_t b = blockIdx.x * kPlanWarps + wid; b < a.num_windows; b += gridDim.x * kPlanWarps) {
        PlanRec *plan = reinterpret_cast<PlanRec *>(a.plan + static_cast<uint64_t>(b) * kZencPlanBytes);
        const uint32_t nlit = a.sec_off[b] ? plan->nlit : 0u;
        uint32_t mode = 0;
        if (nlit) {
            const uint32_t *hist = a.hist + static_cast<uint64_t>(b) * 256u;
            // present bytes: ranks by (count, byte); lane l holds bytes 8l .. 8l+7
            uint32_t c8[8];
            uint32_t present = 0, top = 0;
            for (uint32_t i = 0; i < 8; ++i) {
                c8[i] = hist[lane * 8u + i];
                P.count[lane * 8u + i] = c8[i];
                if (c8[i]) {
                    ++present;
                    top = lane * 8u + i;
                }
            }
            uint32_t n = present;
            for (uint32_t o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(kFull, n, o);
            uint32_t last = top;
            for (uint32_t o = 16; o > 0; o >>= 1) last = max(last, __shfl_xor_sync(kFull, last, o));
            __syncwarp();
            if (n == 0u) {
                // nothing counted although the window has literals: keep the raw section
            } else if (n == 1u) {
                mode = 1;
                if (lane == 0) plan->rle = last;
            } else {
                uint32_t r8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                for (uint32_t s2 = 0; s2 < 256; ++s2) {
                    const uint32_t cs = P.count[s2];
                    if (!cs) continue;
                    for (uint32_t i = 0; i < 8; ++i) {
                        const uint32_t me = lane * 8u + i;
                        r8[i] += (cs < c8[i] || (cs == c8[i] && s2 < me)) ? 1u : 0u;
                    }
                }
                for (uint32_t i = 0; i < 8; ++i)
                    if (c8[i]) P.leaf[r8[i]] = static_cast<uint16_t>(lane * 8u + i);
                __syncwarp();
                // two-queue Huffman construction (serial)
                if (lane == 0) {
                    for (uint32_t k = 0; k < n; ++k) P.node[k] = P.count[P.leaf[k]];
                    uint32_t li = 0, ii = n, nxt = n;
                    while (nxt < 2u * n - 1u) {
                        uint32_t pick[2];
                        for (uint32_t t = 0; t < 2; ++t) {
                            if (li < n && (ii >= nxt || P.node[li] <= P.node[ii])) pick[t] = li++;
                            else pick[t] = ii++;
                        }
                        P.node[nxt] = P.node[pick[0]] + P.node[pick[1]];
                        P.anc[0][pick[0]] = P.anc[0][pick[1]] = static_cast<uint16_t>(nxt);
                        ++nxt;
                    }
                }
                __syncwarp();
                // depths by pointer jumping (parent links, the root points to itself)
                const uint32_t nn = 2u * n - 1u, root = nn - 1u;
                for (uint32_t k = lane; k < nn; k += 32u) {
                    if (k == root) P.anc[0][k] = static_cast<uint16_t>(root);
                    P.dep[0][k] = k == root ? 0u : 1u;
                }
                if (lane < 64u) P.bl[lane] = 0u;
                if (lane + 32u < 64u) P.bl[lane + 32u] = 0u;
                __syncwarp();
                uint32_t cur = 0;
                for (uint32_t r = 0; r < 9; ++r) {
                    for (uint32_t k = lane; k < nn; k += 32u) {
                        const uint32_t an = P.anc[cur][k];
                        P.dep[cur ^ 1u][k] = static_cast<uint8_t>(P.dep[cur][k] + P.dep[cur][an]);
                        P.anc[cur ^ 1u][k] = P.anc[cur][an];
                    }
                    __syncwarp();
                    cur ^= 1u;
                }
                for (uint32_t k = lane; k < n; k += 32u) atomicAdd(&P.bl[min(static_cast<uint32_t>(P.dep[cur][k]), 63u)], 1u);
                __syncwarp();
                if (lane == 0) {  // limit to 11 bits, keeping the code complete
                    uint32_t maxlen = 0;
                    for (uint32_t i = 0; i < 64; ++i)
                        if (P.bl[i]) maxlen = i;
                    for (uint32_t i = maxlen; i > kHufMaxBits; --i) {
                        while (P.bl[i] > 0) {
                            uint32_t j = i - 2u;
                            while (P.bl[j] == 0) --j;
                            P.bl[i] -= 2u;
                            P.bl[i - 1] += 1u;
                            P.bl[j + 1] += 2u;
                            P.bl[j] -= 1u;
                        }
                    }
                    uint32_t maxb = 0;
                    for (uint32_t L = kHufMaxBits; L >= 1u && !maxb; --L)
                        if (P.bl[L]) maxb = L;
                    P.start[maxb] = 0;
                    for (uint32_t L = maxb - 1; L >= 1u; --L) P.start[L] = (P.start[L + 1] + P.bl[L + 1]) >> 1;
                    P.start[0] = maxb;
                }
                __syncwarp();
                const uint32_t maxb = P.start[0];
                // lengths: the longest codes to the least frequent bytes
                for (uint32_t i = 0; i < 8; ++i) P.len[lane * 8u + i] = 0;
                __syncwarp();
                for (uint32_t k = lane; k < n; k += 32u) {
                    uint32_t cum = 0;
                    for (uint32_t L = kHufMaxBits; L >= 1u; --L) {
                        if (k < cum + P.bl[L]) {
                            P.len[P.leaf[k]] = static_cast<uint8_t>(L);
                            break;
                        }
                        cum += P.bl[L];
                    }
                }
                __syncwarp();
                // canonical codes: start[L] + rank among the bytes of length L
                uint32_t l8[8];
                for (uint32_t i = 0; i < 8; ++i) l8[i] = P.len[lane * 8u + i];
                for (uint32_t L = 1; L <= maxb; ++L) {
                    uint32_t m = 0;
                    for (uint32_t i = 0; i < 8; ++i) m += l8[i] == L ? 1u : 0u;
                    uint32_t x = m;
                    for (uint32_t dd = 1; dd < 32; dd <<= 1) {
                        const uint32_t y = __shfl_up_sync(kFull, x, dd);
                        if (lane >= dd) x += y;
                    }
                    uint32_t code = P.start[L] + x - m;
                    for (uint32_t i = 0; i < 8; ++i)
                        if (l8[i] == L) P.code[lane * 8u + i] = static_cast<uint16_t>(code++);
                }
                // weights of bytes 0 .. last-1 (the last one's is implied)
                const uint32_t N = last;
                for (uint32_t i = 0; i < 8; ++i) {
                    const uint32_t s2 = lane * 8u + i;
                    if (s2 < N) P.wts[s2] = l8[i] ? static_cast<uint8_t>(maxb + 1u - l8[i]) : 0u;
                }
                __syncwarp();
                uint32_t tree_bytes = 0;
                if (N <= 128u) {
                    if (lane == 0) P.tree[0] = static_cast<uint8_t>(127u + N);
                    for (uint32_t m2 = lane; m2 < (N + 1u) / 2u; m2 += 32u) {
                        const uint32_t hi4 = P.wts[2u * m2], lo4 = 2u * m2 + 1u < N ? P.wts[2u * m2 + 1u] : 0u;
                        P.tree[1u + m2] = static_cast<uint8_t>((hi4 << 4) | lo4);
                    }
                    tree_bytes = 1u + (N + 1u) / 2u;
                } else {
                    const uint32_t f = plan_fse_weights(P, N);
                    if (f) {
                        if (lane == 0) P.tree[0] = static_cast<uint8_t>(f);
                        tree_bytes = 1u + f;
                    }
                }
                __syncwarp();
                if (tree_bytes) {
                    mode = 2;
                    for (uint32_t i = lane; i < 256u; i += 32u) {
                        plan->len[i] = P.len[i];
                        plan->code[i] = P.code[i];
                    }
                    for (uint32_t i = lane; i < tree_bytes; i += 32u) plan->tree[i] = P.tree[i];
                    if (lane == 0) plan->tree_bytes = tree_bytes;
                }
            }
        }
        if (lane == 0) plan->mode = mode;
        __syncwarp();
    }
}

// Literal runs for the Huffman streams: with 4 streams, threads 64s .. 64s+63
// split stream s; with one stream all threads split it.  Run j of a stream
// covers [lo + j*size, lo + (j+1)*size); the stream's bits start with its last
// literal, so the highest run comes first.
struct LitRun {
    uint32_t stream, j, group, lo, hi;
};
__device__ __forceinline__ LitRun lit_run(uint32_t tid, uint32_t nlit, uint32_t nstreams, uint32_t seg) {
    LitRun r;
    r.group = nstreams == 4u ? kLitThreads / 4u : kLitThreads;
    r.stream = tid / r.group;
    r.j = tid % r.group;
    const uint32_t s_lo = r.stream * seg, s_hi = r.stream == nstreams - 1u ? nlit : s_lo + seg;
    const uint32_t size = (s_hi - s_lo + r.group - 1u) / r.group;
    r.lo = min(s_lo + r.j * size, s_hi);
    r.hi = min(r.lo + size, s_hi);
    return r;
}

struct WriteSmem {
    uint8_t len[256];
    uint16_t code[256];
    uint32_t tbits[kLitThreads];
    uint32_t seg_bits[4];
    uint32_t stream_off[4], stream_bytes[4];
    uint32_t mode, nstreams, seg;
};
constexpr uint32_t kWriteSmem = kMaxWindow + sizeof(WriteSmem);

// Writes the codes of lit[hi-1] .. lit[lo] (in that order) at bit `bitpos` of
// the 32-bit-word array `out`; `marker` appends the end-of-stream bit.  Words
// this run shares with a neighbour are ORed in atomically, the others stored.
__device__ void huf_write_run(const WriteSmem &H, const uint8_t *lit, uint32_t lo, uint32_t hi, uint32_t *out,
                              uint64_t bitpos, bool marker) {
    uint64_t word = bitpos >> 5;
    uint32_t nb = static_cast<uint32_t>(bitpos & 31u);
    uint64_t acc = 0;
    bool first = true;
    auto add = [&](uint32_t code, uint32_t len) {
        acc |= static_cast<uint64_t>(code) << nb;
        nb += len;
        if (nb >= 32u) {
            if (first) atomicOr(out + word, static_cast<uint32_t>(acc));
            else out[word] = static_cast<uint32_t>(acc);
            first = false;
            ++word;
            acc >>= 32;
            nb -= 32u;
        }
    };
    for (uint32_t k = hi; k > lo; --k) {
        const uint32_t x = lit[k - 1];
        add(H.code[x], H.len[x]);
    }
    if (marker) add(1u, 1u);
    if (nb) atomicOr(out + word, static_cast<uint32_t>(acc));
}

// One CTA per window: the RLE or Huffman-coded literal section where it is
// smaller than the raw one already in the slot.
__global__ void __launch_bounds__(kLitThreads) zenc_huf_write_kernel(ZencArgs a) {
    extern __shared__ __align__(16) uint8_t lit[];  // kMaxWindow literal bytes, then WriteSmem
    WriteSmem &H = *reinterpret_cast<WriteSmem *>(lit + kMaxWindow);
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    for (uint32_t b = blockIdx.x; b < a.num_windows; b += gridDim.x) {
        const PlanRec *plan = reinterpret_cast<const PlanRec *>(a.plan + static_cast<uint64_t>(b) * kZencPlanBytes);
        if (a.sec_off[b] == 0u) continue;  // raw frame (uniform over the CTA)
        const uint32_t mode = plan->mode;
        if (mode == 0u) continue;
        const uint32_t w = win_size(a, b);
        const uint32_t fh = frame_header_bytes(w), L0 = fh + 3u;
        const uint32_t nlit = plan->nlit, rh = raw_lit_header_bytes(nlit);
        uint8_t *slot = a.slots + static_cast<uint64_t>(b) * kZencSlot;
        if (mode == 1u) {
            if (tid == 0) {
                write_raw_lit_header(slot + L0, 1u, nlit);
                slot[L0 + rh] = static_cast<uint8_t>(plan->rle);
                a.sec_off[b] = L0 + rh + 1u;
            }
            continue;
        }
        // Huffman: the literals back from the raw section, the code from the plan
        const uint8_t *rawp = slot + L0 + rh;
        for (uint32_t k = tid; k < nlit; k += kLitThreads) lit[k] = rawp[k];
        H.len[tid] = plan->len[tid];
        H.code[tid] = plan->code[tid];
        if (tid < 4u) H.seg_bits[tid] = 0u;
        __syncthreads();
        const uint32_t nst = nlit < 1024u ? 1u : 4u;
        const uint32_t seg = nlit < 1024u ? nlit : (nlit + 3u) / 4u;
        const LitRun run = lit_run(tid, nlit, nst, seg);
        uint32_t v = 0;
        for (uint32_t k = run.lo; k < run.hi; ++k) v += H.len[lit[k]];
        H.tbits[tid] = v;
        uint32_t t = v;
        for (uint32_t o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
        if (lane == 0 && t) atomicAdd(&H.seg_bits[run.stream], t);
        __syncthreads();
        if (tid == 0) {
            const uint32_t tree_bytes = plan->tree_bytes;
            uint32_t streams = 0;
            for (uint32_t s2 = 0; s2 < nst; ++s2) {
                H.stream_bytes[s2] = (H.seg_bits[s2] + 8u) >> 3;  // + end marker, rounded up
                streams += H.stream_bytes[s2];
            }
            const uint32_t body = tree_bytes + (nst == 4u ? 6u : 0u) + streams;
            const uint32_t hdr = nst == 1u ? 3u : (max(nlit, body) < 16384u ? 4u : 5u);
            H.mode = 0;
            if (!((nst == 1u && body >= 1024u) || hdr + body >= rh + nlit)) {
                H.mode = 2;
                H.nstreams = nst;
                uint64_t hv;
                if (hdr == 3u) hv = 2u | (static_cast<uint64_t>(nlit) << 4) | (static_cast<uint64_t>(body) << 14);
                else if (hdr == 4u) hv = 2u | (2u << 2) | (static_cast<uint64_t>(nlit) << 4) | (static_cast<uint64_t>(body) << 18);
                else hv = 2u | (3u << 2) | (static_cast<uint64_t>(nlit) << 4) | (static_cast<uint64_t>(body) << 22);
                uint8_t *h = slot + L0;
                for (uint32_t i = 0; i < hdr; ++i) h[i] = static_cast<uint8_t>(hv >> (8u * i));
                for (uint32_t i = 0; i < tree_bytes; ++i) h[hdr + i] = plan->tree[i];
                uint32_t o = L0 + hdr + tree_bytes;
                if (nst == 4u) {
                    for (uint32_t s2 = 0; s2 < 3; ++s2) {
                        slot[o + 2 * s2] = static_cast<uint8_t>(H.stream_bytes[s2]);
                        slot[o + 2 * s2 + 1] = static_cast<uint8_t>(H.stream_bytes[s2] >> 8);
                    }
                    o += 6u;
                }
                for (uint32_t s2 = 0; s2 < nst; ++s2) {
                    H.stream_off[s2] = o;
                    o += H.stream_bytes[s2];
                }
                a.sec_off[b] = o;
            }
        }
        __syncthreads();
        if (H.mode == 2u) {
            // The streams' bytes start at zero (runs OR their shared words in); the
            // bytes of the headers before them are kept.
            const uint32_t s0b = H.stream_off[0];
            const uint32_t s1b = H.stream_off[nst - 1u] + H.stream_bytes[nst - 1u];
            uint32_t *wslot = reinterpret_cast<uint32_t *>(slot);
            const uint32_t w0 = (s0b + 3u) >> 2, w1 = (s1b + 3u) >> 2;
            for (uint32_t k = s0b + tid; k < min(w0 * 4u, s1b); k += kLitThreads) slot[k] = 0;
            for (uint32_t k = w0 + tid; k < w1; k += kLitThreads) wslot[k] = 0u;
            __syncthreads();
            // bit offset of this run: the runs after it in the stream come first
            uint32_t off = 0;
            for (uint32_t j2 = run.j + 1u; j2 < run.group; ++j2) off += H.tbits[run.stream * run.group + j2];
            const uint64_t bitpos = 8ull * H.stream_off[run.stream] + off;
            if (run.hi > run.lo || run.j == 0u) huf_write_run(H, lit, run.lo, run.hi, wslot, bitpos, run.j == 0u);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- sequences
// One warp per window, kSeqWarps windows per CTA.  Sequences pass through
// shared memory in chunks of kChunk; the only serial work -- the
// repeat-offset history, the three tables and the three FSE state chains --
// runs on single lanes over shared memory, the rest is spread over the warp:
//   R. ascending chunks: lane 0 computes each Offset_Value from the decoder's
//      repeat history; the values go to a per-window global scratch; the
//      lanes count the LL, ML and OF codes.
//   T. lanes 0-2 pick the table of LL, OF and ML (RFC 8878 3.1.1.3.2.1):
//      RLE_Mode when one code is used, else FSE_Compressed_Mode or
//      Predefined_Mode, whichever costs fewer bits by an integer estimate
//      (below); then spread the table and list each code's states.
//   E. descending chunks (the bitstream starts with the last sequence):
//      codes in parallel; lanes 0-2 run the LL / ML / OF chains; a warp scan
//      gives each sequence's bit position; every lane ORs its sequences'
//      fields into the warp's bit buffer; whole 32-bit words are stored, the
//      partial last word carries into the next chunk.
// The cost estimate counts, per code c used k times, k * (A - log2(n_c))
// bits, with log2 taken piecewise linear between powers of two in 1/256 bit
// (lg256 below), plus the table description's bytes.  FSE_Compressed_Mode
// uses accuracy A = max(5, min(Amax, bitlen(ns - 1) - 2)), raised until the
// table has two states per used code (Amax: 9 for LL and ML, 8 for OF), and
// counts normalised to 2^A by rounding k * 2^A / ns (at least 1); the most
// used code takes a positive remainder, a negative one is taken one state at a
// time from the largest count (lowest code first on ties).
// The encoder of any table follows from its decoder (RFC 8878 4.1.1): code c
// with normalised count n owns, in ascending decoder-state order, the states
// numbered x = n .. 2n-1; for the next decoder state D' the encoder takes the
// state x = (D' + 2^A) >> b, with b the bit count that puts x in [n, 2n), and
// writes the low b bits of D' + 2^A.
constexpr uint32_t kChunk = 128;
constexpr uint32_t kSeqWarps = 4;
constexpr uint32_t kPerLane = kChunk / 32;
constexpr uint32_t kBufWords = kChunk * 74u / 32u + 4u;  // <= 74 bits per sequence, plus the carried word
constexpr uint32_t kMaxAl = 9;                           // Accuracy_Log limit of LL and ML (OF: 8)
constexpr uint32_t kTabDesc = 128;                       // bytes of one table description
constexpr uint32_t kOFCodes = 32;                        // offset codes counted (a window's are <= 16)

// One field's (LL, ML or OF) table for one window.
struct FieldTab {
    uint16_t stl[1u << kMaxAl];  // each code's decoder states, ascending, code after code
    uint8_t sym[1u << kMaxAl];   // spread table (building only)
    uint16_t cumul[64];          // first stl entry of code c
    uint16_t norm[64];           // normalised count (>= 1 where used; "less than 1" counts as 1)
    uint32_t hist[64];           // uses of code c in the window
    uint8_t desc[kTabDesc];      // FSE table description, or the RLE code
    uint32_t al;                 // accuracy log (0 for RLE_Mode)
    uint32_t mode;               // 0 Predefined_Mode, 1 RLE_Mode, 2 FSE_Compressed_Mode
    uint32_t desc_len;
};

struct WarpSeq {
    uint4 q[kChunk];          // the chunk's records, in bitstream order (last sequence first)
    uint32_t ov[kChunk];      // Offset_Value
    uint8_t code[3][kChunk];  // LL, ML, OF codes
    uint16_t upd[3][kChunk];  // state-update bits: value | nbBits << 12 (LL, ML, OF)
    uint32_t pos[kChunk];     // bit position within the chunk
    uint32_t buf[kBufWords];
    uint32_t state[3];
    FieldTab tab[3];          // LL, ML, OF
};

struct SeqSmem {
    CodeTables C;
    WarpSeq W[kSeqWarps];
};
static_assert(sizeof(SeqSmem) * 4 + 4 * 1024 <= 233472, "four sequence CTAs per SM");

// log2(x) * 256, piecewise linear between powers of two (x >= 1).
__device__ __forceinline__ uint32_t lg256(uint32_t x) {
    const uint32_t h = highbit(x);
    return 256u * h + ((x << 8) >> h) - 256u;
}

// Picks and builds field f's table from its code histogram (one lane).
// pre: the predefined distribution (-1 = "less than 1"), pre_n codes.
__device__ void build_field_table(FieldTab &T, uint32_t ns, uint32_t ncodes, uint32_t amax, const int8_t *pre,
                                  uint32_t pre_n, uint32_t pre_al) {
    uint32_t used = 0, last = 0;
    for (uint32_t c = 0; c < ncodes; ++c)
        if (T.hist[c]) {
            ++used;
            last = c;
        }
    if (used == 1u) {  // RLE_Mode: one code, no state
        T.mode = 1;
        T.al = 0;
        T.desc[0] = static_cast<uint8_t>(last);
        T.desc_len = 1;
        return;
    }
    // Predefined cost (impossible when a used code has no predefined state).
    uint64_t cost_pre = 0;
    bool pre_ok = true;
    for (uint32_t c = 0; c <= last; ++c) {
        if (!T.hist[c]) continue;
        if (c >= pre_n || pre[c] == 0) {
            pre_ok = false;
            break;
        }
        const uint32_t n = pre[c] < 0 ? 1u : static_cast<uint32_t>(pre[c]);
        cost_pre += static_cast<uint64_t>(T.hist[c]) * (256u * pre_al - lg256(n));
    }
    // FSE_Compressed_Mode: accuracy, normalised counts, description.
    uint32_t al = 32u - static_cast<uint32_t>(__clz(ns - 1u));  // bit length of ns - 1
    al = al > 2u ? al - 2u : 0u;
    al = al < amax ? al : amax;
    al = al > 5u ? al : 5u;
    while ((1u << al) < 2u * used && al < amax) ++al;
    const uint32_t size = 1u << al;
    int32_t sum = 0;
    uint32_t top = 0;
    for (uint32_t c = 0; c < 64u; ++c) {
        uint32_t n = 0;
        if (c <= last && T.hist[c]) {
            n = (T.hist[c] * size + ns / 2u) / ns;
            n = n > 1u ? n : 1u;
            if (T.hist[c] > T.hist[top]) top = c;
        }
        T.norm[c] = static_cast<uint16_t>(n);
        sum += static_cast<int32_t>(n);
    }
    int32_t d = static_cast<int32_t>(size) - sum;
    if (d > 0) T.norm[top] = static_cast<uint16_t>(T.norm[top] + d);
    for (; d < 0; ++d) {
        uint32_t big = 0;
        for (uint32_t c = 1; c <= last; ++c)
            if (T.norm[c] > T.norm[big]) big = c;
        T.norm[big] = static_cast<uint16_t>(T.norm[big] - 1u);
    }
    SmemBits wr{T.desc, kTabDesc, 0u, 0u, 0ull, false};
    {
        wr.add(al - 5u, 4u);
        int remaining = static_cast<int>(size) + 1, threshold = static_cast<int>(size);
        uint32_t nb = al + 1u;
        for (int c = 0; c <= static_cast<int>(last); ++c) {
            const int n = T.norm[c];
            const int v = n + 1, mx = (2 * threshold - 1) - remaining;
            if (v < mx) wr.add(static_cast<uint32_t>(v), nb - 1u);
            else if (v < threshold) wr.add(static_cast<uint32_t>(v), nb);
            else wr.add(static_cast<uint32_t>(v + mx), nb);
            remaining -= n;
            while (remaining < threshold) {
                --nb;
                threshold >>= 1;
            }
            if (n == 0) {
                int z = 0;
                while (c + 1 + z < static_cast<int>(last) && T.norm[c + 1 + z] == 0) ++z;
                c += z;
                for (; z >= 3; z -= 3) wr.add(3u, 2u);
                wr.add(static_cast<uint32_t>(z), 2u);
            }
        }
        wr.flush();
    }
    uint64_t cost_fse = 2048ull * wr.pos;
    for (uint32_t c = 0; c <= last; ++c)
        if (T.hist[c]) cost_fse += static_cast<uint64_t>(T.hist[c]) * (256u * al - lg256(T.norm[c]));
    const bool fse = !wr.ovf && (!pre_ok || cost_fse < cost_pre);
    uint32_t high = 0;
    if (fse) {
        T.mode = 2;
        T.al = al;
        T.desc_len = wr.pos;
        high = size - 1u;
    } else {  // Predefined_Mode
        T.mode = 0;
        T.al = pre_al;
        T.desc_len = 0;
        high = (1u << pre_al) - 1u;
        for (uint32_t c = 0; c < 64u; ++c) T.norm[c] = c < pre_n ? static_cast<uint16_t>(pre[c] < 0 ? 1 : pre[c]) : 0;
    }
    // Spread (RFC 8878 4.1.1): "less than 1" codes at the top, the others
    // stepped through the remaining states.
    const uint32_t tsize = 1u << T.al, mask = tsize - 1u, step = (tsize >> 1) + (tsize >> 3) + 3u;
    const uint32_t ntab = fse ? last + 1u : pre_n;
    for (uint32_t c = 0; c < ntab; ++c)
        if (!fse && pre[c] < 0) T.sym[high--] = static_cast<uint8_t>(c);
    uint32_t pos = 0;
    for (uint32_t c = 0; c < ntab; ++c) {
        const int n = fse ? static_cast<int>(T.norm[c]) : static_cast<int>(pre[c]);
        for (int i = 0; i < n; ++i) {
            T.sym[pos] = static_cast<uint8_t>(c);
            do {
                pos = (pos + step) & mask;
            } while (pos > high);
        }
    }
    uint32_t acc = 0;
    for (uint32_t c = 0; c < 64u; ++c) {
        T.cumul[c] = static_cast<uint16_t>(acc);
        acc += T.norm[c];
    }
    uint16_t fill[64];
    for (uint32_t c = 0; c < 64u; ++c) fill[c] = T.cumul[c];
    for (uint32_t u = 0; u < tsize; ++u) T.stl[fill[T.sym[u]]++] = static_cast<uint16_t>(u);
}

// Decoder state before code c when the next decoder state is dn: the state
// and, in `up`, the bits the decoder reads (value | count << 12).
__device__ __forceinline__ uint32_t fse_encode(const FieldTab &T, uint32_t c, uint32_t dn, uint16_t &up) {
    const uint32_t n = T.norm[c], v = dn + (1u << T.al);
    const uint32_t hi = T.al - highbit(n);
    const uint32_t nb = v >= (n << hi) ? hi : hi - 1u;
    const uint32_t x = v >> nb;
    up = static_cast<uint16_t>((v - (x << nb)) | (nb << 12));
    return T.stl[T.cumul[c] + x - n];
}

__device__ __forceinline__ void or_bits(uint32_t *buf, uint32_t bitpos, uint64_t v, uint32_t nb) {
    if (nb == 0u) return;
    const uint32_t w = bitpos >> 5, sh = bitpos & 31u;
    const uint64_t lo = v << sh;  // nb <= 48, so v << sh spans at most 80 bits: three words
    atomicOr(buf + w, static_cast<uint32_t>(lo));
    if (sh + nb > 32u) atomicOr(buf + w + 1, static_cast<uint32_t>(lo >> 32));
    if (sh + nb > 64u) atomicOr(buf + w + 2, static_cast<uint32_t>(v >> (64u - sh)));
}

// Returns the frame's block content size, or 0 when a raw block is smaller.
__device__ uint32_t encode_sequences_warp(const ZencArgs &a, const SeqSmem &G, WarpSeq &S, uint32_t b, uint32_t w,
                                          uint32_t fh, uint8_t *slot, uint32_t sec) {
    const uint32_t lane = lane_id();
    const uint64_t s0 = a.seq_offsets[b];
    const uint32_t ns = static_cast<uint32_t>(a.seq_offsets[b + 1] - s0);
    const uint4 *sq = a.seqs + s0;
    uint32_t *ovg = a.ovs + static_cast<uint64_t>(b) * kZencMaxSeqs;

    for (uint32_t k = lane; k < 64u; k += 32u) S.tab[0].hist[k] = S.tab[1].hist[k] = S.tab[2].hist[k] = 0u;
    __syncwarp();
    // ---- R: Offset_Values, ascending, with the decoder's repeat history (lane 0); code counts
    uint32_t r1 = 1, r2 = 4, r3 = 8;
    for (uint32_t lo = 0; lo < ns; lo += kChunk) {
        const uint32_t len = min(kChunk, ns - lo);
        for (uint32_t k = lane; k < len; k += 32u) {
            const uint4 q = sq[lo + k];
            S.pos[k] = q.x;               // offset
            S.ov[k] = q.y == 0u ? 1u : 0u;  // literal length is zero
            atomicAdd(&S.tab[0].hist[G.C.ll_code(q.y)], 1u);
            atomicAdd(&S.tab[1].hist[G.C.ml_code(q.z)], 1u);
        }
        __syncwarp();
        if (lane == 0) {
            for (uint32_t k = 0; k < len; ++k) {
                const uint32_t o = S.pos[k], z = S.ov[k];
                uint32_t v;
                if (!z) v = o == r1 ? 1u : (o == r2 ? 2u : (o == r3 ? 3u : o + 3u));
                else v = o == r2 ? 1u : (o == r3 ? 2u : (o == r1 - 1u ? 3u : o + 3u));
                const uint32_t idx = v > 3u ? 3u : v - 1u + z;
                // idx 0: rep1 kept; 1: rep2 swapped to the front; else: o in front, the rest shift
                if (idx == 1u) {
                    r2 = r1;
                    r1 = o;
                } else if (idx >= 2u) {
                    r3 = r2;
                    r2 = r1;
                    r1 = o;
                }
                S.ov[k] = v;
            }
        }
        __syncwarp();
        for (uint32_t k = lane; k < len; k += 32u) {
            ovg[lo + k] = S.ov[k];
            atomicAdd(&S.tab[2].hist[highbit(S.ov[k])], 1u);
        }
        __syncwarp();
    }

    // ---- T: the three tables (lane 0: LL, lane 1: ML, lane 2: OF)
    if (lane == 0) build_field_table(S.tab[0], ns, kLLSyms, kMaxAl, kLLNorm, kLLSyms, kLLLog);
    else if (lane == 1) build_field_table(S.tab[1], ns, kMLSyms, kMaxAl, kMLNorm, kMLSyms, kMLLog);
    else if (lane == 2) build_field_table(S.tab[2], ns, kOFCodes, 8u, kOFNorm, kOFSyms, kOFLog);
    __syncwarp();

    // ---- header: Number_of_Sequences, modes, table descriptions (LL, OF, ML)
    uint8_t *hp = slot + sec;
    const uint32_t nsb = ns < 128u ? 1u : 2u;
    const uint32_t d_ll = S.tab[0].desc_len, d_of = S.tab[2].desc_len, d_ml = S.tab[1].desc_len;
    const uint32_t hl = nsb + 1u + d_ll + d_of + d_ml;
    if (lane == 0) {
        if (ns < 128u) {
            hp[0] = static_cast<uint8_t>(ns);
        } else {
            hp[0] = static_cast<uint8_t>((ns >> 8) + 0x80u);
            hp[1] = static_cast<uint8_t>(ns);
        }
        hp[nsb] = static_cast<uint8_t>((S.tab[0].mode << 6) | (S.tab[2].mode << 4) | (S.tab[1].mode << 2));
    }
    for (uint32_t k = lane; k < d_ll + d_of + d_ml; k += 32u) {
        const uint8_t v = k < d_ll ? S.tab[0].desc[k]
                                   : (k < d_ll + d_of ? S.tab[2].desc[k - d_ll] : S.tab[1].desc[k - d_ll - d_of]);
        hp[nsb + 1u + k] = v;
    }
    uint8_t *bs = hp + hl;
    // bitstream bytes at which the block stops paying (none when the literals alone fill the window)
    const int32_t room = static_cast<int32_t>(fh + 3u + w) - static_cast<int32_t>(sec + hl);
    if (room <= 0) return 0u;
    uint32_t carry_word = 0, carry_bits = 0, out_pos = 0;
    uint32_t D = 0;  // chain state of lanes 0-2
    for (uint32_t hi = ns; hi > 0u;) {
        const uint32_t lo = hi > kChunk ? hi - kChunk : 0u, len = hi - lo;
        // codes, in bitstream order j (sequence hi - 1 - j)
        for (uint32_t j = lane; j < len; j += 32u) {
            const uint32_t i = hi - 1u - j;
            const uint4 q = sq[i];
            const uint32_t v = ovg[i];
            S.q[j] = q;
            S.ov[j] = v;
            S.code[0][j] = static_cast<uint8_t>(G.C.ll_code(q.y));
            S.code[1][j] = static_cast<uint8_t>(G.C.ml_code(q.z));
            S.code[2][j] = static_cast<uint8_t>(highbit(v));
        }
        for (uint32_t k = lane; k < kBufWords; k += 32u) S.buf[k] = 0u;
        __syncwarp();
        if (lane < 3u) {  // the three FSE chains
            const FieldTab &T = S.tab[lane];
            const uint8_t *cd = S.code[lane];
            uint16_t *up = S.upd[lane];
            uint32_t j = 0;
            if (T.mode == 1u) {  // RLE_Mode: no state, no bits
                for (; j < len; ++j) up[j] = 0;
            } else {
                if (hi == ns) {  // last sequence: any state of its code, no bits
                    uint16_t dummy;
                    D = fse_encode(T, cd[0], 0u, dummy);
                    up[0] = 0;
                    j = 1;
                }
                for (; j < len; ++j) D = fse_encode(T, cd[j], D, up[j]);
            }
        }
        __syncwarp();
        // bit widths and their exclusive scan (each lane: kPerLane consecutive j)
        uint32_t wsum = 0;
        const uint32_t j0 = lane * kPerLane;
        for (uint32_t u = 0; u < kPerLane; ++u) {
            const uint32_t j = j0 + u;
            uint32_t nb = 0;
            if (j < len) {
                nb = (S.upd[0][j] >> 12) + (S.upd[1][j] >> 12) + (S.upd[2][j] >> 12) + G.C.ll_bits[S.code[0][j]] +
                     G.C.ml_bits[S.code[1][j]] + S.code[2][j];
            }
            S.pos[j] = wsum;
            wsum += nb;
        }
        uint32_t x = wsum;
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, x, d);
            if (lane >= d) x += y;
        }
        const uint32_t chunk_bits = __shfl_sync(kFull, x, 31);
        const uint32_t base = carry_bits + x - wsum;
        if (lane == 0) S.buf[0] = carry_word;
        __syncwarp();
        for (uint32_t u = 0; u < kPerLane; ++u) {
            const uint32_t j = j0 + u;
            if (j >= len) break;
            const uint32_t p0 = base + S.pos[j];
            // updates: OF, ML, LL (the decoder, reading backwards, takes LL, ML, OF)
            const uint32_t uo = S.upd[2][j], um = S.upd[1][j], ul = S.upd[0][j];
            const uint32_t no = uo >> 12, nm = um >> 12, nl = ul >> 12;
            const uint64_t ga = static_cast<uint64_t>(uo & 0xFFFu) | (static_cast<uint64_t>(um & 0xFFFu) << no) |
                                (static_cast<uint64_t>(ul & 0xFFFu) << (no + nm));
            or_bits(S.buf, p0, ga, no + nm + nl);
            // extra bits: LL, ML, OF
            const uint4 q = S.q[j];
            const uint32_t lc = S.code[0][j], mc = S.code[1][j], oc = S.code[2][j];
            const uint32_t lb = G.C.ll_bits[lc], mb = G.C.ml_bits[mc];
            const uint64_t gb = static_cast<uint64_t>(q.y - G.C.ll_base[lc]) |
                                (static_cast<uint64_t>(q.z - G.C.ml_base[mc]) << lb) |
                                (static_cast<uint64_t>(S.ov[j] - (1u << oc)) << (lb + mb));
            or_bits(S.buf, p0 + no + nm + nl, gb, lb + mb + oc);
        }
        __syncwarp();
        // store the whole words; the partial one carries over
        const uint32_t total = carry_bits + chunk_bits, nfull = total >> 5;
        if (static_cast<int32_t>(out_pos + 4u * nfull) >= room) return 0u;  // warp-uniform
        for (uint32_t k = lane; k < 4u * nfull; k += 32u)
            bs[out_pos + k] = static_cast<uint8_t>(S.buf[k >> 2] >> ((k & 3u) * 8u));
        carry_word = S.buf[nfull];
        carry_bits = total & 31u;
        out_pos += 4u * nfull;
        __syncwarp();
        hi = lo;
    }
    if (lane < 3u) S.state[lane] = D;
    __syncwarp();
    uint32_t content = 0;
    if (lane == 0) {
        BitWriter bw{bs, out_pos, carry_word, carry_bits};
        bw.add(S.state[1], S.tab[1].al);
        bw.add(S.state[2], S.tab[2].al);
        bw.add(S.state[0], S.tab[0].al);
        bw.close();
        content = sec + hl + bw.pos - (fh + 3u);
    }
    content = __shfl_sync(kFull, content, 0);
    return content < w ? content : 0u;
}

__global__ void __launch_bounds__(32 * kSeqWarps) zenc_sequences_kernel(ZencArgs a) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    SeqSmem &G = *reinterpret_cast<SeqSmem *>(smem_raw);
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    G.C.build();
    __syncthreads();
    for (uint32_t b = blockIdx.x * kSeqWarps + wid; b < a.num_windows; b += gridDim.x * kSeqWarps) {
        const uint32_t w = win_size(a, b);
        const uint32_t fh = frame_header_bytes(w);
        uint8_t *slot = a.slots + static_cast<uint64_t>(b) * kZencSlot;
        const uint32_t sec = a.sec_off[b];
        const uint32_t content = sec != 0u ? encode_sequences_warp(a, G, G.W[wid], b, w, fh, slot, sec) : 0u;
        if (lane == 0) {
            if (content) {
                write_block_header(slot + fh, 2u, content);
                a.fsize[b] = fh + 3u + content;
                a.raw[b] = 0;
            } else {
                write_block_header(slot + fh, 0u, w);
                a.fsize[b] = fh + 3u + w;
                a.raw[b] = 1;
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------- compaction
__global__ void __launch_bounds__(256) zenc_compact_kernel(ZencArgs a, const uint64_t *foff, uint8_t *out,
                                                           uint64_t capacity) {
    const uint32_t tid = threadIdx.x;
    for (uint32_t b = blockIdx.x; b < a.num_windows; b += gridDim.x) {
        const uint64_t o = foff[b], size = foff[b + 1] - o;
        if (o + size > capacity) {
            if (tid == 0) atomicOr(a.status, kErrCapacity);
            continue;
        }
        const uint8_t *slot = a.slots + static_cast<uint64_t>(b) * kZencSlot;
        uint8_t *dst = out + o;
        if (!a.raw[b]) {
            cta_copy(dst, slot, static_cast<uint32_t>(size));
        } else {
            const uint32_t w = win_size(a, b);
            const uint32_t hl = frame_header_bytes(w) + 3u;
            cta_copy(dst, slot, hl);
            cta_copy(dst + hl, win_src(a, b), w);
        }
    }
}

ZencArgs args_of(const ZencLaunch &l) {
    ZencArgs a{};
    a.src = l.src;
    a.n = l.n;
    a.window = l.window;
    a.num_windows = l.num_windows;
    a.seqs = reinterpret_cast<const uint4 *>(l.seqs);
    a.seq_offsets = l.seq_offsets;
    a.slots = l.slots;
    a.ovs = l.ovs;
    a.sec_off = l.sec_off;
    a.fsize = l.fsize;
    a.raw = l.raw;
    a.hist = l.hist;
    a.plan = l.plan;
    a.status = l.status;
    a.wins = l.wins;
    return a;
}

SmemOnce g_lit_smem_set{0}, g_seq_smem_set{0}, g_plan_smem_set{0}, g_write_smem_set{0};

}  // namespace

cudaError_t launch_zenc(const ZencLaunch &l, cudaStream_t st) {
    if (l.num_windows == 0) return cudaSuccess;
    const ZencArgs a = args_of(l);
    cudaError_t e = set_smem_once(zenc_literals_kernel, sizeof(GatherSmem), g_lit_smem_set);
    if (e != cudaSuccess) return e;
    if ((e = set_smem_once(zenc_huf_plan_kernel, sizeof(PlanSmem) * kPlanWarps, g_plan_smem_set)) != cudaSuccess)
        return e;
    if ((e = set_smem_once(zenc_huf_write_kernel, kWriteSmem, g_write_smem_set)) != cudaSuccess) return e;
    int grid = l.num_sms;  // one 512-thread CTA per SM (window + literals in shared memory)
    if (static_cast<uint32_t>(grid) > l.num_windows) grid = static_cast<int>(l.num_windows);
    zenc_literals_kernel<<<grid, kGatherThreads, sizeof(GatherSmem), st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    grid = l.num_sms * 3;
    if (static_cast<uint32_t>(grid) > l.num_windows) grid = static_cast<int>(l.num_windows);
    uint32_t pgrid = (l.num_windows + kPlanWarps - 1) / kPlanWarps;
    if (pgrid > static_cast<uint32_t>(l.num_sms * 5)) pgrid = static_cast<uint32_t>(l.num_sms * 5);
    zenc_huf_plan_kernel<<<pgrid, 32 * kPlanWarps, sizeof(PlanSmem) * kPlanWarps, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    zenc_huf_write_kernel<<<grid, kLitThreads, kWriteSmem, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = set_smem_once(zenc_sequences_kernel, sizeof(SeqSmem), g_seq_smem_set)) != cudaSuccess) return e;
    grid = l.num_sms * 4;  // 4 CTAs of ~56 KB per SM
    const uint32_t need = (l.num_windows + kSeqWarps - 1) / kSeqWarps;
    if (static_cast<uint32_t>(grid) > need) grid = static_cast<int>(need);
    zenc_sequences_kernel<<<grid, 32 * kSeqWarps, sizeof(SeqSmem), st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_zenc_compact(const ZencLaunch &l, const uint64_t *frame_offsets, uint8_t *out, uint64_t capacity,
                                cudaStream_t st) {
    if (l.num_windows == 0) return cudaSuccess;
    int grid = l.num_sms * 8;
    if (static_cast<uint32_t>(grid) > l.num_windows) grid = static_cast<int>(l.num_windows);
    zenc_compact_kernel<<<grid, 256, 0, st>>>(args_of(l), frame_offsets, out, capacity);
    return cudaGetLastError();
}

}  // namespace gcz
