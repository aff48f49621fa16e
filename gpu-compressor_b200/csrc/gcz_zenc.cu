// Zstd entropy stage on the GPU: one Zstd frame per 64 KiB window, built from
// the window's ZSTD_Sequence records, decodable by any conforming decoder
// (stock libzstd).
//
// Frame layout (RFC 8878): magic, a single-segment frame header with the
// content size, and one block.  The block is a compressed block when that is
// smaller than the window, else a raw block.  A compressed block holds
//   - a Raw_Literals_Block with every literal byte of the window, in order;
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
//   zenc_literals_kernel   (one CTA):    frame header, literal section
//   zenc_sequences_kernel  (one thread): repeat-code pass, FSE chains, bitstream,
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

// Encoder tables in shared memory: enc[s * size + v] = D | nbBits(D) << 8 | baseline(D) << 16
// for the state D of symbol s whose interval holds decoder state v.
struct FseEnc {
    uint32_t ll[kLLSyms << kLLLog];
    uint32_t ml[kMLSyms << kMLLog];
    uint32_t of[kOFSyms << kOFLog];
    uint8_t sym[64];
    uint8_t nbits[64];
    uint16_t base[64];
};

// Decoder table of a normalised distribution (RFC 8878 4.1.1: symbol spread,
// then nbBits / baseline per state), turned into the encoder table above.
__device__ void build_fse(FseEnc &t, const int8_t *norm, uint32_t nsym, uint32_t al, uint32_t *enc) {
    const uint32_t size = 1u << al;
    if (threadIdx.x == 0) {
        const uint32_t mask = size - 1u, step = (size >> 1) + (size >> 3) + 3u;
        uint32_t high = size - 1u;
        uint16_t next[64];
        for (uint32_t s = 0; s < nsym; ++s) {
            if (norm[s] == -1) {
                t.sym[high--] = static_cast<uint8_t>(s);
                next[s] = 1;
            } else {
                next[s] = static_cast<uint16_t>(norm[s]);
            }
        }
        uint32_t pos = 0;
        for (uint32_t s = 0; s < nsym; ++s) {
            for (int i = 0; i < norm[s]; ++i) {
                t.sym[pos] = static_cast<uint8_t>(s);
                do {
                    pos = (pos + step) & mask;
                } while (pos > high);
            }
        }
        for (uint32_t u = 0; u < size; ++u) {
            const uint32_t x = next[t.sym[u]]++;
            const uint32_t nb = al - highbit(x);
            t.nbits[u] = static_cast<uint8_t>(nb);
            t.base[u] = static_cast<uint16_t>((x << nb) - size);
        }
    }
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < size; u += blockDim.x) {
        const uint32_t s = t.sym[u], nb = t.nbits[u], b = t.base[u];
        const uint32_t e = u | (nb << 8) | (b << 16);
        for (uint32_t v = b; v < b + (1u << nb); ++v) enc[s * size + v] = e;
    }
    __syncthreads();
}

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
    uint32_t *status;
};

__device__ __forceinline__ uint32_t win_size(const ZencArgs &a, uint32_t b) {
    const uint64_t s = static_cast<uint64_t>(b) * a.window;
    return static_cast<uint32_t>(a.n - s < a.window ? a.n - s : a.window);
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

// ---------------------------------------------------------------- literals
__global__ void __launch_bounds__(kLitThreads) zenc_literals_kernel(ZencArgs a) {
    extern __shared__ __align__(16) uint8_t lit[];  // kMaxWindow bytes
    __shared__ uint32_t warp_ll[kLitThreads / 32], warp_pos[kLitThreads / 32];
    __shared__ uint32_t tot_ll, tot_pos, bad;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
    for (uint32_t b = blockIdx.x; b < a.num_windows; b += gridDim.x) {
        const uint32_t w = win_size(a, b);
        const uint8_t *src = a.src + static_cast<uint64_t>(b) * a.window;
        const uint64_t s0 = a.seq_offsets[b];
        const uint32_t ns = static_cast<uint32_t>(a.seq_offsets[b + 1] - s0);
        const uint4 *sq = a.seqs + s0;
        uint8_t *slot = a.slots + static_cast<uint64_t>(b) * kZencSlot;
        if (tid == 0) bad = ns > kZencMaxSeqs ? 1u : 0u;
        __syncthreads();
        // Each thread owns a contiguous run of sequences; a block scan gives
        // its first literal's output index and source position.
        const uint32_t per = (ns + kLitThreads - 1) / kLitThreads;
        const uint32_t i0 = min(tid * per, ns), i1 = min(i0 + per, ns);
        uint32_t sll = 0, spos = 0;
        for (uint32_t i = i0; i < i1; ++i) {
            const uint4 q = sq[i];
            // lengths bounded by the window, so the sums below cannot wrap
            if (q.x == 0u || q.y > kMaxWindow || q.z < 3u || q.z > kMaxWindow) bad = 1u;
            sll += q.y;
            spos += q.y + q.z;
        }
        uint32_t xll = sll, xpos = spos;
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t yl = __shfl_up_sync(kFull, xll, d), yp = __shfl_up_sync(kFull, xpos, d);
            if (lane >= d) {
                xll += yl;
                xpos += yp;
            }
        }
        if (lane == 31) {
            warp_ll[wid] = xll;
            warp_pos[wid] = xpos;
        }
        __syncthreads();
        uint32_t base_ll = 0, base_pos = 0;
        for (uint32_t k = 0; k < wid; ++k) {
            base_ll += warp_ll[k];
            base_pos += warp_pos[k];
        }
        if (tid == kLitThreads - 1) {
            tot_ll = base_ll + xll;
            tot_pos = base_pos + xpos;
        }
        uint32_t d = base_ll + xll - sll, p = base_pos + xpos - spos;
        __syncthreads();
        const uint32_t TP = tot_pos, TLL = tot_ll;
        if (TP > w || bad) {
            if (tid == 0) bad = 1u;
        } else {
            for (uint32_t i = i0; i < i1; ++i) {
                const uint4 q = sq[i];
                if (q.x > p + q.y) bad = 1u;  // match would reach before the window start
                for (uint32_t k = 0; k < q.y; ++k) lit[d + k] = __ldg(src + p + k);
                d += q.y;
                p += q.y + q.z;
            }
            for (uint32_t k = tid; k < w - TP; k += kLitThreads) lit[TLL + k] = __ldg(src + TP + k);
        }
        __syncthreads();
        if (bad) {
            if (tid == 0) {
                atomicOr(a.status, kErrBadSequences);
                write_frame_header(slot, w);
                a.sec_off[b] = 0;  // raw frame
            }
        } else {
            const uint32_t nlit = TLL + (w - TP);
            const uint32_t fh = frame_header_bytes(w);
            const uint32_t lh = nlit < 32u ? 1u : (nlit < 4096u ? 2u : 3u);
            const uint32_t H = fh + 3u + lh;
            for (uint32_t k = tid; k < nlit; k += kLitThreads) slot[H + k] = lit[k];
            if (tid == 0) {
                write_frame_header(slot, w);
                uint8_t *h = slot + fh + 3u;
                if (lh == 1u) {
                    h[0] = static_cast<uint8_t>(nlit << 3);  // Raw_Literals_Block, Size_Format 00
                } else if (lh == 2u) {
                    h[0] = static_cast<uint8_t>(((nlit << 4) & 0xF0u) | (1u << 2));
                    h[1] = static_cast<uint8_t>(nlit >> 4);
                } else {
                    h[0] = static_cast<uint8_t>(((nlit << 4) & 0xF0u) | (3u << 2));
                    h[1] = static_cast<uint8_t>(nlit >> 4);
                    h[2] = static_cast<uint8_t>(nlit >> 12);
                }
                a.sec_off[b] = ns ? H + nlit : 0u;  // no sequences: the raw block is smaller
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- sequences
// One warp per window, kSeqWarps windows per CTA (the FSE tables are shared).
// Sequences pass through shared memory in chunks of kChunk; the only serial
// work -- the repeat-offset history and the three FSE state chains -- runs
// on single lanes over shared memory, the rest is spread over the warp:
//   R. ascending chunks: lane 0 computes each Offset_Value from the decoder's
//      repeat history; the values go to a per-window global scratch.
//   E. descending chunks (the bitstream starts with the last sequence):
//      codes in parallel; lanes 0-2 run the LL / ML / OF chains; a warp scan
//      gives each sequence's bit position; every lane ORs its sequences'
//      fields into the warp's bit buffer; whole 32-bit words are stored, the
//      partial last word carries into the next chunk.
constexpr uint32_t kChunk = 256;
constexpr uint32_t kSeqWarps = 4;
constexpr uint32_t kPerLane = kChunk / 32;
constexpr uint32_t kBufWords = kChunk * 65u / 32u + 4u;  // <= 65 bits per sequence, plus the carried word

struct WarpSeq {
    uint4 q[kChunk];          // the chunk's records, in bitstream order (last sequence first)
    uint32_t ov[kChunk];      // Offset_Value
    uint8_t code[3][kChunk];  // LL, ML, OF codes
    uint16_t upd[3][kChunk];  // state-update bits: value | nbBits << 8 (LL, ML, OF)
    uint32_t pos[kChunk];     // bit position within the chunk
    uint32_t buf[kBufWords];
    uint32_t state[3];
};

struct SeqSmem {
    FseEnc T;
    CodeTables C;
    WarpSeq W[kSeqWarps];
};

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

    // ---- R: Offset_Values, ascending, with the decoder's repeat history (lane 0)
    uint32_t r1 = 1, r2 = 4, r3 = 8;
    for (uint32_t lo = 0; lo < ns; lo += kChunk) {
        const uint32_t len = min(kChunk, ns - lo);
        for (uint32_t k = lane; k < len; k += 32u) {
            const uint4 q = sq[lo + k];
            S.pos[k] = q.x;               // offset
            S.ov[k] = q.y == 0u ? 1u : 0u;  // literal length is zero
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
        for (uint32_t k = lane; k < len; k += 32u) ovg[lo + k] = S.ov[k];
        __syncwarp();
    }

    // ---- E: the bitstream, last sequence first
    uint8_t *hp = slot + sec;
    const uint32_t hl = ns < 128u ? 2u : 3u;  // Number_of_Sequences (1-2 bytes) + modes byte
    if (lane == 0) {
        if (ns < 128u) {
            hp[0] = static_cast<uint8_t>(ns);
        } else {
            hp[0] = static_cast<uint8_t>((ns >> 8) + 0x80u);
            hp[1] = static_cast<uint8_t>(ns);
        }
        hp[hl - 1] = 0;  // Predefined_Mode for all three
    }
    uint8_t *bs = hp + hl;
    // bitstream bytes at which the block stops paying (none when the literals alone fill the window)
    const int32_t room = static_cast<int32_t>(fh + 3u + w) - static_cast<int32_t>(sec + hl);
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
            const uint32_t lg = lane == 2u ? kOFLog : kLLLog;
            const uint32_t *enc = lane == 0u ? G.T.ll : (lane == 1u ? G.T.ml : G.T.of);
            const uint8_t *cd = S.code[lane];
            uint16_t *up = S.upd[lane];
            uint32_t j = 0;
            if (hi == ns) {  // last sequence: any state of its symbol, no bits
                D = enc[static_cast<uint32_t>(cd[0]) << lg] & 0xFFu;
                up[0] = 0;
                j = 1;
            }
            for (; j < len; ++j) {
                const uint32_t e = enc[(static_cast<uint32_t>(cd[j]) << lg) + D];
                up[j] = static_cast<uint16_t>((D - (e >> 16)) | (((e >> 8) & 0xFFu) << 8));
                D = e & 0xFFu;
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
                nb = (S.upd[0][j] >> 8) + (S.upd[1][j] >> 8) + (S.upd[2][j] >> 8) + G.C.ll_bits[S.code[0][j]] +
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
            const uint32_t no = uo >> 8, nm = um >> 8, nl = ul >> 8;
            const uint64_t ga = static_cast<uint64_t>(uo & 0xFFu) | (static_cast<uint64_t>(um & 0xFFu) << no) |
                                (static_cast<uint64_t>(ul & 0xFFu) << (no + nm));
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
        bw.add(S.state[1], kMLLog);
        bw.add(S.state[2], kOFLog);
        bw.add(S.state[0], kLLLog);
        bw.close();
        content = sec + hl + bw.pos - (fh + 3u);
    }
    content = __shfl_sync(kFull, content, 0);
    return content < w ? content : 0u;
}

__global__ void __launch_bounds__(32 * kSeqWarps) zenc_sequences_kernel(ZencArgs a) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    SeqSmem &G = *reinterpret_cast<SeqSmem *>(smem_raw);
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    G.C.build();
    build_fse(G.T, kLLNorm, kLLSyms, kLLLog, G.T.ll);
    build_fse(G.T, kMLNorm, kMLSyms, kMLLog, G.T.ml);
    build_fse(G.T, kOFNorm, kOFSyms, kOFLog, G.T.of);
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
            for (uint32_t k = tid; k < size; k += blockDim.x) dst[k] = slot[k];
        } else {
            const uint32_t w = win_size(a, b);
            const uint32_t hl = frame_header_bytes(w) + 3u;
            const uint8_t *src = a.src + static_cast<uint64_t>(b) * a.window;
            for (uint32_t k = tid; k < hl; k += blockDim.x) dst[k] = slot[k];
            for (uint32_t k = tid; k < w; k += blockDim.x) dst[hl + k] = __ldg(src + k);
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
    a.status = l.status;
    return a;
}

unsigned long long g_lit_smem_set = 0, g_seq_smem_set = 0;

}  // namespace

cudaError_t launch_zenc(const ZencLaunch &l, cudaStream_t st) {
    if (l.num_windows == 0) return cudaSuccess;
    const ZencArgs a = args_of(l);
    cudaError_t e = set_smem_once(zenc_literals_kernel, kMaxWindow, g_lit_smem_set);
    if (e != cudaSuccess) return e;
    int grid = l.num_sms * 3;
    if (static_cast<uint32_t>(grid) > l.num_windows) grid = static_cast<int>(l.num_windows);
    zenc_literals_kernel<<<grid, kLitThreads, kMaxWindow, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = set_smem_once(zenc_sequences_kernel, sizeof(SeqSmem), g_seq_smem_set)) != cudaSuccess) return e;
    grid = l.num_sms * 3;
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
