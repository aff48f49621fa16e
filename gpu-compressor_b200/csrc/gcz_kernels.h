// Host-side launch interface of the libgcz kernels (internal to the library).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gcz {

// One window of a batched launch: bytes [offset, offset + size) of the input
// slab (offset 16-byte aligned, size <= 65536).  Windows of one file follow
// each other at 64 KiB steps; the last one may be short.
struct WinDesc {
    uint64_t offset;
    uint32_t size;
    uint32_t file;
};

struct ZstdLaunch {
    const uint8_t *src;     // 16-byte aligned
    uint64_t n;
    uint32_t window;        // multiple of 16, <= 65536
    uint32_t num_windows;
    uint32_t search_depth;
    uint32_t max_seqs;      // per-window output stride
    void *packed;           // uint2 per sequence at stride max_seqs (compact path), or null
    uint32_t *ref_seqs;     // {ll, ml-3, off} triples at stride max_seqs (reference layout), or null
    uint32_t *seq_counts;
    uint32_t *lit_counts;   // may be null
    uint32_t *status;
    int num_sms;
    int staged;             // 1: TMA-staged window in shared memory, 0: read through L1
};

struct LzmaLaunch {
    const uint8_t *src;
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
    int num_sms;
    int staged;
    const WinDesc *wins = nullptr;  // optional window table (second stage only)
    int ctas_per_sm = 3;            // second-stage CTAs per SM (schedule only)
    int threads = 1024;             // second-stage threads per CTA, 256, 512 or 1024 (schedule only)
};

// Second-stage Zstd parse after the candidate sweep.
struct Zstd2Launch {
    const uint8_t *src;
    const uint16_t *cand;   // from launch_cand_sweep
    uint64_t n;
    uint32_t window;
    uint32_t num_windows;
    uint32_t search_depth;
    uint32_t max_seqs;
    void *seg;              // zstd2_seg_scratch_entries(num_windows) uint2 entries
    void *packed;           // uint2 per sequence at stride max_seqs, or null
    uint32_t *ref_seqs;     // reference triples at stride max_seqs, or null
    uint32_t *seq_counts;
    uint32_t *lit_counts;   // may be null
    uint32_t *status;       // [0] error bits, [1] windows that took the exact fallback
    int num_sms;
    int ctas_per_sm;
    const WinDesc *wins;    // optional window table (null: windows at window * w)
    uint32_t seg_width = 4096;  // speculative segment bytes per warp: 2048, 4096 or 8192 (schedule only)
};

cudaError_t launch_zstd_match(const ZstdLaunch &l, cudaStream_t st);
// sweep_warps: windows swept per CTA (4-7, one 32 KiB table each); sweep_groups:
// lanes with equal hashes in a step grouped by __match_any_sync (0, 2) or by
// bit-sliced ballots (1, 3), after a table read-back in the blocks that have
// such lanes (0, 1) or for every step one block ahead (2, 3).  sweep_prefetch:
// in modes 0 and 1, how many 128-byte blocks ahead of the sweep the input is
// prefetched into L2 (0: none).  Schedule only.
cudaError_t launch_cand_sweep(const uint8_t *src, uint64_t n, uint32_t window, uint32_t num_windows, uint16_t *cand,
                              int num_sms, cudaStream_t st, const WinDesc *wins = nullptr, int sweep_warps = 7,
                              int sweep_groups = 0, int sweep_prefetch = 0);
size_t zstd2_seg_scratch_entries(uint32_t num_windows);
cudaError_t launch_zstd_parse(const Zstd2Launch &l, cudaStream_t st);
cudaError_t launch_scan_counts(const uint32_t *counts, uint32_t num, uint64_t *offsets, cudaStream_t st);
cudaError_t launch_expand_seqs(const void *packed, const uint32_t *counts, const uint64_t *offsets, uint32_t num,
                               uint32_t max_seqs, void *out, uint64_t capacity, uint32_t *status, int num_sms,
                               cudaStream_t st);
// 8-byte records {ll | (ml-3) << 16, off} instead of ZSTD_Sequence.
cudaError_t launch_compact_seqs(const void *packed, const uint32_t *counts, const uint64_t *offsets, uint32_t num,
                                uint32_t max_seqs, void *out, uint64_t capacity, uint32_t *status, int num_sms,
                                cudaStream_t st);
cudaError_t launch_zstd_literals(const uint8_t *src, uint64_t n, uint32_t window, uint32_t num_windows,
                                 const uint32_t *ref_seqs, const uint32_t *seq_counts, uint32_t max_seqs, uint8_t *lits,
                                 int num_sms, cudaStream_t st);

// Zstd entropy stage (gcz_zenc.cu): frames from ZSTD_Sequence records.
constexpr uint32_t kZencSlot = 65536 + 1024;  // per-window frame slot bytes
constexpr uint32_t kZencMaxSeqs = 21845;      // sequences per window (chunk_size / 3)
constexpr uint32_t kZencPlanBytes = 1024;     // per-window Huffman plan record
struct ZencLaunch {
    const uint8_t *src;           // windows at b * window
    uint64_t n;
    uint32_t window;
    uint32_t num_windows;
    const void *seqs;             // ZSTD_Sequence records (16 B)
    const uint64_t *seq_offsets;  // num_windows + 1
    uint8_t *slots;               // num_windows * kZencSlot
    uint32_t *ovs;                // num_windows * kZencMaxSeqs
    uint32_t *sec_off;            // num_windows
    uint32_t *fsize;              // num_windows
    uint8_t *raw;                 // num_windows
    uint32_t *hist;               // num_windows * 256
    uint8_t *plan;                // num_windows * kZencPlanBytes
    uint32_t *status;
    int num_sms;
    const WinDesc *wins = nullptr;  // optional window table (16-byte-aligned offsets)
};
cudaError_t launch_zenc(const ZencLaunch &l, cudaStream_t st);
cudaError_t launch_zenc_compact(const ZencLaunch &l, const uint64_t *frame_offsets, uint8_t *out, uint64_t capacity,
                                cudaStream_t st);

cudaError_t launch_lzma_match(const LzmaLaunch &l, cudaStream_t st);
cudaError_t launch_lzma_verify(const LzmaLaunch &l, const uint16_t *cand, cudaStream_t st);
cudaError_t launch_lzma_unpack(const uint32_t *packed, uint64_t n, uint32_t window, uint32_t num_windows,
                               uint32_t max_matches, uint32_t *dists, uint32_t *lens, uint32_t *counts, int num_sms,
                               cudaStream_t st);

}  // namespace gcz
