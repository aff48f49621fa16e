/*
 * gcz.h -- C ABI of libgcz, the B200 (sm_100a) match finders behind
 * gpu-compressor's Zstd L1/L2 and LZMA2 L1+ levels.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (GCZ_OK == 0, negative on error; gcz_last_error() gives the message).  No
 * call aborts or traps.  Results are bit-identical to the reference kernels:
 *
 *   zstd_match_find    zstd_compress.cu:179-355   (Zstd L1 and L2)
 *   lzma2_match_find   lzma2_match_find.cu:54-194 (LZMA2 L1+)
 *
 * Windows: inputs are cut into independent 64 KiB windows
 * (CUSTOM_ZSTD_CHUNK_SIZE / LZMA2_CUSTOM_CHUNK_SIZE, constants.rs:5,10); no match
 * crosses a window.  The last window may be short.
 *
 * Host-buffer calls (`const uint8_t *src` is host memory) copy in, run and copy
 * out internally; when the host buffers are pinned the copies overlap the
 * kernels.  `_device` calls take device pointers and a cudaStream_t (passed as
 * void*) and only enqueue work.
 */
#ifndef GCZ_H
#define GCZ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GCZ_WINDOW 65536u              /* constants.rs:5 (Zstd), constants.rs:10 (LZMA2) */
#define GCZ_ZSTD_MAX_SEQ_PER_WINDOW 21845u /* chunk_size / 3, compress_zstd_custom.rs:55 */
#define GCZ_LZMA2_MAX_MATCHES 8u       /* LZMA2_MAX_MATCHES_PER_POS, constants.rs:12 */
#define GCZ_LZMA2_SEARCH_DEPTH 32u     /* LZMA2_HC4_SEARCH_DEPTH, constants.rs:13 */

enum {
    GCZ_OK = 0,
    GCZ_EINVAL = -1,     /* bad argument (null pointer, size, alignment) */
    GCZ_ECUDA = -2,      /* a CUDA runtime call failed */
    GCZ_ENOMEM = -3,     /* device or pinned-host allocation failed */
    GCZ_ECAPACITY = -4,  /* an output buffer is too small */
    GCZ_EDEVICE = -5,    /* a kernel reported an error status (bounded wait expired) */
    GCZ_ETOOLARGE = -6,  /* input larger than gcz_zstd_match_find_device_noalloc's static scratch */
    GCZ_EUNAVAILABLE = -7, /* a run-time library the call needs (libzstd) could not be loaded */
    GCZ_ECODEC = -8,     /* the CPU entropy coder failed */
    GCZ_ETIMEOUT = -9,   /* gcz_server_wait gave up; the request is still queued or running */
};

typedef struct gcz_ctx gcz_ctx;

/* ZSTD_Sequence (zstd.h), the record ZSTD_compressSequences consumes.  The
 * reference builds exactly these on the host from the kernel's {ll, ml-3, off}
 * triples: offset=off, litLength=ll, matchLength=ml+3, rep=0
 * (compress_zstd_custom.rs:8-14,137-153). */
typedef struct {
    uint32_t offset;
    uint32_t litLength;
    uint32_t matchLength;
    uint32_t rep;
} gcz_zstd_sequence;

/* ---------------------------------------------------------------- context */

/* Replaces the per-call cudaSetDevice + CudaDevice::new + load_ptx of both
 * adapters (compress_zstd_custom.rs:63-77, compress_lzma2_custom.rs:494-506):
 * the context is created once per device and reused; it owns the stream and
 * device/pinned staging buffers (grown on demand, freed by gcz_destroy). */
int gcz_create(int device_id, gcz_ctx **out);
void gcz_destroy(gcz_ctx *ctx);
const char *gcz_last_error(const gcz_ctx *ctx);
int gcz_device(const gcz_ctx *ctx);
const char *gcz_version(void);

/* Schedule-only knobs (they never change results): "algo" = 2 (default) runs
 * the candidate sweep then the per-window second stage, 1 the fused
 * single-warp kernels; "staged" (algo 1) = 1 stages each window into shared
 * memory with bulk copies, 0 reads it through L1; "parse_ctas" = Zstd
 * second-stage CTAs per SM (1-8); "parse_seg" = the Zstd second stage's
 * speculative segment: 1024 bytes per 8-lane group (default), 512 bytes per
 * 4-lane group, or 2048, 4096 or 8192 bytes per warp; "sweep_warps" = windows per candidate-sweep CTA
 * (4-7, default 7); "sweep_groups" = how the sweep groups the lanes of a step
 * that share a hash bucket: after a table read-back, only in blocks that have
 * such lanes, with __match_any_sync (0, default) or bit-sliced ballots (1), or
 * for every step one block ahead of the table work (2, 3 likewise);
 * "sweep_prefetch" = how many 128-byte blocks ahead of itself the read-back
 * sweep (groups 0, 1) prefetches its input into L2: 0, 4 (default) or 8;
 * "lzma_ctas" = LZMA2 second-stage CTAs per SM (1-8, default 3; values above
 * what fits on an SM -- 3, or 2 with 1024 threads -- run as that many);
 * "lzma_threads" = LZMA2 second-stage threads per CTA (256, 512 or 1024,
 * default 1024);
 * "slice_windows" = windows per slice of the host-buffer
 * pipelines (default 512 = 32 MiB; four slots, three slices in flight;
 * slices ramp up from a quarter of it and back down at the end);
 * "frames_slice_windows" =
 * the same for gcz_zstd_compress_frames_gpu (default 512 = 32 MiB; four
 * slots, three slices in flight). */
int gcz_set_option(gcz_ctx *ctx, const char *key, long value);
/* Read a knob or a counter: "algo" (1: fused single-warp kernels, 2: candidate
 * sweep + second stage, the default), "fallback_windows" (Zstd windows whose
 * speculative parse fell back to the exact warp-wide parse, since creation),
 * "binary_version" / "ptx_version" (the architecture of the loaded kernel
 * image as the CUDA runtime reports it, major*10+minor: 100 for sm_100a). */
int gcz_query(gcz_ctx *ctx, const char *key, long *value);

/* Synchronise `stream` (NULL = the context's stream) and report any error
 * status a kernel enqueued by a _device call recorded since the last check
 * (GCZ_ECAPACITY when a compact output overflowed its capacity). */
int gcz_sync(gcz_ctx *ctx, void *stream);

/* ---------------------------------------------------------------- Zstd L1/L2 */

/* level -> search_depth exactly as compress_zstd_custom.rs:57-61 (1->16, 2->64,
 * else 1).  Only search_depth > 1 matters to the kernel (lazy step on/off,
 * zstd_compress.cu:278), so levels 1 and 2 give identical sequences. */
uint32_t gcz_zstd_search_depth_for_level(uint32_t level);

size_t gcz_num_windows(size_t n);
/* Upper bound on the total sequence count for n input bytes. */
size_t gcz_zstd_max_sequences(size_t n);

/* GPU half of compress_chunk_zstd_custom (compress_zstd_custom.rs:47-153):
 * the sequences of every 64 KiB window of src[0..n), already converted to
 * ZSTD_Sequence.  Window b's sequences are seqs[offsets[b] .. offsets[b+1]);
 * offsets has num_windows+1 entries.  Feeding them with the window's bytes to
 * ZSTD_compressSequences gives the reference's frames byte for byte. */
int gcz_zstd_match_find(gcz_ctx *ctx, const uint8_t *src, size_t n, uint32_t search_depth,
                        gcz_zstd_sequence *seqs, size_t seq_capacity, uint64_t *offsets);

/* No counterpart in the reference.  gcz_zstd_match_find with 8-byte records
 * instead of 16-byte ZSTD_Sequence: record i = litLength | (matchLength - 3) << 16
 * | (uint64_t)offset << 32 (a 64 KiB window's lengths and offsets fit 16 bits).
 * Half the bytes cross PCIe back, next to the input going in; the caller
 * expands each record to ZSTD_Sequence{offset, litLength, matchLength, 0}
 * before ZSTD_compressSequences (a loop in INTEGRATION.md).  Offsets and
 * order as gcz_zstd_match_find. */
int gcz_zstd_match_find_packed(gcz_ctx *ctx, const uint8_t *src, size_t n, uint32_t search_depth, uint64_t *records,
                               size_t record_capacity, uint64_t *window_offsets);

/* Same on device memory.  d_src must be 16-byte aligned.  d_seqs needs
 * gcz_zstd_max_sequences(n) entries (or the actual count), d_offsets
 * num_windows+1 entries.  Enqueued on `stream` (cudaStream_t; NULL = the
 * context's stream). */
int gcz_zstd_match_find_device(gcz_ctx *ctx, const uint8_t *d_src, size_t n, uint32_t search_depth,
                               gcz_zstd_sequence *d_seqs, size_t seq_capacity, uint64_t *d_offsets,
                               void *stream);

/* No counterpart in the reference.  The Zstd step of
 * gcz_zstd_match_find_device without any device allocation, for callers that
 * cannot allocate device memory when they call in: a process whose device
 * memory is already carved up by another allocator (a serving engine's or a
 * framework's reserved pool, where one more cudaMalloc can fail or fragment
 * it), a latency-bound loop that cudaMalloc / cudaFree would stall (cudaFree
 * synchronises the whole device), or code that cannot hold a gcz_ctx, since
 * gcz_create itself allocates.  Its scratch is a file-scope device array of
 * about 21.3 MiB that every GPU loading this library keeps until exit; inputs
 * above GCZ_NOALLOC_MAX_INPUT (8 MiB, one ZSTD_CHUNK_SIZE pipeline chunk) are
 * rejected with GCZ_ETOOLARGE.  The caller passes device memory for input and
 * outputs, as for gcz_zstd_match_find_device; `stream` is a cudaStream_t (NULL
 * = the legacy default stream) and the call returns once the work on it is
 * done, with GCZ_ECAPACITY when d_seqs was too small.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) for that
 * device, so make that first call before any stream capture.  All calls on a
 * device share the one array: calls that overlap on the GPU race. */
#define GCZ_NOALLOC_MAX_INPUT (8u << 20)
int gcz_zstd_match_find_device_noalloc(int device, const uint8_t *d_src, size_t n, uint32_t search_depth,
                                       gcz_zstd_sequence *d_seqs, size_t seq_capacity, uint64_t *d_offsets,
                                       void *stream);

/* Kernel-level drop-in for zstd_match_find (zstd_compress.cu:179-190): same
 * arguments, same output layout -- {literal_length, match_length-3, offset}
 * u32 triples at stride max_sequences_per_chunk per window, literal bytes at
 * stride chunk_size (d_literals may be NULL), per-window counts (d_lit_counts
 * may be NULL).  chunk_size must be a multiple of 16 and <= 65536. */
int gcz_zstd_match_find_ref_layout_device(gcz_ctx *ctx, const uint8_t *d_input, uint32_t *d_sequences,
                                          uint8_t *d_literals, uint32_t *d_seq_counts,
                                          uint32_t *d_lit_counts, uint32_t chunk_size, uint32_t num_chunks,
                                          uint32_t total_input_size, uint32_t search_depth,
                                          uint32_t max_sequences_per_chunk, void *stream);

/* ---------------------------------------------------------------- LZMA2 L1+ */

/* Packed per-position result: 0 when the position has no match, else
 * (length << 16) | distance.  The reference records at most one match per
 * position (its chain loop stops after the first candidate,
 * lzma2_match_find.cu:157-160), so this holds everything it finds. */
#define GCZ_LZMA2_DIST(p) ((p) & 0xFFFFu)
#define GCZ_LZMA2_LEN(p) ((p) >> 16)

/* Compact form: packed[q] for every q < n (n entries), and has_matches[b]
 * (num_windows bytes, 0/1) = any(match_counts > 0) over window b -- the one bit
 * encode_single_sub_block consumes (compress_lzma2_custom.rs:577).  Either
 * output may be NULL; with packed == NULL only the has_matches bytes cross
 * back to the host (the triage call of the LZMA2 L1+ path). */
int gcz_lzma2_match_find(gcz_ctx *ctx, const uint8_t *src, size_t n, uint32_t search_depth,
                         uint32_t *packed, uint8_t *has_matches);
int gcz_lzma2_match_find_device(gcz_ctx *ctx, const uint8_t *d_src, size_t n, uint32_t search_depth,
                                uint32_t *d_packed, uint8_t *d_has_matches, void *stream);

/* gpu_find_matches (compress_lzma2_custom.rs:483-560): the GpuMatchData arrays,
 * de-interleaved and zero-filled exactly like the reference's alloc_zeros +
 * split loop: match_counts[b*W + q], match_distances / match_lengths at
 * [(b*W + q)*max_matches + k].  W = 65536.  Any output may be NULL. */
int gcz_lzma2_find_matches(gcz_ctx *ctx, const uint8_t *src, size_t n, uint32_t max_matches,
                           uint32_t *match_distances, uint32_t *match_lengths, uint32_t *match_counts);

/* Kernel-level drop-in for lzma2_match_find (lzma2_match_find.cu:54-63): same
 * arguments and layout -- LzmaMatch{distance,length} u32 pairs at
 * [(b*sub_block_size + q)*max_matches_per_pos + k] and match_counts[b*sub_block_size + q].
 * Slots past a position's count are not written (the reference host zero-fills
 * them).  sub_block_size must be a multiple of 16 and <= 65536. */
int gcz_lzma2_match_find_ref_layout_device(gcz_ctx *ctx, const uint8_t *d_input, uint32_t *d_matches,
                                           uint32_t *d_match_counts, uint32_t sub_block_size,
                                           uint32_t num_sub_blocks, uint32_t total_input_size,
                                           uint32_t max_matches_per_pos, uint32_t search_depth,
                                           void *stream);

/* ---------------------------------------------------------------- batches */

/* Many inputs of uneven size in one launch.  Each input is cut into 64 KiB
 * windows exactly as the reference cuts a file (its 8 MiB / 128 MiB pipeline
 * chunks are multiples of 64 KiB, pipeline.rs:110, pipeline_lzma2.rs:40), so a
 * batched window gives the same sequences or matches as the same window
 * processed alone.  Inputs sit in one device slab at 16-byte aligned offsets;
 * the window table says where each window is. */
typedef struct {
    uint64_t offset;  /* first byte of the window in the slab (16-byte aligned) */
    uint32_t size;    /* 1 .. 65536 */
    uint32_t file;    /* index of the input the window belongs to */
} gcz_window;

size_t gcz_batch_num_windows(const size_t *sizes, size_t count);
/* Slab layout of `count` inputs: file_offsets[count] (may be NULL),
 * windows[gcz_batch_num_windows] (may be NULL), total slab bytes. */
int gcz_batch_layout(const size_t *sizes, size_t count, uint64_t *file_offsets, gcz_window *windows,
                     uint64_t *slab_bytes);

/* Zstd over a window table (device memory): sequences of window w at
 * d_seqs[d_offsets[w] .. d_offsets[w+1]).  After a first call of the same
 * sizes it allocates nothing, so it can be enqueued repeatedly or captured. */
int gcz_zstd_match_find_batch_device(gcz_ctx *ctx, const uint8_t *d_slab, uint64_t slab_bytes,
                                     const gcz_window *d_windows, uint32_t num_windows, uint32_t search_depth,
                                     gcz_zstd_sequence *d_seqs, size_t seq_capacity, uint64_t *d_offsets,
                                     void *stream);
/* LZMA2 over a window table: packed results at the slab offsets of each
 * window's bytes (d_packed has slab_bytes entries), one has-match byte per window. */
int gcz_lzma2_match_find_batch_device(gcz_ctx *ctx, const uint8_t *d_slab, uint64_t slab_bytes,
                                      const gcz_window *d_windows, uint32_t num_windows, uint32_t search_depth,
                                      uint32_t *d_packed, uint8_t *d_has_matches, void *stream);
/* Host inputs: srcs[i] of sizes[i] bytes.  window_offsets has
 * gcz_batch_num_windows+1 entries (windows in input order). */
int gcz_zstd_match_find_files(gcz_ctx *ctx, const uint8_t *const *srcs, const size_t *sizes, size_t count,
                              uint32_t search_depth, gcz_zstd_sequence *seqs, size_t seq_capacity,
                              uint64_t *window_offsets);

/* ---------------------------------------------------------------- serving */

/* A request loop over one context (continuous batching).  Requests of any
 * kind and size are submitted at any time.  The loop keeps up to 8 slots, each
 * a stream with every device buffer a batch of max_batch_bytes needs, of any mix
 * of kinds, allocated once by gcz_server_create (~22 device bytes per input
 * byte per slot; the slot count is hbm_budget / (22 * max_batch_bytes), at
 * most 8, so the budget holds and serving never calls cudaMalloc or cudaFree).
 * Whenever a slot is free and requests are pending, one worker thread admits
 * the oldest pending requests -- Zstd sequences, Zstd frames and LZMA2
 * together, each counted in whole 64 KiB windows as it is laid out on the
 * device -- into a batch of at most max_batch_bytes and launches it at once:
 * one candidate sweep over all its windows, then each kind's second stage.
 * Batches on different slots run on the GPU at the same time; a batch's
 * results are copied out as soon as its kernels finish (a host callback wakes
 * the worker).  Every request gets exactly the result it would get alone
 * (windows are independent).  src and the output buffers must stay valid until
 * gcz_server_wait returns the request's own status (not GCZ_ETIMEOUT), or until
 * gcz_server_destroy returns.  max_batch_bytes = 0 splits the budget over four
 * slots.  Each batch has its own device status words, cleared at its launch, so
 * an error affects only the batch that hit it. */
typedef struct gcz_server gcz_server;
enum { GCZ_REQ_ZSTD = 0, GCZ_REQ_LZMA2 = 1, GCZ_REQ_ZSTD_FRAMES = 2 };

int gcz_server_create(gcz_ctx *ctx, uint64_t hbm_budget, uint64_t max_batch_bytes, uint32_t max_batch_requests,
                      gcz_server **out);
void gcz_server_destroy(gcz_server *server);  /* finishes every submitted request first */
uint64_t gcz_server_max_batch_bytes(const gcz_server *server);
/* Slots (batches that can be on the GPU at once) and device bytes the loop holds. */
int gcz_server_info(const gcz_server *server, uint32_t *slots, uint64_t *device_bytes);
/* GCZ_REQ_ZSTD: out_a = gcz_zstd_sequence[cap_a], out_b = uint64_t[num_windows+1] offsets.
 * GCZ_REQ_LZMA2: out_a = uint32_t[n] packed (or NULL), out_b = uint8_t[num_windows] has-match bytes
 * (or NULL).  GCZ_REQ_ZSTD_FRAMES: the GPU frames of gcz_zstd_compress_frames_gpu -- out_a =
 * uint8_t[cap_a] frames back to back (gcz_zstd_frames_bound(n) always suffices), out_b =
 * uint64_t[num_windows] frame sizes.  search_depth as for the direct calls.  GCZ_ETOOLARGE if
 * n > max batch bytes. */
int gcz_server_submit(gcz_server *server, int kind, uint32_t search_depth, const uint8_t *src, size_t n, void *out_a,
                      size_t cap_a, void *out_b, uint64_t *request_id);
/* Blocks until the request is done and returns its status; latency_ms =
 * submit-to-completion time.  Each request is collected by one wait: GCZ_EINVAL
 * for an unknown id or one already collected.  When timeout_s passes first the
 * call returns GCZ_ETIMEOUT and the request stays in the loop (queued or
 * running): its input and output buffers are still in use until a later wait
 * collects it or gcz_server_destroy returns. */
int gcz_server_wait(gcz_server *server, uint64_t request_id, double timeout_s, double *latency_ms);
/* Failure detection without a GPU fault: submits a request whose batch runs
 * one CTA that waits on an mbarrier nothing completes, with the same kind of
 * bounded wait the kernels use (max_iterations tries).  The wait runs out, the
 * kernel records it in that batch's status word and returns; waiting on the
 * id gives GCZ_EDEVICE, for every request of that batch, while batches before
 * and after it complete normally. */
int gcz_server_selftest_wait_timeout(gcz_server *server, uint32_t max_iterations, uint64_t *request_id);
/* Completed requests, their input bytes, batches launched, and the p50/p99 of
 * submit-to-completion latency (ms) over the most recent 2^20 completed requests. */
int gcz_server_stats(gcz_server *server, uint64_t *completed, uint64_t *bytes, uint64_t *batches, double *p50_ms,
                     double *p99_ms);

/* ---------------------------------------------------------------- frames */

/* Zstd L1/L2 frames of a host buffer: compress_chunk_zstd_custom
 * (compress_zstd_custom.rs:47-203) over the whole input, one Zstd frame per
 * 64 KiB window, written back to back into `out` in window order with
 * frame_sizes[b] (num_windows entries) -- the frames and size table an NVZS
 * container holds (pipeline.rs:163-168,217-225).  The GPU finds the sequences
 * of one 32 MiB slice while `threads` CPU threads (0 = all cores) run libzstd's
 * ZSTD_compressSequences on the previous slice, each window exactly as the
 * reference does it, so the frames equal the reference's byte for byte.
 * libzstd (>= 1.5) is loaded at run time; GCZ_EUNAVAILABLE without it.
 * out_capacity >= gcz_zstd_frames_bound(n) always suffices. */
size_t gcz_zstd_frames_bound(size_t n);
int gcz_zstd_compress_frames(gcz_ctx *ctx, const uint8_t *src, size_t n, uint32_t level, uint32_t threads,
                             uint8_t *out, size_t out_capacity, uint64_t *frame_sizes, size_t *out_size);

/* Zstd frames built on the GPU (no reference counterpart: the reference's
 * GPU block encoder, zstd_compress.cu:756-1038, is unused and its output is
 * not decodable).  Each 64 KiB window becomes one frame with a single block:
 * literals raw, RLE or Huffman-coded (whichever is smallest), sequences
 * FSE-coded (RFC 8878) with, per field and window, an RLE, a normalised
 * FSE-compressed or the predefined table (whichever an integer size estimate
 * finds smallest), repeat offsets used where they apply, or a raw block when
 * that is smaller.  Every frame decodes with stock libzstd to its window.
 * The frames differ from libzstd's bytes, but their total size is within
 * 0.1 percentage point of gcz_zstd_compress_frames' on the bench data.
 *
 * gcz_zstd_compress_frames_gpu: host bytes in, frames back to back in `out`
 * (out_capacity >= gcz_zstd_frames_bound(n) always suffices) with
 * frame_sizes[num_windows]; copy-in, match finding, encoding and copy-out of
 * 32 MiB slices overlap over four streams ("frames_slice_windows").
 * gcz_zstd_encode_frames_device: the entropy stage alone, on device memory,
 * from the output of gcz_zstd_match_find_device (records + per-window
 * offsets): frames back to back in d_out, byte offsets of the frames in
 * d_frame_offsets[num_windows + 1].  d_src must be 16-byte aligned.  Sequences that do not describe their
 * window give GCZ_EINVAL at the next synchronising call (gcz_sync). */
int gcz_zstd_compress_frames_gpu(gcz_ctx *ctx, const uint8_t *src, size_t n, uint32_t level, uint8_t *out,
                                 size_t out_capacity, uint64_t *frame_sizes, size_t *out_size);
int gcz_zstd_encode_frames_device(gcz_ctx *ctx, const uint8_t *d_src, size_t n, const gcz_zstd_sequence *d_seqs,
                                  const uint64_t *d_seq_offsets, uint8_t *d_out, size_t out_capacity,
                                  uint64_t *d_frame_offsets, void *stream);

/* GPU frames for a batch of files (window table as for
 * gcz_zstd_match_find_batch_device): the entropy stage over the records and
 * per-window offsets of gcz_zstd_match_find_batch_device, frames of all
 * windows back to back in window order (file by file), byte offsets in
 * d_frame_offsets[num_windows + 1].  gcz_zstd_compress_files_gpu is the
 * host form: k host files in, their frames back to back in `out` and one
 * size per window in frame_sizes (gcz_batch_num_windows entries); one
 * launch of each kernel covers every file.  out_capacity >= the sum of
 * gcz_zstd_frames_bound(sizes[i]) always suffices.  Each frame equals the
 * one gcz_zstd_compress_frames_gpu gives for that window. */
int gcz_zstd_encode_frames_batch_device(gcz_ctx *ctx, const uint8_t *d_slab, uint64_t slab_bytes,
                                        const gcz_window *d_windows, uint32_t num_windows,
                                        const gcz_zstd_sequence *d_seqs, const uint64_t *d_seq_offsets,
                                        uint8_t *d_out, size_t out_capacity, uint64_t *d_frame_offsets, void *stream);
int gcz_zstd_compress_files_gpu(gcz_ctx *ctx, const uint8_t *const *srcs, const size_t *sizes, size_t count,
                                uint32_t level, uint8_t *out, size_t out_capacity, uint64_t *frame_sizes,
                                size_t *out_size);

/* ---------------------------------------------------------------- self-test, timing */

/* Self-test of the error path (no counterpart in the reference): one CTA waits
 * on an mbarrier that nothing completes, with the same kind of bounded wait
 * the kernels use around their bulk copies; the wait runs out after
 * max_iterations tries and the kernel records it, so this returns GCZ_EDEVICE
 * and the context stays usable.  No fault, trap or hang is involved. */
int gcz_selftest_wait_timeout(gcz_ctx *ctx, uint32_t max_iterations);

/* Between gcz_profile_start and gcz_profile_stop every match-find step this
 * context launches is bracketed by CUDA events on its own launch stream.
 * gcz_profile_stop synchronises those events and returns the summed device
 * time of the match-find steps, their count, and the count of all kernels
 * the library launched in that interval (match finding, compaction and the
 * entropy stage). */
int gcz_profile_start(gcz_ctx *ctx);
int gcz_profile_stop(gcz_ctx *ctx, double *match_kernel_ms, uint64_t *match_kernel_launches,
                     uint64_t *all_kernel_launches);

#ifdef __cplusplus
}
#endif

#endif /* GCZ_H */
