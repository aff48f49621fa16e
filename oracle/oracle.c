/*
 * oracle.c -- CPU restatement of gpu-compressor's two match-finding kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the B200 kernels
 * are compared against; it is never linked into the product library and the
 * product path never calls it.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it.
 *
 * Both reference kernels are single-thread sequential code per 64 KiB window
 * (only threadIdx.x == 0 works after the table init), so this restatement is a
 * direct, statement-by-statement transcription of their behaviour:
 *
 *   zstd_match_find   zstd_compress.cu:179-355
 *   lzma2_match_find  lzma2_match_find.cu:54-194
 *
 * Windows are independent, so the buffer-level entry points split the window
 * range over `threads` POSIX threads (results do not depend on `threads`).
 *
 * Parity is pinned against the reference kernels themselves: the fixtures in
 * tests/golden/ were produced by running the reference's own PTX (compiled from
 * its unmodified .cu sources) on a B200, and tests/test_oracle.py checks this
 * file against them.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define OR_HASH_LOG 14
#define OR_HASH_SIZE (1u << OR_HASH_LOG)

/* zstd_compress.cu:32-35 / lzma2_match_find.cu:32-35: little-endian u32 */
static inline uint32_t or_load_u32(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

/* zstd_compress.cu:228 / lzma2_match_find.cu:92: multiplicative 14-bit hash */
static inline uint32_t or_hash4(const uint8_t *p) {
    return (or_load_u32(p) * 2654435761u) >> (32 - OR_HASH_LOG);
}

/* ------------------------------------------------------------------------ */
/* Zstd match finder, one window.  zstd_compress.cu:192-354                  */
/* seqs: 3 u32 per sequence {literal_length, match_length-3, offset}         */
/* (struct Sequence, zstd_compress.cu:38-42).  lits may be NULL.             */
/* ------------------------------------------------------------------------ */
#define OR_ZSTD_MIN_MATCH 3u        /* zstd_compress.cu:28 */
#define OR_ZSTD_MAX_MATCH 131074u   /* zstd_compress.cu:29 */

void oracle_zstd_window(const uint8_t *src, uint32_t size, uint32_t search_depth,
                        uint32_t max_seqs, uint32_t *seqs, uint8_t *lits,
                        uint32_t *out_nseq, uint32_t *out_nlit)
{
    uint16_t table[OR_HASH_SIZE];
    memset(table, 0, sizeof(table));              /* :195-200, empty == position 0 */

    uint32_t pos = 0, num_seqs = 0, num_lits = 0, literal_start = 0;
    uint32_t rep[3] = {1, 4, 8};                   /* :225 */

    while (pos + 3 < size) {                       /* :230 */
        uint32_t h = or_hash4(src + pos);
        uint32_t match_pos = table[h];
        table[h] = (uint16_t)(pos & 0xFFFF);       /* :235 */

        uint32_t match_offset = pos - match_pos;
        uint32_t match_len = 0;
        if (match_offset > 0 && match_offset <= pos && match_pos < size) {   /* :241 */
            if (src[match_pos] == src[pos] && src[match_pos + 1] == src[pos + 1] &&
                src[match_pos + 2] == src[pos + 2]) {
                match_len = 3;
                while (pos + match_len < size && match_pos + match_len < size &&
                       src[match_pos + match_len] == src[pos + match_len] &&
                       match_len < OR_ZSTD_MAX_MATCH)
                    match_len++;
            }
        }

        /* repeat offsets, first hit wins (:259-275) */
        for (int r = 0; r < 3 && match_len < OR_ZSTD_MIN_MATCH; r++) {
            if (rep[r] <= pos) {
                uint32_t rp = pos - rep[r];
                if (src[rp] == src[pos] && src[rp + 1] == src[pos + 1] && src[rp + 2] == src[pos + 2]) {
                    uint32_t rlen = 3;
                    while (pos + rlen < size && rp + rlen < size && src[rp + rlen] == src[pos + rlen] &&
                           rlen < OR_ZSTD_MAX_MATCH)
                        rlen++;
                    if (rlen >= OR_ZSTD_MIN_MATCH) {
                        match_len = rlen;
                        match_offset = rep[r];
                        break;
                    }
                }
            }
        }

        /* one lazy step at pos+1 (:278-307) */
        if (match_len >= OR_ZSTD_MIN_MATCH && search_depth > 1 && pos + 4 < size) {
            uint32_t h2 = or_hash4(src + pos + 1);
            uint32_t mp2 = table[h2];
            uint32_t off2 = (pos + 1) - mp2;
            if (off2 > 0 && off2 <= (pos + 1) && mp2 < size) {
                if (src[mp2] == src[pos + 1] && src[mp2 + 1] == src[pos + 2] && src[mp2 + 2] == src[pos + 3]) {
                    uint32_t len2 = 3;
                    while (pos + 1 + len2 < size && mp2 + len2 < size &&
                           src[mp2 + len2] == src[pos + 1 + len2] && len2 < OR_ZSTD_MAX_MATCH)
                        len2++;
                    if (len2 > match_len + 1) {
                        pos++;
                        match_len = len2;
                        match_offset = off2;
                        table[h2] = (uint16_t)(pos & 0xFFFF);
                    }
                }
            }
        }

        if (match_len >= OR_ZSTD_MIN_MATCH && num_seqs < max_seqs) {   /* :309 */
            uint32_t lit_len = pos - literal_start;
            if (lits)
                for (uint32_t i = literal_start; i < pos; i++) lits[num_lits++] = src[i];
            else
                num_lits += pos - literal_start;
            seqs[3 * num_seqs + 0] = lit_len;
            seqs[3 * num_seqs + 1] = match_len - OR_ZSTD_MIN_MATCH;
            seqs[3 * num_seqs + 2] = match_offset;
            num_seqs++;
            rep[2] = rep[1];
            rep[1] = rep[0];
            rep[0] = match_offset;                                   /* :323-325 */
            for (uint32_t i = 1; i < match_len && pos + i + 3 < size; i++)   /* :328-331 */
                table[or_hash4(src + pos + i)] = (uint16_t)((pos + i) & 0xFFFF);
            pos += match_len;
            literal_start = pos;
        } else {
            pos++;
        }
    }
    /* trailing literals (:341-343) */
    if (lits)
        for (uint32_t i = literal_start; i < size; i++) lits[num_lits++] = src[i];
    else if (size > literal_start)
        num_lits += size - literal_start;
    *out_nseq = num_seqs;
    *out_nlit = num_lits;
}

/* ------------------------------------------------------------------------ */
/* LZMA2 match finder, one window.  lzma2_match_find.cu:66-191.             */
/* Writes, for every position < size, count[pos] and the count slots of     */
/* match[pos*max_matches + k] = {distance, length}.  Positions in           */
/* [size, window) get count 0 (:188-190).  Unwritten slots are untouched.   */
/* ------------------------------------------------------------------------ */
#define OR_LZMA_MIN_MATCH 2u     /* lzma2_match_find.cu:20 */
#define OR_LZMA_MAX_MATCH 273u   /* lzma2_match_find.cu:21 */

void oracle_lzma2_window(const uint8_t *src, uint32_t size, uint32_t window,
                         uint32_t max_matches, uint32_t search_depth,
                         uint32_t *match /* [window*max_matches*2] or NULL */,
                         uint32_t *counts /* [window] or NULL */,
                         uint32_t *packed /* [size]: len<<16 | dist, or NULL */)
{
    uint16_t table[OR_HASH_SIZE];
    for (uint32_t i = 0; i < OR_HASH_SIZE; i++) table[i] = 0xFFFF;   /* :72-74 */

    for (uint32_t pos = 0; pos < size; pos++) {                     /* :96 */
        uint32_t n_matches = 0;
        uint32_t d_out = 0, l_out = 0;
        if (pos + 1 < size) {
            uint32_t best_len = 1;
            if (pos + 3 < size) {
                uint32_t h4 = or_hash4(src + pos);
                uint32_t cur = table[h4];
                table[h4] = (uint16_t)(pos & 0xFFFF);                   /* :108 */
                uint32_t chain_count = 0;
                while (cur != 0xFFFF && chain_count < search_depth && n_matches < max_matches) {
                    uint32_t match_pos = cur;
                    if (match_pos >= pos) break;
                    uint32_t distance = pos - match_pos;
                    if (distance > 0 && match_pos + 1 < size) {
                        uint32_t len = 0;
                        uint32_t max_len = size - pos;
                        if (max_len > OR_LZMA_MAX_MATCH) max_len = OR_LZMA_MAX_MATCH;
                        uint32_t max_match_check = size - match_pos;
                        if (max_match_check < max_len) max_len = max_match_check;
                        if (pos + 3 < size && match_pos + 3 < size &&
                            or_load_u32(src + match_pos) == or_load_u32(src + pos)) {
                            len = 4;
                            while (len < max_len && src[match_pos + len] == src[pos + len]) len++;
                        } else if (src[match_pos] == src[pos] && src[match_pos + 1] == src[pos + 1]) {
                            len = 2;
                            while (len < max_len && src[match_pos + len] == src[pos + len]) len++;
                        }
                        if (len >= OR_LZMA_MIN_MATCH && len > best_len) {
                            d_out = distance;
                            l_out = len;
                            if (match) {
                                uint32_t *slot = match + ((size_t)pos * max_matches + n_matches) * 2;
                                slot[0] = distance;
                                slot[1] = len;
                            }
                            n_matches++;
                            best_len = len;
                            if (len >= OR_LZMA_MAX_MATCH) break;
                        }
                    }
                    break;   /* single-level table (:157-160) */
                }
            }
            /* distance-1 run check (:164-181) */
            if (n_matches == 0 && pos + 1 < size) {
                if (pos > 0 && src[pos] == src[pos - 1] && src[pos + 1] == src[pos]) {
                    uint32_t len = 2;
                    uint32_t max_len = size - pos;
                    if (max_len > OR_LZMA_MAX_MATCH) max_len = OR_LZMA_MAX_MATCH;
                    while (len < max_len && src[pos + len] == src[pos]) len++;
                    if (len >= OR_LZMA_MIN_MATCH) {
                        d_out = 1;
                        l_out = len;
                        if (match) {
                            uint32_t *slot = match + ((size_t)pos * max_matches + n_matches) * 2;
                            slot[0] = 1;
                            slot[1] = len;
                        }
                        n_matches++;
                    }
                }
            }
        }
        if (counts) counts[pos] = n_matches;
        if (packed) packed[pos] = n_matches ? ((l_out << 16) | d_out) : 0u;
    }
    if (counts)
        for (uint32_t pos = size; pos < window; pos++) counts[pos] = 0;   /* :188-190 */
}

/* ------------------------------------------------------------------------ */
/* Buffer-level entry points (windows of `window` bytes, split over threads) */
/* ------------------------------------------------------------------------ */
typedef struct {
    int kind;   /* 0 zstd, 1 lzma */
    const uint8_t *in;
    uint64_t n;
    uint32_t window, depth, max_per;  /* max_per: max_seqs (zstd) / max_matches (lzma) */
    uint64_t b0, b1;                  /* window range */
    /* zstd outputs */
    uint32_t *seqs; uint8_t *lits; uint32_t *seq_counts; uint32_t *lit_counts;
    /* lzma outputs */
    uint32_t *match; uint32_t *counts; uint32_t *packed;
} or_job;

static void *or_worker(void *arg)
{
    or_job *j = (or_job *)arg;
    for (uint64_t b = j->b0; b < j->b1; b++) {
        uint64_t start = b * j->window;
        uint32_t size = (uint32_t)((j->n - start) < j->window ? (j->n - start) : j->window);
        if (j->kind == 0) {
            uint32_t ns, nl;
            oracle_zstd_window(j->in + start, size, j->depth, j->max_per,
                               j->seqs + b * (uint64_t)j->max_per * 3,
                               j->lits ? j->lits + start : NULL, &ns, &nl);
            j->seq_counts[b] = ns;
            if (j->lit_counts) j->lit_counts[b] = nl;
        } else {
            oracle_lzma2_window(j->in + start, size, j->window, j->max_per, j->depth,
                                j->match ? j->match + start * (uint64_t)j->max_per * 2 : NULL,
                                j->counts ? j->counts + start : NULL,
                                j->packed ? j->packed + start : NULL);
        }
    }
    return NULL;
}

static void or_run(or_job proto, int threads)
{
    uint64_t nb = proto.n ? (proto.n + proto.window - 1) / proto.window : 0;
    if (threads < 1) threads = 1;
    if ((uint64_t)threads > nb) threads = nb ? (int)nb : 1;
    pthread_t tid[256];
    or_job jobs[256];
    if (threads > 256) threads = 256;
    for (int t = 0; t < threads; t++) {
        jobs[t] = proto;
        jobs[t].b0 = nb * t / threads;
        jobs[t].b1 = nb * (t + 1) / threads;
    }
    if (threads == 1) { or_worker(&jobs[0]); return; }
    for (int t = 0; t < threads; t++) pthread_create(&tid[t], NULL, or_worker, &jobs[t]);
    for (int t = 0; t < threads; t++) pthread_join(tid[t], NULL);
}

/* Reference layout of zstd_match_find's outputs (sequences at stride max_seqs*3 u32 per window,
 * literals at stride `window` bytes per window, one count each per window). */
void oracle_zstd_match_find(const uint8_t *in, uint64_t n, uint32_t window, uint32_t search_depth,
                            uint32_t max_seqs, uint32_t *seqs, uint8_t *lits,
                            uint32_t *seq_counts, uint32_t *lit_counts, int threads)
{
    or_job j;
    memset(&j, 0, sizeof(j));
    j.kind = 0; j.in = in; j.n = n; j.window = window; j.depth = search_depth; j.max_per = max_seqs;
    j.seqs = seqs; j.lits = lits; j.seq_counts = seq_counts; j.lit_counts = lit_counts;
    or_run(j, threads);
}

/* Reference layout of lzma2_match_find's outputs: match[(b*window + pos)*max_matches + k] =
 * {distance, length} (u32 pairs), counts[b*window + pos].  Either may be NULL; `packed`
 * (n entries, len<<16|dist, 0 when count is 0) may be NULL. */
void oracle_lzma2_match_find(const uint8_t *in, uint64_t n, uint32_t window, uint32_t max_matches,
                             uint32_t search_depth, uint32_t *match, uint32_t *counts,
                             uint32_t *packed, int threads)
{
    or_job j;
    memset(&j, 0, sizeof(j));
    j.kind = 1; j.in = in; j.n = n; j.window = window; j.depth = search_depth; j.max_per = max_matches;
    j.match = match; j.counts = counts; j.packed = packed;
    or_run(j, threads);
}
