/*
 * ref_runner.c -- loads the reference's own kernels (PTX compiled from its
 * unmodified zstd_compress.cu / lzma2_match_find.cu with its own nvcc flags,
 * build.rs:59-95) through the CUDA driver JIT and launches them exactly as its
 * adapters do: grid = number of 64 KiB windows, block = 256, no dynamic shared
 * memory (compress_zstd_custom.rs:91-111, compress_lzma2_custom.rs:518-536).
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the reference baseline); never part
 * of the product.  Device pointers come from the caller (the primary context
 * of the current device is used).
 */
#include <cuda.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static CUmodule g_mod_zstd, g_mod_lzma;
static CUfunction g_zstd, g_lzma;
static char g_err[512];

const char *ref_last_error(void) { return g_err; }

static int check(CUresult r, const char *what) {
    if (r == CUDA_SUCCESS) return 0;
    const char *s = NULL;
    cuGetErrorString(r, &s);
    snprintf(g_err, sizeof(g_err), "%s: %s", what, s ? s : "?");
    return -1;
}

static char *slurp(const char *path) {
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *b = (char *)malloc((size_t)n + 1);
    if (b && fread(b, 1, (size_t)n, f) != (size_t)n) {
        free(b);
        b = NULL;
    }
    if (b) b[n] = 0;
    fclose(f);
    return b;
}

/* Load both PTX modules (JIT to the current GPU).  device: CUDA ordinal. */
int ref_load(const char *zstd_ptx, const char *lzma_ptx, int device) {
    if (check(cuInit(0), "cuInit")) return -1;
    CUcontext ctx = NULL;
    cuCtxGetCurrent(&ctx);
    if (!ctx) {
        CUdevice dev;
        if (check(cuDeviceGet(&dev, device), "cuDeviceGet")) return -1;
        if (check(cuDevicePrimaryCtxRetain(&ctx, dev), "cuDevicePrimaryCtxRetain")) return -1;
        if (check(cuCtxSetCurrent(ctx), "cuCtxSetCurrent")) return -1;
    }
    char *a = slurp(zstd_ptx), *b = slurp(lzma_ptx);
    if (!a || !b) {
        snprintf(g_err, sizeof(g_err), "cannot read %s / %s", zstd_ptx, lzma_ptx);
        free(a);
        free(b);
        return -1;
    }
    int rc = 0;
    if (check(cuModuleLoadData(&g_mod_zstd, a), "cuModuleLoadData(zstd)") ||
        check(cuModuleGetFunction(&g_zstd, g_mod_zstd, "zstd_match_find"), "get zstd_match_find") ||
        check(cuModuleLoadData(&g_mod_lzma, b), "cuModuleLoadData(lzma)") ||
        check(cuModuleGetFunction(&g_lzma, g_mod_lzma, "lzma2_match_find"), "get lzma2_match_find"))
        rc = -1;
    free(a);
    free(b);
    return rc;
}

/* zstd_match_find(input, sequences, literals, seq_counts, lit_counts,
 *                 chunk_size, num_chunks, total_input_size, search_depth,
 *                 max_sequences_per_chunk)   zstd_compress.cu:179-190 */
int ref_zstd_launch(uint64_t input, uint64_t sequences, uint64_t literals, uint64_t seq_counts,
                    uint64_t lit_counts, uint32_t chunk_size, uint32_t num_chunks, uint32_t total_input_size,
                    uint32_t search_depth, uint32_t max_seqs, uint64_t stream) {
    CUdeviceptr p0 = input, p1 = sequences, p2 = literals, p3 = seq_counts, p4 = lit_counts;
    void *args[] = {&p0, &p1, &p2, &p3, &p4, &chunk_size, &num_chunks, &total_input_size, &search_depth, &max_seqs};
    return check(cuLaunchKernel(g_zstd, num_chunks, 1, 1, 256, 1, 1, 0, (CUstream)stream, args, NULL),
                 "launch zstd_match_find");
}

/* lzma2_match_find(input, matches, match_counts, sub_block_size, num_sub_blocks,
 *                  total_input_size, max_matches_per_pos, search_depth)
 *                  lzma2_match_find.cu:54-63 */
int ref_lzma_launch(uint64_t input, uint64_t matches, uint64_t counts, uint32_t sub_block_size,
                    uint32_t num_sub_blocks, uint32_t total_input_size, uint32_t max_matches, uint32_t search_depth,
                    uint64_t stream) {
    CUdeviceptr p0 = input, p1 = matches, p2 = counts;
    void *args[] = {&p0, &p1, &p2, &sub_block_size, &num_sub_blocks, &total_input_size, &max_matches, &search_depth};
    return check(cuLaunchKernel(g_lzma, num_sub_blocks, 1, 1, 256, 1, 1, 0, (CUstream)stream, args, NULL),
                 "launch lzma2_match_find");
}
