/*
 * gcz_compress -- compress a file into an NVZS container with libgcz, using
 * only the C ABI (include/gcz.h).  This is what a host program does in place
 * of gpu-compressor's Zstd L1/L2 path (compress_zstd_custom.rs:47-203 and the
 * NVZS writer, pipeline.rs:196-203,245-253): one Zstd frame per 64 KiB
 * window, a size table, the frames.
 *
 *   gcz_compress [-l LEVEL] [-g] INPUT OUTPUT
 *     -l 1|2  match-finder level (default 1)
 *     -g      entropy stage on the GPU (default: libzstd on all host cores)
 *
 * Build: gcc -O2 -I include gcz_compress.c -L gpu-compressor_b200/gcz -lgcz -Wl,-rpath,<dir of libgcz.so>
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gcz.h"

static int die(const char *what, gcz_ctx *ctx) {
    fprintf(stderr, "gcz_compress: %s%s%s\n", what, ctx ? ": " : "", ctx ? gcz_last_error(ctx) : "");
    return 1;
}

static void put_u64(FILE *f, uint64_t v) {
    unsigned char b[8];
    for (int i = 0; i < 8; i++) b[i] = (unsigned char)(v >> (8 * i));
    fwrite(b, 1, 8, f);
}

int main(int argc, char **argv) {
    uint32_t level = 1;
    int gpu_coder = 0, a = 1;
    for (; a < argc && argv[a][0] == '-'; a++) {
        if (!strcmp(argv[a], "-g")) gpu_coder = 1;
        else if (!strcmp(argv[a], "-l") && a + 1 < argc) level = (uint32_t)atoi(argv[++a]);
        else return die("usage: gcz_compress [-l LEVEL] [-g] INPUT OUTPUT", NULL);
    }
    if (argc - a != 2) return die("usage: gcz_compress [-l LEVEL] [-g] INPUT OUTPUT", NULL);

    FILE *in = fopen(argv[a], "rb");
    if (!in) return die("cannot open input", NULL);
    fseek(in, 0, SEEK_END);
    const long len = ftell(in);
    fseek(in, 0, SEEK_SET);
    const size_t n = len > 0 ? (size_t)len : 0;
    uint8_t *src = malloc(n ? n : 1);
    if (!src || fread(src, 1, n, in) != n) return die("cannot read input", NULL);
    fclose(in);

    gcz_ctx *ctx = NULL;
    if (gcz_create(0, &ctx) != GCZ_OK) return die("gcz_create failed", NULL);
    const size_t nb = gcz_num_windows(n);
    const size_t cap = gcz_zstd_frames_bound(n);
    uint8_t *frames = malloc(cap ? cap : 1);
    uint64_t *sizes = calloc(nb ? nb : 1, sizeof(uint64_t));
    size_t used = 0;
    if (!frames || !sizes) return die("out of host memory", NULL);
    const int rc = gpu_coder ? gcz_zstd_compress_frames_gpu(ctx, src, n, level, frames, cap, sizes, &used)
                             : gcz_zstd_compress_frames(ctx, src, n, level, 0, frames, cap, sizes, &used);
    if (rc != GCZ_OK) return die("compression failed", ctx);

    FILE *out = fopen(argv[a + 1], "wb");
    if (!out) return die("cannot open output", ctx);
    fwrite("NVZS", 1, 4, out);
    put_u64(out, n);
    put_u64(out, GCZ_WINDOW);
    put_u64(out, nb);
    for (size_t i = 0; i < nb; i++) put_u64(out, sizes[i]);
    fwrite(frames, 1, used, out);
    fclose(out);
    printf("%zu -> %zu bytes (%zu frames, %s coder)\n", n, used + 28 + 8 * nb, nb, gpu_coder ? "GPU" : "libzstd");
    gcz_destroy(ctx);
    free(frames);
    free(sizes);
    free(src);
    return 0;
}
