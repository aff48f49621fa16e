// Zstd L1/L2 frames: GPU match finding overlapped with a pool of CPU coder
// threads running libzstd's ZSTD_compressSequences, one frame per 64 KiB
// window.
//
// Per window this is exactly the reference's loop (compress_zstd_custom.rs:
// 115-199): one ZSTD_CCtx with parameter 1001 set to 0 (:128), a session reset
// before every window (:161), ZSTD_compressSequences over the window's
// sequences and bytes (:163-171), ZSTD_compress level 1 if that fails
// (:173-190).  The same sequences through the same libzstd give the same
// frame bytes, so the frames equal the reference's; only the schedule
// differs: the input is cut into slices, the GPU finds the sequences of slice
// k+1 while the coder threads encode slice k, and every thread owns a
// ZSTD_CCtx.  libzstd is loaded at run time by its soname, as the reference's
// zstd-sys link does not pin a version.
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "gcz.h"
#include "gcz_internal.h"

namespace {

constexpr size_t kW = GCZ_WINDOW;
constexpr int kResetSessionOnly = 1;  // ZSTD_reset_session_only
constexpr int kParam1001 = 1001;      // set to 0 by compress_zstd_custom.rs:128

struct ZstdApi {
    void *(*createCCtx)();
    size_t (*freeCCtx)(void *);
    size_t (*reset)(void *, int);
    size_t (*setParameter)(void *, int, int);
    size_t (*compressSequences)(void *, void *, size_t, const void *, size_t, const void *, size_t);
    size_t (*compress)(void *, size_t, const void *, size_t, int);
    unsigned (*isError)(size_t);
    const char *(*errorName)(size_t);
    bool ok = false;
    std::string why;
};

const ZstdApi &zstd_api() {
    static ZstdApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = nullptr;
        for (const char *name : {"libzstd.so.1", "libzstd.so"})
            if ((h = dlopen(name, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) {
            api.why = "libzstd not found (libzstd.so.1)";
            return;
        }
        bool all = true;
        auto sym = [&](auto &fn, const char *name) {
            void *p = dlsym(h, name);
            if (!p) all = false;
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(p);
        };
        sym(api.createCCtx, "ZSTD_createCCtx");
        sym(api.freeCCtx, "ZSTD_freeCCtx");
        sym(api.reset, "ZSTD_CCtx_reset");
        sym(api.setParameter, "ZSTD_CCtx_setParameter");
        sym(api.compressSequences, "ZSTD_compressSequences");
        sym(api.compress, "ZSTD_compress");
        sym(api.isError, "ZSTD_isError");
        sym(api.errorName, "ZSTD_getErrorName");
        api.ok = all;
        if (!all) api.why = "libzstd lacks ZSTD_compressSequences (needs >= 1.5)";
    });
    return api;
}

// ZSTD_COMPRESSBOUND (zstd.h): the largest frame ZSTD_compress can produce.
size_t frame_bound(size_t s) { return s + (s >> 8) + (s < (128u << 10) ? ((128u << 10) - s) >> 11 : 0); }

struct SliceBufs {
    // Sized to the slice's worst case (a third of its bytes) but left
    // uninitialised: only the pages the sequences land on are ever touched.
    gcz_zstd_sequence *seqs = nullptr;
    size_t cap = 0;
    std::vector<uint64_t> offsets;
    int rc = GCZ_OK;
    ~SliceBufs() { std::free(seqs); }
    bool reserve(size_t n) {
        if (seqs && cap >= n) return true;
        std::free(seqs);
        seqs = static_cast<gcz_zstd_sequence *>(std::malloc(std::max<size_t>(n, 1) * sizeof(gcz_zstd_sequence)));
        cap = seqs ? n : 0;
        return seqs != nullptr;
    }
};

// Everything a coder thread needs for one slice.
struct EncodeJob {
    const uint8_t *src;  // slice start
    size_t len;          // slice bytes
    size_t nb;           // windows in the slice
    const SliceBufs *in;
    uint8_t *stage;  // nb frames at stride frame_bound(kW)
    uint64_t *sizes;
    std::atomic<size_t> next{0};
    std::atomic<int> failed{0};
    std::mutex err_mu;
    std::string err;
};

void encode_windows(const ZstdApi &z, void *cctx, EncodeJob &job) {
    const size_t stride = frame_bound(kW);
    for (;;) {
        const size_t b = job.next.fetch_add(1, std::memory_order_relaxed);
        if (b >= job.nb || job.failed.load(std::memory_order_relaxed)) return;
        const uint8_t *win = job.src + b * kW;
        const size_t wlen = std::min(kW, job.len - b * kW);
        const uint64_t s0 = job.in->offsets[b], s1 = job.in->offsets[b + 1];
        uint8_t *dst = job.stage + b * stride;
        z.reset(cctx, kResetSessionOnly);
        size_t r = z.compressSequences(cctx, dst, stride, s1 > s0 ? job.in->seqs + s0 : nullptr, s1 - s0, win, wlen);
        if (z.isError(r)) {
            const size_t fb = z.compress(dst, stride, win, wlen, 1);
            if (z.isError(fb)) {
                std::lock_guard<std::mutex> lk(job.err_mu);
                job.err = std::string("ZSTD_compressSequences: ") + z.errorName(r);
                job.failed.store(1);
                return;
            }
            r = fb;
        }
        job.sizes[b] = r;
    }
}

}  // namespace

extern "C" size_t gcz_zstd_frames_bound(size_t n) {
    size_t total = 0;
    for (size_t off = 0; off < n; off += kW) total += frame_bound(std::min(kW, n - off));
    return total;
}

extern "C" int gcz_zstd_compress_frames(gcz_ctx *c, const uint8_t *src, size_t n, uint32_t level, uint32_t threads,
                                        uint8_t *out, size_t out_capacity, uint64_t *frame_sizes, size_t *out_size) {
    if (!c) return GCZ_EINVAL;
    if ((n && (!src || !out || !frame_sizes)) || !out_size)
        return gcz_internal_fail(c, GCZ_EINVAL, "null pointer");
    *out_size = 0;
    if (n == 0) return GCZ_OK;
    const ZstdApi &z = zstd_api();
    if (!z.ok) return gcz_internal_fail(c, GCZ_EUNAVAILABLE, z.why.c_str());
    const uint32_t depth = gcz_zstd_search_depth_for_level(level);
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());

    // 512-window (32 MiB) slices: small enough that filling and draining the
    // pipeline costs little, large enough for one GPU call to amortise its launches.
    constexpr size_t kSliceWindows = 512;
    // Allocation failures before any coder thread runs are reported, not
    // thrown through the C ABI.
    std::vector<void *> cctx;
    std::vector<uint8_t> stage;
    try {
        cctx.assign(threads, nullptr);
        stage.resize(kSliceWindows * frame_bound(kW));
    } catch (const std::bad_alloc &) {
        return gcz_internal_fail(c, GCZ_ENOMEM, "host buffer allocation failed");
    }
    auto free_all = [&] {
        for (void *p : cctx)
            if (p) z.freeCCtx(p);
    };
    for (void *&p : cctx) {
        if (!(p = z.createCCtx())) {
            free_all();
            return gcz_internal_fail(c, GCZ_ENOMEM, "ZSTD_createCCtx failed");
        }
        z.setParameter(p, kParam1001, 0);
    }

    const size_t nb_all = gcz_num_windows(n);
    const size_t slice_w = kSliceWindows;
    const size_t nslices = (nb_all + slice_w - 1) / slice_w;
    SliceBufs bufs[2];
    auto find = [&](size_t k, SliceBufs &sb) {
        const size_t off = k * slice_w * kW, len = std::min(n - off, slice_w * kW);
        const size_t cap = gcz_zstd_max_sequences(len);
        if (!sb.reserve(cap)) {
            sb.rc = gcz_internal_fail(c, GCZ_ENOMEM, "host sequence buffer allocation failed");
            return;
        }
        sb.offsets.assign(gcz_num_windows(len) + 1, 0);
        sb.rc = gcz_zstd_match_find(c, src + off, len, depth, sb.seqs, cap, sb.offsets.data());
    };

    int rc = GCZ_OK;
    size_t written = 0;
    find(0, bufs[0]);
    for (size_t k = 0; k < nslices && rc == GCZ_OK; ++k) {
        SliceBufs &cur = bufs[k & 1];
        if (cur.rc != GCZ_OK) {
            rc = cur.rc;  // the match finder's message is already the context's last error
            break;
        }
        const size_t off = k * slice_w * kW, len = std::min(n - off, slice_w * kW);
        EncodeJob job;
        job.src = src + off;
        job.len = len;
        job.nb = gcz_num_windows(len);
        job.in = &cur;
        job.stage = stage.data();
        job.sizes = frame_sizes + k * slice_w;
        std::vector<std::thread> pool;
        uint32_t started = 0;
        try {
            pool.reserve(threads);
            for (; started < threads; ++started)
                pool.emplace_back([&, t = started] { encode_windows(z, cctx[t], job); });
        } catch (const std::exception &) {
            // Fewer threads than asked (a thread limit): windows are claimed one
            // at a time by whoever is free, so the calling thread takes a share.
        }
        if (k + 1 < nslices) find(k + 1, bufs[(k + 1) & 1]);  // GPU works on the next slice meanwhile
        if (started < threads) encode_windows(z, cctx[started], job);
        for (std::thread &th : pool) th.join();
        if (job.failed.load()) {
            rc = gcz_internal_fail(c, GCZ_ECODEC, job.err.c_str());
            break;
        }
        const size_t stride = frame_bound(kW);
        for (size_t b = 0; b < job.nb; ++b) {
            const size_t s = job.sizes[b];
            if (written + s > out_capacity) {
                rc = gcz_internal_fail(c, GCZ_ECAPACITY, "frame output buffer too small");
                break;
            }
            std::memcpy(out + written, stage.data() + b * stride, s);
            written += s;
        }
    }
    free_all();
    if (rc == GCZ_OK) *out_size = written;
    return rc;
}
