// libgcz C ABI (include/gcz.h): context, buffers, host and device entry points.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "gcz.h"
#include "gcz_internal.h"
#include "gcz_common.cuh"
#include "gcz_kernels.h"

namespace {

constexpr uint32_t kW = GCZ_WINDOW;
constexpr uint32_t kMaxSeqs = GCZ_ZSTD_MAX_SEQ_PER_WINDOW;  // chunk_size / 3

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};
struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
};

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
};

// Device scratch of one match-find step.
struct Scratch {
    DevBuf packed, counts, cand, seg;
    DevBuf zslots, zovs, zaux, zplan;  // Zstd entropy stage: frame slots, offset codes, per-window words, plans
};

// One stage of the host-buffer pipeline: its own stream, input, scratch and
// outputs, so that the copies of one slice overlap the kernels of another.
struct Slot {
    Scratch sc;
    DevBuf in, offsets, seqs, lz_packed, lz_has, frames, foff;
    HostBuf h_off, h_packed, h_foff;
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;      // the slice's kernels (and small copies) are done
    cudaEvent_t ev_out = nullptr;  // the slice's results have left its device buffers
    bool busy = false;
    size_t b0 = 0, sb = 0, off = 0, len = 0;
};

}  // namespace

struct gcz_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t out_stream = nullptr;  // copies of results back to the host (host-buffer pipeline)
    std::mutex mu;
    std::string err;
    uint32_t *d_status = nullptr;
    Scratch sc;      // scratch of the _device entry points
    Slot slots[4];   // host-buffer pipelines: each rotates over all four, three slices in flight
    uint32_t slice_windows = 512;          // windows per pipeline slice (32 MiB)
    uint32_t frames_slice_windows = 512;   // ... of the GPU frames pipeline (32 MiB, four slots)
    int staged = 1;
    int algo = 2;          // 1: fused single-warp kernels, 2: candidate sweep + second stage
    int parse_ctas = 3;    // second-stage CTAs per SM
    int seg_width = 1024;  // Zstd speculative segment: 1024 per 8-lane group, or 2048/4096/8192 per warp
    int sweep_warps = 7;   // candidate-sweep windows per CTA (4-7)
    int sweep_groups = 0;  // candidate sweep's equal-hash grouping: 0/1 after a read-back (match_any/ballots), 2/3 one block ahead
    int sweep_prefetch = 4;  // candidate sweep's L2 prefetch distance of the input, in 128-byte blocks (0, 4, 8)
    int lzma_ctas = 3;     // LZMA2 second-stage CTAs per SM
    int lzma_threads = 1024;  // LZMA2 second-stage threads per CTA (256, 512 or 1024)
    // profiling
    bool prof = false;
    std::vector<EventPair> events;
    size_t ev_used = 0;
    uint64_t match_launches = 0, all_launches = 0;
};

namespace {

int fail(gcz_ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

}  // namespace

int gcz_internal_fail(gcz_ctx *c, int code, const char *msg) {
    if (!c) return code;
    std::lock_guard<std::mutex> lk(c->mu);
    c->err = msg;
    return code;
}

namespace {

#define GCZ_CUDA(c, call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail((c), GCZ_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                 \
    } while (0)

int ensure_dev(gcz_ctx *c, DevBuf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return GCZ_OK;
    // Grow by at least a quarter, in 2 MiB steps: inputs that creep upwards
    // (request batches) reallocate a few times, not on every new maximum --
    // each cudaFree waits for the whole device.
    if (b.cap) bytes = std::max(bytes, b.cap + b.cap / 4);
    bytes = (bytes + (2u << 20) - 1) & ~static_cast<size_t>((2u << 20) - 1);
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GCZ_ENOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    b.cap = bytes;
    return GCZ_OK;
}

int ensure_host(gcz_ctx *c, HostBuf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return GCZ_OK;
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMallocHost(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GCZ_ENOMEM, "cudaMallocHost(%zu): %s", bytes, cudaGetErrorString(e));
    }
    b.cap = bytes;
    return GCZ_OK;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

cudaStream_t pick_stream(gcz_ctx *c, void *s) { return s ? static_cast<cudaStream_t>(s) : c->stream; }

// Bracket one match-find launch with events when profiling.
struct ProfScope {
    gcz_ctx *c;
    cudaStream_t st;
    EventPair *ev = nullptr;
    ProfScope(gcz_ctx *c_, cudaStream_t s) : c(c_), st(s) {
        c->match_launches++;
        if (!c->prof) return;
        if (c->ev_used == c->events.size()) {
            if (c->events.size() >= 65536) return;
            EventPair p;
            if (cudaEventCreate(&p.a) != cudaSuccess || cudaEventCreate(&p.b) != cudaSuccess) return;
            c->events.push_back(p);
        }
        ev = &c->events[c->ev_used++];
        cudaEventRecord(ev->a, st);
    }
    ~ProfScope() {
        if (ev) cudaEventRecord(ev->b, st);
    }
};

int read_status(gcz_ctx *c, cudaStream_t st) {
    uint32_t h = 0;
    GCZ_CUDA(c, cudaMemcpyAsync(&h, c->d_status, 4, cudaMemcpyDeviceToHost, st));
    GCZ_CUDA(c, cudaStreamSynchronize(st));
    if (h) {
        GCZ_CUDA(c, cudaMemsetAsync(c->d_status, 0, 4, st));
        GCZ_CUDA(c, cudaStreamSynchronize(st));
        if (h & 2u) return fail(c, GCZ_ECAPACITY, "output capacity exceeded (device status %u)", h);
        if (h & 4u) return fail(c, GCZ_EINVAL, "sequences do not describe their windows (device status %u)", h);
        return fail(c, GCZ_EDEVICE, "kernel reported status %u (bounded wait expired)", h);
    }
    return GCZ_OK;
}

size_t nwin(size_t n) { return (n + kW - 1) / kW; }

// Zstd on device memory for one contiguous range of windows: packed sequences
// into ctx scratch, counts, offsets (num+1, relative), compact expansion.
// With `wins`, n is the slab size and nbw the number of windows in the table.
int zstd_device_core(gcz_ctx *c, Scratch &sc, const uint8_t *d_src, size_t n, uint32_t depth, void *d_seqs,
                     uint64_t capacity, uint64_t *d_offsets, cudaStream_t st, const gcz::WinDesc *wins = nullptr,
                     size_t nbw = 0, bool rec8 = false) {
    const size_t nb = wins ? nbw : nwin(n);
    int r;
    if ((r = ensure_dev(c, sc.packed, nb * (size_t)kMaxSeqs * 8)) != GCZ_OK) return r;
    if ((r = ensure_dev(c, sc.counts, nb * 4)) != GCZ_OK) return r;
    uint32_t *counts = static_cast<uint32_t *>(sc.counts.p);
    const bool split = c->algo == 2 || wins;  // window tables run on the split kernels only
    if (split) {
        if ((r = ensure_dev(c, sc.cand, n * 2 + 64)) != GCZ_OK) return r;
        if ((r = ensure_dev(c, sc.seg, gcz::zstd2_seg_scratch_entries((uint32_t)nb) * 8)) != GCZ_OK) return r;
    }
    // The profiled interval covers the whole match-find step (all its kernels).
    ProfScope ps(c, st);
    if (split) {
        uint16_t *cand = static_cast<uint16_t *>(sc.cand.p);
        GCZ_CUDA(c, gcz::launch_cand_sweep(d_src, n, kW, (uint32_t)nb, cand, c->num_sms, st, wins, c->sweep_warps,
                                           c->sweep_groups, c->sweep_prefetch));
        gcz::Zstd2Launch l{};
        l.src = d_src;
        l.cand = cand;
        l.n = n;
        l.window = kW;
        l.num_windows = (uint32_t)nb;
        l.search_depth = depth;
        l.max_seqs = kMaxSeqs;
        l.seg = sc.seg.p;
        l.packed = sc.packed.p;
        l.seq_counts = counts;
        l.status = c->d_status;
        l.num_sms = c->num_sms;
        l.ctas_per_sm = c->parse_ctas;
        l.seg_width = (uint32_t)c->seg_width;
        l.wins = wins;
        GCZ_CUDA(c, gcz::launch_zstd_parse(l, st));
        c->all_launches += 2;
    } else {
        gcz::ZstdLaunch l{};
        l.src = d_src;
        l.n = n;
        l.window = kW;
        l.num_windows = (uint32_t)nb;
        l.search_depth = depth;
        l.max_seqs = kMaxSeqs;
        l.packed = sc.packed.p;
        l.seq_counts = counts;
        l.status = c->d_status;
        l.num_sms = c->num_sms;
        l.staged = c->staged;
        GCZ_CUDA(c, gcz::launch_zstd_match(l, st));
        c->all_launches += 1;
    }
    GCZ_CUDA(c, gcz::launch_scan_counts(counts, (uint32_t)nb, d_offsets, st));
    if (rec8)
        GCZ_CUDA(c, gcz::launch_compact_seqs(sc.packed.p, counts, d_offsets, (uint32_t)nb, kMaxSeqs, d_seqs, capacity,
                                             c->d_status, c->num_sms, st));
    else
        GCZ_CUDA(c, gcz::launch_expand_seqs(sc.packed.p, counts, d_offsets, (uint32_t)nb, kMaxSeqs, d_seqs, capacity,
                                            c->d_status, c->num_sms, st));
    c->all_launches += 2;
    return GCZ_OK;
}

int lzma_run(gcz_ctx *c, Scratch &sc, const gcz::LzmaLaunch &l, cudaStream_t st) {
    int r;
    const bool split = c->algo == 2 || l.wins;
    if (split && (r = ensure_dev(c, sc.cand, l.n * 2 + 64)) != GCZ_OK) return r;
    ProfScope ps(c, st);
    if (split) {
        uint16_t *cand = static_cast<uint16_t *>(sc.cand.p);
        GCZ_CUDA(c, gcz::launch_cand_sweep(l.src, l.n, l.window, l.num_windows, cand, c->num_sms, st, l.wins,
                                           c->sweep_warps, c->sweep_groups, c->sweep_prefetch));
        gcz::LzmaLaunch lv = l;
        lv.ctas_per_sm = c->lzma_ctas;
        lv.threads = c->lzma_threads;
        GCZ_CUDA(c, gcz::launch_lzma_verify(lv, cand, st));
        c->all_launches += 2;
    } else {
        GCZ_CUDA(c, gcz::launch_lzma_match(l, st));
        c->all_launches += 1;
    }
    return GCZ_OK;
}

// Zstd frames of windows [0, nwin(n)) from their ZSTD_Sequence records:
// frames back to back in d_out, frame offsets (nwin+1) in d_frame_offsets.
int zenc_core(gcz_ctx *c, Scratch &sc, const uint8_t *d_src, size_t n, const void *d_seqs,
              const uint64_t *d_seq_offsets, uint8_t *d_out, uint64_t out_capacity, uint64_t *d_frame_offsets,
              cudaStream_t st, const gcz::WinDesc *wins = nullptr, size_t nbw = 0) {
    const size_t nb = wins ? nbw : nwin(n);
    int r;
    if ((r = ensure_dev(c, sc.zslots, nb * (size_t)gcz::kZencSlot)) != GCZ_OK) return r;
    if ((r = ensure_dev(c, sc.zovs, nb * (size_t)gcz::kZencMaxSeqs * 4)) != GCZ_OK) return r;
    if ((r = ensure_dev(c, sc.zaux, nb * 12 + 64)) != GCZ_OK) return r;
    if ((r = ensure_dev(c, sc.zplan, nb * ((size_t)gcz::kZencPlanBytes + 1024))) != GCZ_OK) return r;
    gcz::ZencLaunch l{};
    l.src = d_src;
    l.n = n;
    l.window = kW;
    l.num_windows = (uint32_t)nb;
    l.seqs = d_seqs;
    l.seq_offsets = d_seq_offsets;
    l.slots = static_cast<uint8_t *>(sc.zslots.p);
    l.ovs = static_cast<uint32_t *>(sc.zovs.p);
    l.sec_off = static_cast<uint32_t *>(sc.zaux.p);
    l.fsize = l.sec_off + nb;
    l.raw = reinterpret_cast<uint8_t *>(l.fsize + nb);
    l.plan = static_cast<uint8_t *>(sc.zplan.p);
    l.hist = reinterpret_cast<uint32_t *>(l.plan + nb * (size_t)gcz::kZencPlanBytes);
    l.status = c->d_status;
    l.num_sms = c->num_sms;
    l.wins = wins;
    GCZ_CUDA(c, gcz::launch_zenc(l, st));
    GCZ_CUDA(c, gcz::launch_scan_counts(l.fsize, (uint32_t)nb, d_frame_offsets, st));
    GCZ_CUDA(c, gcz::launch_zenc_compact(l, d_frame_offsets, d_out, out_capacity, st));
    c->all_launches += 6;
    return GCZ_OK;
}

int lzma_device_core(gcz_ctx *c, Scratch &sc, const uint8_t *d_src, size_t n, uint32_t depth, uint32_t *d_packed,
                     uint8_t *d_has, cudaStream_t st) {
    const size_t nb = nwin(n);
    gcz::LzmaLaunch l{};
    l.src = d_src;
    l.n = n;
    l.window = kW;
    l.num_windows = (uint32_t)nb;
    l.search_depth = depth;
    l.max_matches = GCZ_LZMA2_MAX_MATCHES;
    l.packed = d_packed;
    l.has_matches = d_has;
    l.status = c->d_status;
    l.num_sms = c->num_sms;
    l.staged = c->staged;
    return lzma_run(c, sc, l, st);
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

// =========================================================================== context

extern "C" int gcz_create(int device_id, gcz_ctx **out) {
    if (!out) return GCZ_EINVAL;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device_id < 0 || device_id >= count) {
        cudaGetLastError();
        return GCZ_EINVAL;
    }
    gcz_ctx *c = new (std::nothrow) gcz_ctx();
    if (!c) return GCZ_ENOMEM;
    c->device = device_id;
    DeviceGuard g(device_id);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device_id) != cudaSuccess) {
        delete c;
        return GCZ_ECUDA;
    }
    c->num_sms = prop.multiProcessorCount;
    bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&c->d_status, 16) == cudaSuccess && cudaMemset(c->d_status, 0, 16) == cudaSuccess;
    for (Slot &sl : c->slots)
        ok = ok && cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&sl.ev_out, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return GCZ_ECUDA;
    }
    *out = c;
    return GCZ_OK;
}

extern "C" void gcz_destroy(gcz_ctx *c) {
    if (!c) return;
    {
        DeviceGuard g(c->device);
        cudaStreamSynchronize(c->stream);
        auto free_scratch = [](Scratch &x) {
            for (DevBuf *b : {&x.packed, &x.counts, &x.cand, &x.seg, &x.zslots, &x.zovs, &x.zaux, &x.zplan})
                if (b->p) cudaFree(b->p);
        };
        free_scratch(c->sc);
        for (Slot &sl : c->slots) {
            if (sl.st) cudaStreamSynchronize(sl.st);
            free_scratch(sl.sc);
            for (DevBuf *b : {&sl.in, &sl.offsets, &sl.seqs, &sl.lz_packed, &sl.lz_has, &sl.frames, &sl.foff})
                if (b->p) cudaFree(b->p);
            for (HostBuf *b : {&sl.h_off, &sl.h_packed, &sl.h_foff})
                if (b->p) cudaFreeHost(b->p);
            if (sl.ev) cudaEventDestroy(sl.ev);
            if (sl.ev_out) cudaEventDestroy(sl.ev_out);
            if (sl.st) cudaStreamDestroy(sl.st);
        }
        if (c->out_stream) {
            cudaStreamSynchronize(c->out_stream);
            cudaStreamDestroy(c->out_stream);
        }
        for (auto &e : c->events) {
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
        if (c->d_status) cudaFree(c->d_status);
        cudaStreamDestroy(c->stream);
    }
    delete c;
}

extern "C" const char *gcz_last_error(const gcz_ctx *c) { return c ? c->err.c_str() : "null context"; }
extern "C" int gcz_device(const gcz_ctx *c) { return c ? c->device : -1; }
extern "C" const char *gcz_version(void) { return "gcz 0.1 (sm_100a)"; }

extern "C" int gcz_set_option(gcz_ctx *c, const char *key, long value) {
    if (!c || !key) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!strcmp(key, "staged")) {
        c->staged = value ? 1 : 0;
        return GCZ_OK;
    }
    if (!strcmp(key, "algo") && (value == 1 || value == 2)) {
        c->algo = (int)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "slice_windows") && value >= 1 && value <= (1L << 20)) {
        c->slice_windows = (uint32_t)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "frames_slice_windows") && value >= 1 && value <= (1L << 20)) {
        c->frames_slice_windows = (uint32_t)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "parse_ctas") && value >= 1 && value <= 8) {
        c->parse_ctas = (int)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "parse_seg") && (value == 512 || value == 1024 || value == 2048 || value == 4096 || value == 8192)) {
        c->seg_width = (int)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "sweep_warps") && value >= 4 && value <= 7) {
        c->sweep_warps = (int)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "sweep_groups") && value >= 0 && value <= 3) {
        c->sweep_groups = (int)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "sweep_prefetch") && value >= 0 && value <= 64) {
        c->sweep_prefetch = (int)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "lzma_ctas") && value >= 1 && value <= 8) {
        c->lzma_ctas = (int)value;
        return GCZ_OK;
    }
    if (!strcmp(key, "lzma_threads") && (value == 256 || value == 512 || value == 1024)) {
        c->lzma_threads = (int)value;
        return GCZ_OK;
    }
    return fail(c, GCZ_EINVAL, "unknown option '%s'", key);
}

namespace {
// One CTA waits on an mbarrier that nothing will ever complete.  The wait is
// bounded like every wait in the match finders; when it runs out the kernel
// records the timeout in the status word and returns.
__global__ void selftest_wait_kernel(uint32_t *status, uint32_t max_iter) {
    __shared__ alignas(8) uint64_t bar;
    if (threadIdx.x == 0) {
        gcz::mbar_init(&bar, 1);
        gcz::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !gcz::mbar_wait(&bar, 0u, max_iter)) atomicOr(status, gcz::kErrTmaTimeout);
}
}  // namespace

extern "C" int gcz_query(gcz_ctx *c, const char *key, long *value) {
    if (!c || !key || !value) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!strcmp(key, "algo")) {
        *value = c->algo;
        return GCZ_OK;
    }
    const struct {
        const char *k;
        long v;
    } knobs[] = {{"staged", c->staged},          {"parse_ctas", c->parse_ctas},
                 {"parse_seg", c->seg_width},    {"sweep_warps", c->sweep_warps},
                 {"sweep_groups", c->sweep_groups}, {"sweep_prefetch", c->sweep_prefetch},
                 {"lzma_ctas", c->lzma_ctas},    {"lzma_threads", c->lzma_threads},
                 {"slice_windows", (long)c->slice_windows},
                 {"frames_slice_windows", (long)c->frames_slice_windows}};
    for (const auto &kv : knobs)
        if (!strcmp(key, kv.k)) {
            *value = kv.v;
            return GCZ_OK;
        }
    if (!strcmp(key, "fallback_windows")) {  // windows whose speculative parse fell back (since creation)
        DeviceGuard g(c->device);
        uint32_t h[2] = {0, 0};
        GCZ_CUDA(c, cudaMemcpy(h, c->d_status, 8, cudaMemcpyDeviceToHost));
        *value = (long)h[1];
        return GCZ_OK;
    }
    if (!strcmp(key, "binary_version") || !strcmp(key, "ptx_version")) {
        // The architecture the loaded kernel image was compiled for, as the
        // runtime reports it (major * 10 + minor: 100 for sm_100a).
        DeviceGuard g(c->device);
        cudaFuncAttributes fa{};
        GCZ_CUDA(c, cudaFuncGetAttributes(&fa, selftest_wait_kernel));
        *value = key[0] == 'b' ? (long)fa.binaryVersion : (long)fa.ptxVersion;
        return GCZ_OK;
    }
    return fail(c, GCZ_EINVAL, "unknown key '%s'", key);
}

extern "C" int gcz_sync(gcz_ctx *c, void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    return read_status(c, pick_stream(c, stream));
}


extern "C" int gcz_selftest_wait_timeout(gcz_ctx *c, uint32_t max_iterations) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    selftest_wait_kernel<<<1, 32, 0, c->stream>>>(c->d_status, max_iterations);
    GCZ_CUDA(c, cudaGetLastError());
    return read_status(c, c->stream);
}

// =========================================================================== Zstd

extern "C" uint32_t gcz_zstd_search_depth_for_level(uint32_t level) {
    return level == 1 ? 16u : (level == 2 ? 64u : 1u);  // compress_zstd_custom.rs:57-61
}
extern "C" size_t gcz_num_windows(size_t n) { return nwin(n); }
extern "C" size_t gcz_zstd_max_sequences(size_t n) {
    // A window of s bytes holds at most floor((s-1)/3) sequences (position 0 is
    // always a literal and every match is >= 3 bytes); never more than the
    // kernel's per-window stride.
    size_t total = 0, full = n / kW, rem = n % kW;
    total = full * std::min<size_t>((kW - 1) / 3, kMaxSeqs);
    if (rem) total += rem > 1 ? (rem - 1) / 3 : 0;
    return total;
}

extern "C" int gcz_zstd_match_find_device(gcz_ctx *c, const uint8_t *d_src, size_t n, uint32_t search_depth,
                                          gcz_zstd_sequence *d_seqs, size_t seq_capacity, uint64_t *d_offsets,
                                          void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if ((n && (!d_src || !d_seqs)) || !d_offsets) return fail(c, GCZ_EINVAL, "null pointer");
    if (!aligned16(d_src)) return fail(c, GCZ_EINVAL, "d_src must be 16-byte aligned");
    if (nwin(n) > 0xFFFFFFFFu) return fail(c, GCZ_EINVAL, "input too large");
    DeviceGuard g(c->device);
    cudaStream_t st = pick_stream(c, stream);
    if (n == 0) {
        GCZ_CUDA(c, cudaMemsetAsync(d_offsets, 0, 8, st));
        return GCZ_OK;
    }
    return zstd_device_core(c, c->sc, d_src, n, search_depth, d_seqs, seq_capacity, d_offsets, st);
}

namespace {
// Second half of a Zstd pipeline slice: wait for its offsets, then queue the
// copy of its sequences into the caller's array.
int zstd_finish_slot(gcz_ctx *c, Slot &sl, void *seqs, size_t cap, uint64_t *offsets, uint64_t &done,
                     uint32_t rec_bytes) {
    GCZ_CUDA(c, cudaEventSynchronize(sl.ev));
    const uint64_t *ho = static_cast<const uint64_t *>(sl.h_off.p);
    const uint64_t total = ho[sl.sb];
    sl.busy = false;
    if (done + total > cap)
        return fail(c, GCZ_ECAPACITY, "need %llu sequences, capacity %zu", (unsigned long long)(done + total), cap);
    // On the copy-out stream, so that the slot's next copy-in does not queue behind it.
    if (total)
        GCZ_CUDA(c, cudaMemcpyAsync(static_cast<uint8_t *>(seqs) + done * rec_bytes, sl.seqs.p, total * rec_bytes,
                                    cudaMemcpyDeviceToHost, c->out_stream));
    GCZ_CUDA(c, cudaEventRecord(sl.ev_out, c->out_stream));
    for (size_t i = 1; i <= sl.sb; i++) offsets[sl.b0 + i] = done + ho[i];
    done += total;
    return GCZ_OK;
}

// Windows in the pipeline slice that starts at window b0 of nb.  Slices ramp
// up from a quarter of `maxw` (the first copy-in and the last kernels and
// copy-out overlap nothing, so short ones there shorten the whole call) to
// maxw, and halve again over the last 2*maxw windows.
size_t next_slice(size_t b0, size_t nb, size_t maxw) {
    const size_t q = std::max<size_t>(maxw / 4, 1), rem = nb - b0;
    size_t s = std::min(maxw, std::max(q, b0));
    if (rem <= 2 * maxw) s = std::min(s, std::max(q, rem / 2));
    return std::min(s, rem);
}

int drain_slots(gcz_ctx *c) {
    for (Slot &sl : c->slots) GCZ_CUDA(c, cudaStreamSynchronize(sl.st));
    GCZ_CUDA(c, cudaStreamSynchronize(c->out_stream));
    return read_status(c, c->stream);
}
}  // namespace

// Slices of slice_windows windows rotate over the S = 4 slots (streams): the
// H2D copy and kernels of slice k run while earlier slices' sequences are
// copied back.  Slice k is queued before the host waits for slice k-(S-1) and
// queues its copy-out, so the host's wait never holds back the next copy-in
// (two slots, finishing slice k-1: 47.7 GB/s for 1 GiB; four: 48.8, against
// 51.8 for the same copies with no kernels).
namespace {
// The host-buffer Zstd pipeline: records of rec_bytes (16: ZSTD_Sequence, 8:
// packed {ll | (ml-3) << 16, off}) back to back in `seqs`.
int zstd_host_pipeline(gcz_ctx *c, const uint8_t *src, size_t n, uint32_t search_depth, void *seqs,
                       size_t seq_capacity, uint64_t *offsets, uint32_t rec_bytes) {
    DeviceGuard g(c->device);
    const size_t nb = nwin(n);
    offsets[0] = 0;
    int r = GCZ_OK;
    uint64_t done = 0;  // sequences copied so far
    constexpr size_t kS = sizeof(c->slots) / sizeof(c->slots[0]);
    size_t k = 0;
    for (size_t b0 = 0, sb = 0; b0 < nb && r == GCZ_OK; b0 += sb, ++k) {
        Slot &sl = c->slots[k % kS];  // slice k-S, its last user, was finished one iteration ago
        sb = next_slice(b0, nb, c->slice_windows);
        sl.b0 = b0;
        sl.sb = sb;
        sl.off = b0 * (size_t)kW;
        sl.len = std::min(n - sl.off, sb * (size_t)kW);
        const size_t slice_cap = gcz_zstd_max_sequences(sl.len);
        if ((r = ensure_dev(c, sl.in, sb * (size_t)kW + 64)) != GCZ_OK) break;
        if ((r = ensure_dev(c, sl.offsets, (sb + 1) * 8)) != GCZ_OK) break;
        if ((r = ensure_dev(c, sl.seqs, std::max<size_t>(slice_cap, 1) * 16)) != GCZ_OK) break;
        if ((r = ensure_host(c, sl.h_off, (sb + 1) * 8)) != GCZ_OK) break;
        GCZ_CUDA(c, cudaMemcpyAsync(sl.in.p, src + sl.off, sl.len, cudaMemcpyHostToDevice, sl.st));
        GCZ_CUDA(c, cudaStreamWaitEvent(sl.st, sl.ev_out, 0));  // sl.seqs free again
        if ((r = zstd_device_core(c, sl.sc, static_cast<const uint8_t *>(sl.in.p), sl.len, search_depth, sl.seqs.p,
                                  slice_cap, static_cast<uint64_t *>(sl.offsets.p), sl.st, nullptr, 0,
                                  rec_bytes == 8)) != GCZ_OK)
            break;
        GCZ_CUDA(c, cudaMemcpyAsync(sl.h_off.p, sl.offsets.p, (sb + 1) * 8, cudaMemcpyDeviceToHost, sl.st));
        GCZ_CUDA(c, cudaEventRecord(sl.ev, sl.st));
        sl.busy = true;
        if (k >= kS - 1) {  // finish slice k-(S-1); slices finish in order, so records stay in order
            Slot &old = c->slots[(k - (kS - 1)) % kS];
            if (old.busy) r = zstd_finish_slot(c, old, seqs, seq_capacity, offsets, done, rec_bytes);
        }
    }
    for (size_t j = k >= kS - 1 ? k - (kS - 1) : 0; j < k && r == GCZ_OK; ++j) {
        Slot &rest = c->slots[j % kS];
        if (rest.busy) r = zstd_finish_slot(c, rest, seqs, seq_capacity, offsets, done, rec_bytes);
    }
    for (Slot &sl : c->slots) sl.busy = false;
    const int r2 = drain_slots(c);
    return r != GCZ_OK ? r : r2;
}
}  // namespace

extern "C" int gcz_zstd_match_find(gcz_ctx *c, const uint8_t *src, size_t n, uint32_t search_depth,
                                   gcz_zstd_sequence *seqs, size_t seq_capacity, uint64_t *offsets) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if ((n && (!src || !seqs)) || !offsets) return fail(c, GCZ_EINVAL, "null pointer");
    return zstd_host_pipeline(c, src, n, search_depth, seqs, seq_capacity, offsets, 16);
}

extern "C" int gcz_zstd_match_find_packed(gcz_ctx *c, const uint8_t *src, size_t n, uint32_t search_depth,
                                          uint64_t *records, size_t record_capacity, uint64_t *offsets) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if ((n && (!src || !records)) || !offsets) return fail(c, GCZ_EINVAL, "null pointer");
    return zstd_host_pipeline(c, src, n, search_depth, records, record_capacity, offsets, 8);
}

extern "C" int gcz_zstd_encode_frames_device(gcz_ctx *c, const uint8_t *d_src, size_t n,
                                             const gcz_zstd_sequence *d_seqs, const uint64_t *d_seq_offsets,
                                             uint8_t *d_out, size_t out_capacity, uint64_t *d_frame_offsets,
                                             void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if ((n && (!d_src || !d_seqs || !d_seq_offsets || !d_out)) || !d_frame_offsets)
        return fail(c, GCZ_EINVAL, "null pointer");
    if (!aligned16(d_src)) return fail(c, GCZ_EINVAL, "d_src must be 16-byte aligned");
    if (nwin(n) > 0xFFFFFFFFu) return fail(c, GCZ_EINVAL, "input too large");
    DeviceGuard g(c->device);
    cudaStream_t st = pick_stream(c, stream);
    if (n == 0) {
        GCZ_CUDA(c, cudaMemsetAsync(d_frame_offsets, 0, 8, st));
        return GCZ_OK;
    }
    return zenc_core(c, c->sc, d_src, n, d_seqs, d_seq_offsets, d_out, out_capacity, d_frame_offsets, st);
}

// Host bytes to Zstd frames entirely on the GPU.  Slices rotate over the S = 4
// pipeline slots, and slice k is queued before the host waits for slice
// k-(S-1) and queues the copy-out of its frames.  Slice k's copy-in then waits
// on the GPU only for the kernels of slice k-S, the last user of its slot, so
// the copy engine keeps streaming while the kernels of up to S-1 slices share
// the SMs.  (With two slots the copy-in waited for slice k-2's kernels; the
// kernels take about as long as the copies, so copies and kernels took turns:
// 33 GB/s for 1 GiB against 42 with four slots of 32 MiB.)
extern "C" int gcz_zstd_compress_frames_gpu(gcz_ctx *c, const uint8_t *src, size_t n, uint32_t level, uint8_t *out,
                                            size_t out_capacity, uint64_t *frame_sizes, size_t *out_size) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if ((n && (!src || !out || !frame_sizes)) || !out_size) return fail(c, GCZ_EINVAL, "null pointer");
    *out_size = 0;
    DeviceGuard g(c->device);
    const uint32_t depth = gcz_zstd_search_depth_for_level(level);
    const size_t nb = nwin(n);
    size_t written = 0;
    int r = GCZ_OK;
    auto finish = [&](Slot &sl) -> int {
        GCZ_CUDA(c, cudaEventSynchronize(sl.ev));
        sl.busy = false;
        const uint64_t *ho = static_cast<const uint64_t *>(sl.h_foff.p);
        const uint64_t total = ho[sl.sb];
        if (written + total > out_capacity)
            return fail(c, GCZ_ECAPACITY, "frames need %llu bytes, capacity %zu",
                        (unsigned long long)(written + total), out_capacity);
        if (total)
            GCZ_CUDA(c, cudaMemcpyAsync(out + written, sl.frames.p, total, cudaMemcpyDeviceToHost, c->out_stream));
        GCZ_CUDA(c, cudaEventRecord(sl.ev_out, c->out_stream));
        for (size_t i = 0; i < sl.sb; ++i) frame_sizes[sl.b0 + i] = ho[i + 1] - ho[i];
        written += total;
        return GCZ_OK;
    };
    constexpr size_t kFrameSlots = sizeof(c->slots) / sizeof(c->slots[0]);
    size_t k = 0;
    for (size_t b0 = 0, sb = 0; b0 < nb && r == GCZ_OK; b0 += sb, ++k) {
        Slot &sl = c->slots[k % kFrameSlots];  // slice k-S, its last user, was finished one iteration ago
        sb = next_slice(b0, nb, c->frames_slice_windows);
        sl.b0 = b0;
        sl.sb = sb;
        sl.off = b0 * (size_t)kW;
        sl.len = std::min(n - sl.off, sb * (size_t)kW);
        const size_t slice_cap = gcz_zstd_max_sequences(sl.len);
        const size_t fbound = gcz_zstd_frames_bound(sl.len);
        if ((r = ensure_dev(c, sl.in, sb * (size_t)kW + 64)) != GCZ_OK) break;
        if ((r = ensure_dev(c, sl.offsets, (sb + 1) * 8)) != GCZ_OK) break;
        if ((r = ensure_dev(c, sl.seqs, std::max<size_t>(slice_cap, 1) * 16)) != GCZ_OK) break;
        if ((r = ensure_dev(c, sl.frames, fbound)) != GCZ_OK) break;
        if ((r = ensure_dev(c, sl.foff, (sb + 1) * 8)) != GCZ_OK) break;
        if ((r = ensure_host(c, sl.h_foff, (sb + 1) * 8)) != GCZ_OK) break;
        GCZ_CUDA(c, cudaMemcpyAsync(sl.in.p, src + sl.off, sl.len, cudaMemcpyHostToDevice, sl.st));
        const uint8_t *d_in = static_cast<const uint8_t *>(sl.in.p);
        uint64_t *d_off = static_cast<uint64_t *>(sl.offsets.p);
        if ((r = zstd_device_core(c, sl.sc, d_in, sl.len, depth, sl.seqs.p, slice_cap, d_off, sl.st)) != GCZ_OK) break;
        GCZ_CUDA(c, cudaStreamWaitEvent(sl.st, sl.ev_out, 0));  // sl.frames free again
        if ((r = zenc_core(c, sl.sc, d_in, sl.len, sl.seqs.p, d_off, static_cast<uint8_t *>(sl.frames.p), fbound,
                           static_cast<uint64_t *>(sl.foff.p), sl.st)) != GCZ_OK)
            break;
        GCZ_CUDA(c, cudaMemcpyAsync(sl.h_foff.p, sl.foff.p, (sb + 1) * 8, cudaMemcpyDeviceToHost, sl.st));
        GCZ_CUDA(c, cudaEventRecord(sl.ev, sl.st));
        sl.busy = true;
        if (k >= kFrameSlots - 1) {  // finish slice k-(S-1); slices finish in order, so frames stay in order
            Slot &old = c->slots[(k - (kFrameSlots - 1)) % kFrameSlots];
            if (old.busy) r = finish(old);
        }
    }
    for (size_t j = k >= kFrameSlots - 1 ? k - (kFrameSlots - 1) : 0; j < k && r == GCZ_OK; ++j) {
        Slot &rest = c->slots[j % kFrameSlots];
        if (rest.busy) r = finish(rest);
    }
    for (Slot &sl : c->slots) sl.busy = false;
    const int r2 = drain_slots(c);
    if (r == GCZ_OK && r2 == GCZ_OK) *out_size = written;
    return r != GCZ_OK ? r : r2;
}

extern "C" int gcz_zstd_match_find_ref_layout_device(gcz_ctx *c, const uint8_t *d_input, uint32_t *d_sequences,
                                                     uint8_t *d_literals, uint32_t *d_seq_counts,
                                                     uint32_t *d_lit_counts, uint32_t chunk_size, uint32_t num_chunks,
                                                     uint32_t total_input_size, uint32_t search_depth,
                                                     uint32_t max_sequences_per_chunk, void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (chunk_size == 0 || chunk_size > 65536 || (chunk_size & 15u))
        return fail(c, GCZ_EINVAL, "chunk_size must be a multiple of 16 in [16, 65536]");
    if (!d_input || !d_sequences || !d_seq_counts) return fail(c, GCZ_EINVAL, "null pointer");
    if (!aligned16(d_input)) return fail(c, GCZ_EINVAL, "d_input must be 16-byte aligned");
    // Windows past the input (the reference computes a negative size there) are not processed.
    uint64_t nb = ((uint64_t)total_input_size + chunk_size - 1) / chunk_size;
    if (nb > num_chunks) nb = num_chunks;
    DeviceGuard g(c->device);
    cudaStream_t st = pick_stream(c, stream);
    uint64_t n_eff = std::min<uint64_t>(total_input_size, nb * chunk_size);
    if (c->algo == 2) {
        int r;
        if ((r = ensure_dev(c, c->sc.cand, n_eff * 2 + 64)) != GCZ_OK) return r;
        if ((r = ensure_dev(c, c->sc.seg, gcz::zstd2_seg_scratch_entries((uint32_t)nb) * 8)) != GCZ_OK) return r;
        ProfScope ps(c, st);
        uint16_t *cand = static_cast<uint16_t *>(c->sc.cand.p);
        GCZ_CUDA(c, gcz::launch_cand_sweep(d_input, n_eff, chunk_size, (uint32_t)nb, cand, c->num_sms, st, nullptr,
                                           c->sweep_warps, c->sweep_groups, c->sweep_prefetch));
        gcz::Zstd2Launch l{};
        l.src = d_input;
        l.cand = cand;
        l.n = n_eff;
        l.window = chunk_size;
        l.num_windows = (uint32_t)nb;
        l.search_depth = search_depth;
        l.max_seqs = max_sequences_per_chunk;
        l.seg = c->sc.seg.p;
        l.ref_seqs = d_sequences;
        l.seq_counts = d_seq_counts;
        l.lit_counts = d_lit_counts;
        l.status = c->d_status;
        l.num_sms = c->num_sms;
        l.ctas_per_sm = c->parse_ctas;
        l.seg_width = (uint32_t)c->seg_width;
        GCZ_CUDA(c, gcz::launch_zstd_parse(l, st));
        c->all_launches += 2;
    } else {
        gcz::ZstdLaunch l{};
        l.src = d_input;
        l.n = n_eff;
        l.window = chunk_size;
        l.num_windows = (uint32_t)nb;
        l.search_depth = search_depth;
        l.max_seqs = max_sequences_per_chunk;
        l.ref_seqs = d_sequences;
        l.seq_counts = d_seq_counts;
        l.lit_counts = d_lit_counts;
        l.status = c->d_status;
        l.num_sms = c->num_sms;
        l.staged = c->staged;
        ProfScope ps(c, st);
        GCZ_CUDA(c, gcz::launch_zstd_match(l, st));
        c->all_launches++;
    }
    if (d_literals) {
        GCZ_CUDA(c, gcz::launch_zstd_literals(d_input, n_eff, chunk_size, (uint32_t)nb, d_sequences, d_seq_counts,
                                              max_sequences_per_chunk, d_literals, c->num_sms, st));
        c->all_launches++;
    }
    return GCZ_OK;
}

// =========================================================================== LZMA2

extern "C" int gcz_lzma2_match_find_device(gcz_ctx *c, const uint8_t *d_src, size_t n, uint32_t search_depth,
                                           uint32_t *d_packed, uint8_t *d_has_matches, void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (n && !d_src) return fail(c, GCZ_EINVAL, "null pointer");
    if (!aligned16(d_src)) return fail(c, GCZ_EINVAL, "d_src must be 16-byte aligned");
    if (nwin(n) > 0xFFFFFFFFu) return fail(c, GCZ_EINVAL, "input too large");
    DeviceGuard g(c->device);
    if (n == 0) return GCZ_OK;
    return lzma_device_core(c, c->sc, d_src, n, search_depth, d_packed, d_has_matches, pick_stream(c, stream));
}

namespace {
// Host-side slices for the two LZMA2 host entry points, rotating over the
// S = 4 pipeline slots like the Zstd pipeline (slice k is queued before the
// host finishes slice k-(S-1)); `consume` sees each slice's packed results on
// the host once they have arrived, in slice order.
template <class Consume>
int lzma_host_slices(gcz_ctx *c, const uint8_t *src, size_t n, uint32_t depth, uint32_t *packed_out,
                     uint8_t *has_out, bool copy_packed, Consume consume) {
    const size_t nb = nwin(n);
    int r = GCZ_OK;
    auto finish = [&](Slot &sl) -> int {
        GCZ_CUDA(c, cudaEventSynchronize(sl.ev));
        sl.busy = false;
        consume(sl.off, sl.len, packed_out ? packed_out + sl.off : static_cast<const uint32_t *>(sl.h_packed.p));
        return GCZ_OK;
    };
    constexpr size_t kS = sizeof(c->slots) / sizeof(c->slots[0]);
    size_t k = 0;
    for (size_t b0 = 0, sb = 0; b0 < nb && r == GCZ_OK; b0 += sb, ++k) {
        Slot &sl = c->slots[k % kS];  // slice k-S, its last user, was finished one iteration ago
        sb = next_slice(b0, nb, c->slice_windows);
        sl.b0 = b0;
        sl.sb = sb;
        sl.off = b0 * (size_t)kW;
        sl.len = std::min(n - sl.off, sb * (size_t)kW);
        if ((r = ensure_dev(c, sl.in, sb * (size_t)kW + 64)) != GCZ_OK) break;
        if ((r = ensure_dev(c, sl.lz_packed, sb * (size_t)kW * 4)) != GCZ_OK) break;
        if ((r = ensure_dev(c, sl.lz_has, sb + 16)) != GCZ_OK) break;
        GCZ_CUDA(c, cudaMemcpyAsync(sl.in.p, src + sl.off, sl.len, cudaMemcpyHostToDevice, sl.st));
        if ((r = lzma_device_core(c, sl.sc, static_cast<const uint8_t *>(sl.in.p), sl.len, depth,
                                  static_cast<uint32_t *>(sl.lz_packed.p), static_cast<uint8_t *>(sl.lz_has.p),
                                  sl.st)) != GCZ_OK)
            break;
        if (copy_packed) {  // a has-only call (packed == NULL) copies back one byte per window
            uint32_t *dst = packed_out ? packed_out + sl.off : nullptr;
            if (!dst) {
                if ((r = ensure_host(c, sl.h_packed, sb * (size_t)kW * 4)) != GCZ_OK) break;
                dst = static_cast<uint32_t *>(sl.h_packed.p);
            }
            GCZ_CUDA(c, cudaMemcpyAsync(dst, sl.lz_packed.p, sl.len * 4, cudaMemcpyDeviceToHost, sl.st));
        }
        if (has_out) GCZ_CUDA(c, cudaMemcpyAsync(has_out + b0, sl.lz_has.p, sb, cudaMemcpyDeviceToHost, sl.st));
        GCZ_CUDA(c, cudaEventRecord(sl.ev, sl.st));
        sl.busy = true;
        if (k >= kS - 1) {  // finish slice k-(S-1), in slice order
            Slot &old = c->slots[(k - (kS - 1)) % kS];
            if (old.busy) r = finish(old);
        }
    }
    for (size_t j = k >= kS - 1 ? k - (kS - 1) : 0; j < k && r == GCZ_OK; ++j) {
        Slot &rest = c->slots[j % kS];
        if (rest.busy) r = finish(rest);
    }
    for (Slot &sl : c->slots) sl.busy = false;
    const int r2 = drain_slots(c);
    return r != GCZ_OK ? r : r2;
}
}  // namespace

extern "C" int gcz_lzma2_match_find(gcz_ctx *c, const uint8_t *src, size_t n, uint32_t search_depth,
                                    uint32_t *packed, uint8_t *has_matches) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (n && !src) return fail(c, GCZ_EINVAL, "null pointer");
    DeviceGuard g(c->device);
    return lzma_host_slices(c, src, n, search_depth, packed, has_matches, packed != nullptr,
                            [](size_t, size_t, const uint32_t *) {});
}

extern "C" int gcz_lzma2_find_matches(gcz_ctx *c, const uint8_t *src, size_t n, uint32_t max_matches,
                                      uint32_t *match_distances, uint32_t *match_lengths, uint32_t *match_counts) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (n && !src) return fail(c, GCZ_EINVAL, "null pointer");
    if (max_matches == 0) return fail(c, GCZ_EINVAL, "max_matches must be >= 1");
    DeviceGuard g(c->device);
    const size_t total_pos = nwin(n) * (size_t)kW;
    // Zero-fill first (alloc_zeros in the reference), then scatter the found matches.
    auto zero = [&](uint32_t *p, size_t count) {
        if (!p) return;
        const unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; t++)
            th.emplace_back([=] {
                const size_t a = count * t / nt, b = count * (t + 1) / nt;
                memset(p + a, 0, (b - a) * 4);
            });
        for (auto &x : th) x.join();
    };
    zero(match_counts, total_pos);
    zero(match_distances, total_pos * max_matches);
    zero(match_lengths, total_pos * max_matches);
    return lzma_host_slices(c, src, n, GCZ_LZMA2_SEARCH_DEPTH, nullptr, nullptr, true,
                            [&](size_t off, size_t len, const uint32_t *pk) {
                                for (size_t i = 0; i < len; i++) {
                                    const uint32_t v = pk[i];
                                    if (!v) continue;
                                    const size_t q = off + i;
                                    if (match_counts) match_counts[q] = 1;
                                    if (match_distances) match_distances[q * max_matches] = v & 0xFFFFu;
                                    if (match_lengths) match_lengths[q * max_matches] = v >> 16;
                                }
                            });
}

extern "C" int gcz_lzma2_match_find_ref_layout_device(gcz_ctx *c, const uint8_t *d_input, uint32_t *d_matches,
                                                      uint32_t *d_match_counts, uint32_t sub_block_size,
                                                      uint32_t num_sub_blocks, uint32_t total_input_size,
                                                      uint32_t max_matches_per_pos, uint32_t search_depth,
                                                      void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (sub_block_size == 0 || sub_block_size > 65536 || (sub_block_size & 15u))
        return fail(c, GCZ_EINVAL, "sub_block_size must be a multiple of 16 in [16, 65536]");
    if (max_matches_per_pos == 0) return fail(c, GCZ_EINVAL, "max_matches_per_pos must be >= 1");
    if (!d_input || !d_matches || !d_match_counts) return fail(c, GCZ_EINVAL, "null pointer");
    if (!aligned16(d_input)) return fail(c, GCZ_EINVAL, "d_input must be 16-byte aligned");
    uint64_t nb = ((uint64_t)total_input_size + sub_block_size - 1) / sub_block_size;
    if (nb > num_sub_blocks) nb = num_sub_blocks;
    DeviceGuard g(c->device);
    cudaStream_t st = pick_stream(c, stream);
    gcz::LzmaLaunch l{};
    l.src = d_input;
    l.n = std::min<uint64_t>(total_input_size, nb * sub_block_size);
    l.window = sub_block_size;
    l.num_windows = (uint32_t)nb;
    l.search_depth = search_depth;
    l.max_matches = max_matches_per_pos;
    l.ref_matches = d_matches;
    l.ref_counts = d_match_counts;
    l.status = c->d_status;
    l.num_sms = c->num_sms;
    l.staged = c->staged;
    return lzma_run(c, c->sc, l, st);
}

// =========================================================================== batches

static_assert(sizeof(gcz_window) == sizeof(gcz::WinDesc), "gcz_window mirrors the kernels' window table");

extern "C" size_t gcz_batch_num_windows(const size_t *sizes, size_t count) {
    size_t nb = 0;
    for (size_t i = 0; sizes && i < count; i++) nb += nwin(sizes[i]);
    return nb;
}

extern "C" int gcz_batch_layout(const size_t *sizes, size_t count, uint64_t *file_offsets, gcz_window *windows,
                                uint64_t *slab_bytes) {
    if ((count && !sizes) || !slab_bytes) return GCZ_EINVAL;
    uint64_t off = 0;
    size_t w = 0;
    for (size_t i = 0; i < count; i++) {
        off = (off + 15u) & ~uint64_t(15);
        if (file_offsets) file_offsets[i] = off;
        for (uint64_t s = 0; s < sizes[i]; s += kW, ++w) {
            if (windows) {
                windows[w].offset = off + s;
                windows[w].size = (uint32_t)std::min<uint64_t>(kW, sizes[i] - s);
                windows[w].file = (uint32_t)i;
            }
        }
        off += sizes[i];
    }
    *slab_bytes = (off + 15u) & ~uint64_t(15);
    return GCZ_OK;
}

extern "C" int gcz_zstd_match_find_batch_device(gcz_ctx *c, const uint8_t *d_slab, uint64_t slab_bytes,
                                                const gcz_window *d_windows, uint32_t num_windows,
                                                uint32_t search_depth, gcz_zstd_sequence *d_seqs,
                                                size_t seq_capacity, uint64_t *d_offsets, void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!d_offsets || (num_windows && (!d_slab || !d_windows || !d_seqs))) return fail(c, GCZ_EINVAL, "null pointer");
    if (!aligned16(d_slab)) return fail(c, GCZ_EINVAL, "d_slab must be 16-byte aligned");
    DeviceGuard g(c->device);
    cudaStream_t st = pick_stream(c, stream);
    if (num_windows == 0) {
        GCZ_CUDA(c, cudaMemsetAsync(d_offsets, 0, 8, st));
        return GCZ_OK;
    }
    return zstd_device_core(c, c->sc, d_slab, slab_bytes, search_depth, d_seqs, seq_capacity, d_offsets, st,
                            reinterpret_cast<const gcz::WinDesc *>(d_windows), num_windows);
}

extern "C" int gcz_lzma2_match_find_batch_device(gcz_ctx *c, const uint8_t *d_slab, uint64_t slab_bytes,
                                                 const gcz_window *d_windows, uint32_t num_windows,
                                                 uint32_t search_depth, uint32_t *d_packed, uint8_t *d_has_matches,
                                                 void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (num_windows && (!d_slab || !d_windows)) return fail(c, GCZ_EINVAL, "null pointer");
    if (!aligned16(d_slab)) return fail(c, GCZ_EINVAL, "d_slab must be 16-byte aligned");
    DeviceGuard g(c->device);
    if (num_windows == 0) return GCZ_OK;
    gcz::LzmaLaunch l{};
    l.src = d_slab;
    l.n = slab_bytes;
    l.window = kW;
    l.num_windows = num_windows;
    l.search_depth = search_depth;
    l.max_matches = GCZ_LZMA2_MAX_MATCHES;
    l.packed = d_packed;
    l.has_matches = d_has_matches;
    l.status = c->d_status;
    l.num_sms = c->num_sms;
    l.staged = 1;
    l.wins = reinterpret_cast<const gcz::WinDesc *>(d_windows);
    return lzma_run(c, c->sc, l, pick_stream(c, stream));
}

extern "C" int gcz_zstd_match_find_files(gcz_ctx *c, const uint8_t *const *srcs, const size_t *sizes, size_t count,
                                         uint32_t search_depth, gcz_zstd_sequence *seqs, size_t seq_capacity,
                                         uint64_t *window_offsets) {
    if (!c) return GCZ_EINVAL;
    if ((count && (!srcs || !sizes)) || !window_offsets) return fail(c, GCZ_EINVAL, "null pointer");
    const size_t nb = gcz_batch_num_windows(sizes, count);
    if (nb > 0xFFFFFFFFu) return fail(c, GCZ_EINVAL, "too many windows");
    std::vector<uint64_t> foff(count);
    std::vector<gcz_window> wins(nb);
    uint64_t slab = 0;
    gcz_batch_layout(sizes, count, foff.data(), wins.data(), &slab);
    window_offsets[0] = 0;
    if (nb == 0) return GCZ_OK;
    int r;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        Slot &sl = c->slots[0];
        if ((r = ensure_dev(c, sl.in, slab + 64)) != GCZ_OK) return r;
        if ((r = ensure_dev(c, sl.lz_has, nb * sizeof(gcz_window))) != GCZ_OK) return r;  // window table
        if ((r = ensure_dev(c, sl.offsets, (nb + 1) * 8)) != GCZ_OK) return r;
        size_t cap = 0;
        for (size_t i = 0; i < count; i++) cap += gcz_zstd_max_sequences(sizes[i]);
        if ((r = ensure_dev(c, sl.seqs, std::max<size_t>(cap, 1) * 16)) != GCZ_OK) return r;
        uint8_t *slab_p = static_cast<uint8_t *>(sl.in.p);
        for (size_t i = 0; i < count; i++)
            if (sizes[i]) GCZ_CUDA(c, cudaMemcpyAsync(slab_p + foff[i], srcs[i], sizes[i], cudaMemcpyHostToDevice, sl.st));
        GCZ_CUDA(c, cudaMemcpyAsync(sl.lz_has.p, wins.data(), nb * sizeof(gcz_window), cudaMemcpyHostToDevice, sl.st));
        if ((r = zstd_device_core(c, sl.sc, slab_p, slab, search_depth, sl.seqs.p, cap,
                                  static_cast<uint64_t *>(sl.offsets.p), sl.st,
                                  static_cast<const gcz::WinDesc *>(sl.lz_has.p), nb)) != GCZ_OK)
            return r;
        GCZ_CUDA(c, cudaMemcpyAsync(window_offsets, sl.offsets.p, (nb + 1) * 8, cudaMemcpyDeviceToHost, sl.st));
        GCZ_CUDA(c, cudaStreamSynchronize(sl.st));
        const uint64_t total = window_offsets[nb];
        if (total > seq_capacity)
            return fail(c, GCZ_ECAPACITY, "need %llu sequences, capacity %zu", (unsigned long long)total, seq_capacity);
        if (total) GCZ_CUDA(c, cudaMemcpyAsync(seqs, sl.seqs.p, total * 16, cudaMemcpyDeviceToHost, sl.st));
        GCZ_CUDA(c, cudaStreamSynchronize(sl.st));
        return read_status(c, sl.st);
    }
}

extern "C" int gcz_zstd_encode_frames_batch_device(gcz_ctx *c, const uint8_t *d_slab, uint64_t slab_bytes,
                                                   const gcz_window *d_windows, uint32_t num_windows,
                                                   const gcz_zstd_sequence *d_seqs, const uint64_t *d_seq_offsets,
                                                   uint8_t *d_out, size_t out_capacity, uint64_t *d_frame_offsets,
                                                   void *stream) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!d_frame_offsets || (num_windows && (!d_slab || !d_windows || !d_seqs || !d_seq_offsets || !d_out)))
        return fail(c, GCZ_EINVAL, "null pointer");
    if (!aligned16(d_slab)) return fail(c, GCZ_EINVAL, "d_slab must be 16-byte aligned");
    DeviceGuard g(c->device);
    cudaStream_t st = pick_stream(c, stream);
    if (num_windows == 0) {
        GCZ_CUDA(c, cudaMemsetAsync(d_frame_offsets, 0, 8, st));
        return GCZ_OK;
    }
    return zenc_core(c, c->sc, d_slab, slab_bytes, d_seqs, d_seq_offsets, d_out, out_capacity, d_frame_offsets, st,
                     reinterpret_cast<const gcz::WinDesc *>(d_windows), num_windows);
}

extern "C" int gcz_zstd_compress_files_gpu(gcz_ctx *c, const uint8_t *const *srcs, const size_t *sizes, size_t count,
                                           uint32_t level, uint8_t *out, size_t out_capacity, uint64_t *frame_sizes,
                                           size_t *out_size) {
    if (!c) return GCZ_EINVAL;
    if ((count && (!srcs || !sizes)) || !out_size) return fail(c, GCZ_EINVAL, "null pointer");
    *out_size = 0;
    const size_t nb = gcz_batch_num_windows(sizes, count);
    if (nb > 0xFFFFFFFFu) return fail(c, GCZ_EINVAL, "too many windows");
    if (nb && (!out || !frame_sizes)) return fail(c, GCZ_EINVAL, "null pointer");
    std::vector<uint64_t> foff(count);
    std::vector<gcz_window> wins(nb);
    uint64_t slab = 0;
    gcz_batch_layout(sizes, count, foff.data(), wins.data(), &slab);
    if (nb == 0) return GCZ_OK;
    const uint32_t depth = gcz_zstd_search_depth_for_level(level);
    int r;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    Slot &sl = c->slots[0];
    size_t cap = 0, fbound = 0;
    for (size_t i = 0; i < count; i++) {
        cap += gcz_zstd_max_sequences(sizes[i]);
        fbound += gcz_zstd_frames_bound(sizes[i]);
    }
    if ((r = ensure_dev(c, sl.in, slab + 64)) != GCZ_OK) return r;
    if ((r = ensure_dev(c, sl.lz_has, nb * sizeof(gcz_window))) != GCZ_OK) return r;  // window table
    if ((r = ensure_dev(c, sl.offsets, (nb + 1) * 8)) != GCZ_OK) return r;
    if ((r = ensure_dev(c, sl.seqs, std::max<size_t>(cap, 1) * 16)) != GCZ_OK) return r;
    if ((r = ensure_dev(c, sl.frames, fbound)) != GCZ_OK) return r;
    if ((r = ensure_dev(c, sl.foff, (nb + 1) * 8)) != GCZ_OK) return r;
    if ((r = ensure_host(c, sl.h_foff, (nb + 1) * 8)) != GCZ_OK) return r;
    uint8_t *slab_p = static_cast<uint8_t *>(sl.in.p);
    for (size_t i = 0; i < count; i++)
        if (sizes[i]) GCZ_CUDA(c, cudaMemcpyAsync(slab_p + foff[i], srcs[i], sizes[i], cudaMemcpyHostToDevice, sl.st));
    GCZ_CUDA(c, cudaMemcpyAsync(sl.lz_has.p, wins.data(), nb * sizeof(gcz_window), cudaMemcpyHostToDevice, sl.st));
    const gcz::WinDesc *dw = static_cast<const gcz::WinDesc *>(sl.lz_has.p);
    uint64_t *d_off = static_cast<uint64_t *>(sl.offsets.p);
    if ((r = zstd_device_core(c, sl.sc, slab_p, slab, depth, sl.seqs.p, cap, d_off, sl.st, dw, nb)) != GCZ_OK) return r;
    if ((r = zenc_core(c, sl.sc, slab_p, slab, sl.seqs.p, d_off, static_cast<uint8_t *>(sl.frames.p), fbound,
                       static_cast<uint64_t *>(sl.foff.p), sl.st, dw, nb)) != GCZ_OK)
        return r;
    GCZ_CUDA(c, cudaMemcpyAsync(sl.h_foff.p, sl.foff.p, (nb + 1) * 8, cudaMemcpyDeviceToHost, sl.st));
    GCZ_CUDA(c, cudaStreamSynchronize(sl.st));
    if ((r = read_status(c, sl.st)) != GCZ_OK) return r;
    const uint64_t *ho = static_cast<const uint64_t *>(sl.h_foff.p);
    const uint64_t total = ho[nb];
    if (total > out_capacity)
        return fail(c, GCZ_ECAPACITY, "frames need %llu bytes, capacity %zu", (unsigned long long)total, out_capacity);
    GCZ_CUDA(c, cudaMemcpyAsync(out, sl.frames.p, total, cudaMemcpyDeviceToHost, sl.st));
    for (size_t i = 0; i < nb; ++i) frame_sizes[i] = ho[i + 1] - ho[i];
    GCZ_CUDA(c, cudaStreamSynchronize(sl.st));
    *out_size = total;
    return GCZ_OK;
}

// =========================================================================== serving

namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device bytes per input byte of one slot, pre-sized at creation for a batch of
// max_batch_bytes of any mix of kinds: slab 1, candidates 2, Zstd speculative
// lists 3.9 (sized for the widest segment layout), packed sequences 2.67, ZSTD_Sequence output 5.33, LZMA2 packed
// matches 4, and for frames the frames 1.02, frame slots 1.02, offset codes
// 1.33 and plans 0.03.
constexpr double kDeviceBytesPerInputByte = 23.0;
constexpr int kMaxServerSlots = 8;

// Request groups, in window order inside a batch: every group's windows are one
// contiguous range of the batch's window table, so each runs as one launch.
enum { kGrpSeqLazy = 0, kGrpSeqGreedy, kGrpFramesLazy, kGrpFramesGreedy, kGrpLzma, kGroups };

struct ServerReq {
    uint64_t id = 0;
    int kind = 0;
    uint32_t depth = 0;
    const uint8_t *src = nullptr;
    size_t n = 0;
    void *out_a = nullptr;
    size_t cap_a = 0;
    void *out_b = nullptr;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int status = 1;  // 1 = pending; written under the server's mutex only (waiters read it there)
    int fail = 0;    // the worker's own note of this request's failure, published as status on completion
    int group = 0;
    uint32_t w0 = 0, nw = 0;
    uint64_t slab_off = 0;
    uint32_t selftest_iters = 0;  // > 0: a failure-detection probe (gcz_server_selftest_wait_timeout)
};

int req_group(const ServerReq *q) {
    const bool lazy = q->depth > 1;
    if (q->kind == GCZ_REQ_ZSTD) return lazy ? kGrpSeqLazy : kGrpSeqGreedy;
    if (q->kind == GCZ_REQ_ZSTD_FRAMES) return lazy ? kGrpFramesLazy : kGrpFramesGreedy;
    return kGrpLzma;
}

}  // namespace

namespace {
// One batch in flight: its stream, its own status words and every device
// buffer a max_batch_bytes batch of any mix of kinds needs, allocated once at
// creation (so serving never calls cudaMalloc or cudaFree).
struct ServerSlot {
    gcz_server *sv = nullptr;
    int index = 0;
    cudaStream_t st = nullptr;
    DevBuf in, wins, status, cand, seg, packed, counts, offsets, seqs, lz_packed, lz_has, frames, foff;
    DevBuf zslots, zovs, zaux, zplan;
    HostBuf h_off, h_foff, h_status;
    std::vector<gcz_window> hwins;
    std::vector<ServerReq *> reqs;
    uint32_t wb[kGroups + 1] = {};  // window bounds of the groups
    int phase = 0;                  // 0 free, 1 kernels and fixed-size copies queued, 2 result copies queued
    bool signaled = false;          // the queued phase has finished on the GPU (host callback)
    int err = GCZ_OK;
};
}  // namespace

struct gcz_server {
    gcz_ctx *c = nullptr;
    uint64_t max_batch_bytes = 0;
    uint32_t max_batch_requests = 0;
    uint64_t device_bytes = 0;
    int nslots = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<ServerReq *> pending;
    std::unordered_map<uint64_t, ServerReq *> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    ServerSlot slots[kMaxServerSlots];
    // Latencies of the most recent kLatWindow completed requests (a ring once
    // full), so that a long-running loop's memory and stats cost stay bounded.
    static constexpr size_t kLatWindow = size_t(1) << 20;
    std::vector<double> lat_ms;
    size_t lat_next = 0;
    uint64_t completed = 0, bytes_done = 0, batches = 0, max_in_flight = 0;
    int worker_error = GCZ_OK;
};

namespace {

// Runs on a CUDA callback thread when a slot's queued work has finished: only
// flags the slot and wakes the worker (no CUDA calls are allowed here).
void CUDART_CB slot_signal(void *p) {
    ServerSlot *s = static_cast<ServerSlot *>(p);
    {
        std::lock_guard<std::mutex> lk(s->sv->mu);
        s->signaled = true;
    }
    s->sv->cv_work.notify_one();
}

int slot_alloc(gcz_ctx *c, ServerSlot &s, uint64_t max_bytes) {
    const size_t W = max_bytes / kW;  // admission counts whole windows, so a batch has at most W
    int r;
    const size_t seq_cap = W * (size_t)kMaxSeqs;
    const size_t fbound = gcz_zstd_frames_bound(max_bytes);
    struct {
        DevBuf *b;
        size_t bytes;
    } dev[] = {{&s.in, max_bytes + 64},
               {&s.wins, W * sizeof(gcz_window) + 64},
               {&s.status, 256},
               {&s.cand, max_bytes * 2 + 64},
               {&s.seg, gcz::zstd2_seg_scratch_entries((uint32_t)W) * 8},
               {&s.packed, seq_cap * 8},
               {&s.counts, W * 4 + 64},
               {&s.offsets, (W + 1) * 8},
               {&s.seqs, seq_cap * 16},
               {&s.lz_packed, max_bytes * 4 + 64},
               {&s.lz_has, W + 64},
               {&s.frames, fbound},
               {&s.foff, (W + 1) * 8},
               {&s.zslots, W * (size_t)gcz::kZencSlot},
               {&s.zovs, W * (size_t)gcz::kZencMaxSeqs * 4},
               {&s.zaux, W * 12 + 64},
               {&s.zplan, W * ((size_t)gcz::kZencPlanBytes + 1024)}};
    for (auto &d : dev)
        if ((r = ensure_dev(c, *d.b, d.bytes)) != GCZ_OK) return r;
    if ((r = ensure_host(c, s.h_off, (W + 1) * 8)) != GCZ_OK) return r;
    if ((r = ensure_host(c, s.h_foff, (W + 1) * 8)) != GCZ_OK) return r;
    if ((r = ensure_host(c, s.h_status, 64)) != GCZ_OK) return r;
    return GCZ_OK;
}

void slot_release(ServerSlot &s) {
    for (DevBuf *b : {&s.in, &s.wins, &s.status, &s.cand, &s.seg, &s.packed, &s.counts, &s.offsets, &s.seqs,
                      &s.lz_packed, &s.lz_has, &s.frames, &s.foff, &s.zslots, &s.zovs, &s.zaux, &s.zplan})
        if (b->p) {
            cudaFree(b->p);
            b->p = nullptr;
            b->cap = 0;
        }
    for (HostBuf *b : {&s.h_off, &s.h_foff, &s.h_status})
        if (b->p) {
            cudaFreeHost(b->p);
            b->p = nullptr;
            b->cap = 0;
        }
    if (s.st) cudaStreamDestroy(s.st);
    s.st = nullptr;
}

// Enqueue one batch on its slot: the H2D of every request, the window table,
// one candidate sweep over all windows, then per group the second stage (Zstd
// parse, lazy and greedy; GPU frames; LZMA2 verification), the copies whose
// sizes are known already, the status words, and the signal.
int server_launch(gcz_server *sv, ServerSlot &s) {
    gcz_ctx *c = sv->c;
    std::stable_sort(s.reqs.begin(), s.reqs.end(),
                     [](const ServerReq *a, const ServerReq *b) { return a->group < b->group; });
    std::vector<size_t> sizes;
    for (ServerReq *r : s.reqs) sizes.push_back(r->n);
    std::vector<uint64_t> foff(sizes.size());
    const size_t nb = gcz_batch_num_windows(sizes.data(), sizes.size());
    s.hwins.resize(nb);
    uint64_t slab = 0;
    gcz_batch_layout(sizes.data(), sizes.size(), foff.data(), s.hwins.data(), &slab);
    uint32_t w = 0;
    for (int g = 0; g <= kGroups; g++) s.wb[g] = 0;
    for (size_t i = 0; i < s.reqs.size(); i++) {
        ServerReq *q = s.reqs[i];
        q->slab_off = foff[i];
        q->w0 = w;
        q->nw = (uint32_t)nwin(sizes[i]);
        w += q->nw;
        s.wb[q->group + 1] = w;
    }
    for (int g = 1; g <= kGroups; g++) s.wb[g] = std::max(s.wb[g], s.wb[g - 1]);
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    uint32_t *status = static_cast<uint32_t *>(s.status.p);
    uint8_t *slab_p = static_cast<uint8_t *>(s.in.p);
    const gcz::WinDesc *dw = static_cast<const gcz::WinDesc *>(s.wins.p);
    uint16_t *cand = static_cast<uint16_t *>(s.cand.p);
    GCZ_CUDA(c, cudaMemsetAsync(status, 0, 8, s.st));  // this batch's error bits start clear
    for (ServerReq *q : s.reqs)
        if (q->selftest_iters) {  // a bounded wait that runs out: the batch must report GCZ_EDEVICE
            selftest_wait_kernel<<<1, 32, 0, s.st>>>(status, q->selftest_iters);
            GCZ_CUDA(c, cudaGetLastError());
        }
    for (ServerReq *q : s.reqs)
        if (q->n) GCZ_CUDA(c, cudaMemcpyAsync(slab_p + q->slab_off, q->src, q->n, cudaMemcpyHostToDevice, s.st));
    if (nb) {
        GCZ_CUDA(c, cudaMemcpyAsync(s.wins.p, s.hwins.data(), nb * sizeof(gcz_window), cudaMemcpyHostToDevice, s.st));
        GCZ_CUDA(c, gcz::launch_cand_sweep(slab_p, slab, kW, (uint32_t)nb, cand, c->num_sms, s.st, dw, c->sweep_warps,
                                           c->sweep_groups, c->sweep_prefetch));
    }
    const uint32_t nz = s.wb[kGrpLzma];  // Zstd windows: sequences and frames groups
    uint64_t *d_off = static_cast<uint64_t *>(s.offsets.p);
    if (nz) {
        uint32_t *counts = static_cast<uint32_t *>(s.counts.p);
        for (int g = kGrpSeqLazy; g <= kGrpFramesGreedy; g++) {
            const uint32_t a = s.wb[g], b = s.wb[g + 1];
            if (a == b) continue;
            gcz::Zstd2Launch l{};
            l.src = slab_p;
            l.cand = cand;
            l.n = slab;
            l.window = kW;
            l.num_windows = b - a;
            l.search_depth = (g == kGrpSeqLazy || g == kGrpFramesLazy) ? 16u : 1u;
            l.max_seqs = kMaxSeqs;
            l.seg = s.seg.p;  // groups run one after another on this stream
            l.packed = static_cast<uint8_t *>(s.packed.p) + (size_t)a * kMaxSeqs * 8;
            l.seq_counts = counts + a;
            l.status = status;
            l.num_sms = c->num_sms;
            l.ctas_per_sm = c->parse_ctas;
            l.seg_width = (uint32_t)c->seg_width;
        l.seg_width = (uint32_t)c->seg_width;
            l.wins = dw + a;
            GCZ_CUDA(c, gcz::launch_zstd_parse(l, s.st));
        }
        GCZ_CUDA(c, gcz::launch_scan_counts(counts, nz, d_off, s.st));
        GCZ_CUDA(c, gcz::launch_expand_seqs(s.packed.p, counts, d_off, nz, kMaxSeqs, s.seqs.p,
                                            s.seqs.cap / 16, status, c->num_sms, s.st));
        if (s.wb[kGrpFramesLazy])  // offsets of the sequences groups
            GCZ_CUDA(c, cudaMemcpyAsync(s.h_off.p, d_off, (s.wb[kGrpFramesLazy] + 1) * 8, cudaMemcpyDeviceToHost,
                                        s.st));
    }
    const uint32_t f0 = s.wb[kGrpFramesLazy], nf = nz - f0;
    if (nf) {
        gcz::ZencLaunch l{};
        l.src = slab_p;
        l.n = slab;
        l.window = kW;
        l.num_windows = nf;
        l.seqs = s.seqs.p;
        l.seq_offsets = d_off + f0;
        l.slots = static_cast<uint8_t *>(s.zslots.p);
        l.ovs = static_cast<uint32_t *>(s.zovs.p);
        l.sec_off = static_cast<uint32_t *>(s.zaux.p);
        l.fsize = l.sec_off + nf;
        l.raw = reinterpret_cast<uint8_t *>(l.fsize + nf);
        l.plan = static_cast<uint8_t *>(s.zplan.p);
        l.hist = reinterpret_cast<uint32_t *>(l.plan + nf * (size_t)gcz::kZencPlanBytes);
        l.status = status;
        l.num_sms = c->num_sms;
        l.wins = dw + f0;
        uint64_t *d_foff = static_cast<uint64_t *>(s.foff.p);
        GCZ_CUDA(c, gcz::launch_zenc(l, s.st));
        GCZ_CUDA(c, gcz::launch_scan_counts(l.fsize, nf, d_foff, s.st));
        GCZ_CUDA(c, gcz::launch_zenc_compact(l, d_foff, static_cast<uint8_t *>(s.frames.p), s.frames.cap, s.st));
        GCZ_CUDA(c, cudaMemcpyAsync(s.h_foff.p, d_foff, (nf + 1) * 8, cudaMemcpyDeviceToHost, s.st));
    }
    const uint32_t l0 = s.wb[kGrpLzma], nl = (uint32_t)nb - l0;
    if (nl) {
        gcz::LzmaLaunch l{};
        l.src = slab_p;
        l.n = slab;
        l.window = kW;
        l.num_windows = nl;
        l.search_depth = GCZ_LZMA2_SEARCH_DEPTH;
        l.max_matches = GCZ_LZMA2_MAX_MATCHES;
        l.packed = static_cast<uint32_t *>(s.lz_packed.p);  // indexed by slab offset
        l.has_matches = static_cast<uint8_t *>(s.lz_has.p);  // indexed from this group's first window
        l.status = status;
        l.num_sms = c->num_sms;
        l.staged = 1;
        l.wins = dw + l0;
        l.ctas_per_sm = c->lzma_ctas;
        l.threads = c->lzma_threads;
        GCZ_CUDA(c, gcz::launch_lzma_verify(l, cand, s.st));
        for (ServerReq *q : s.reqs) {
            if (q->group != kGrpLzma || !q->n) continue;
            if (q->out_a)
                GCZ_CUDA(c, cudaMemcpyAsync(q->out_a, static_cast<uint32_t *>(s.lz_packed.p) + q->slab_off, q->n * 4,
                                            cudaMemcpyDeviceToHost, s.st));
            if (q->out_b)
                GCZ_CUDA(c, cudaMemcpyAsync(q->out_b, static_cast<uint8_t *>(s.lz_has.p) + (q->w0 - l0), q->nw,
                                            cudaMemcpyDeviceToHost, s.st));
        }
    }
    GCZ_CUDA(c, cudaMemcpyAsync(s.h_status.p, status, 8, cudaMemcpyDeviceToHost, s.st));
    GCZ_CUDA(c, cudaLaunchHostFunc(s.st, slot_signal, &s));
    return GCZ_OK;
}

// The batch's kernels are done: check its status, copy each Zstd request's
// sequences and each frames request's frames out (their sizes are known now)
// and queue the signal again, or, with nothing left to copy, complete it.
// Returns true when the slot's batch is complete.
bool server_results(gcz_server *sv, ServerSlot &s) {
    gcz_ctx *c = sv->c;
    const uint32_t h = static_cast<const uint32_t *>(s.h_status.p)[0];
    if (h & 2u) s.err = GCZ_ECAPACITY;
    else if (h & 4u) s.err = GCZ_EINVAL;
    else if (h) s.err = GCZ_EDEVICE;
    if (s.err != GCZ_OK) return true;
    DeviceGuard dg(c->device);
    bool queued = false;
    const uint64_t *ho = static_cast<const uint64_t *>(s.h_off.p);
    const uint64_t *hf = static_cast<const uint64_t *>(s.h_foff.p);
    const uint32_t f0 = s.wb[kGrpFramesLazy];
    for (ServerReq *q : s.reqs) {
        if (q->group == kGrpLzma) continue;
        const bool frames = q->group == kGrpFramesLazy || q->group == kGrpFramesGreedy;
        const uint64_t *o = frames ? hf + (q->w0 - f0) : ho + q->w0;
        const uint64_t a = o[0], e = o[q->nw];
        uint64_t *ob = static_cast<uint64_t *>(q->out_b);
        if (ob) {
            if (frames)
                for (uint32_t i = 0; i < q->nw; i++) ob[i] = o[i + 1] - o[i];
            else
                for (uint32_t i = 0; i <= q->nw; i++) ob[i] = o[i] - a;
        }
        if (e - a > q->cap_a) {
            q->fail = GCZ_ECAPACITY;
            continue;
        }
        if (e == a) continue;
        const cudaError_t ce =
            frames ? cudaMemcpyAsync(q->out_a, static_cast<uint8_t *>(s.frames.p) + a, e - a, cudaMemcpyDeviceToHost,
                                     s.st)
                   : cudaMemcpyAsync(q->out_a, static_cast<gcz_zstd_sequence *>(s.seqs.p) + a, (e - a) * 16,
                                     cudaMemcpyDeviceToHost, s.st);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            s.err = GCZ_ECUDA;
            break;
        }
        queued = true;
    }
    if (s.err != GCZ_OK) {
        cudaStreamSynchronize(s.st);  // copies already queued end before the requests go back
        cudaGetLastError();
        return true;
    }
    if (!queued) return true;
    if (cudaLaunchHostFunc(s.st, slot_signal, &s) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamSynchronize(s.st);
        cudaGetLastError();
    } else {
        return false;
    }
    return true;
}

// Complete a slot's requests with the batch status (or their own failure) and free the slot.
void server_complete(gcz_server *sv, ServerSlot &s) {
    const double t = now_ms();
    std::lock_guard<std::mutex> lk(sv->mu);
    for (ServerReq *q : s.reqs) {
        if (q->status == 1) q->status = q->fail != GCZ_OK ? q->fail : s.err;
        q->t_done = t;
        const double lat = q->t_done - q->t_submit;
        if (sv->lat_ms.size() < gcz_server::kLatWindow) {
            sv->lat_ms.push_back(lat);
        } else {
            sv->lat_ms[sv->lat_next] = lat;
            sv->lat_next = (sv->lat_next + 1) % gcz_server::kLatWindow;
        }
        sv->completed++;
        sv->bytes_done += q->n;
    }
    if (s.err != GCZ_OK) sv->worker_error = s.err;
    sv->batches++;
    s.reqs.clear();
    s.phase = 0;
    s.signaled = false;
    s.err = GCZ_OK;
    sv->cv_done.notify_all();
    sv->cv_work.notify_one();
}

// The worker: completes batches as their signals arrive and, whenever a slot
// is free and requests are pending, admits the oldest pending requests of any
// kind into a new batch and launches it at once, so up to nslots batches run
// on the GPU together.
void server_loop(gcz_server *sv) {
    for (;;) {
        std::vector<ServerSlot *> ready;
        ServerSlot *launch = nullptr;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            auto free_slot = [&]() -> ServerSlot * {
                for (int k = 0; k < sv->nslots; k++)
                    if (sv->slots[k].phase == 0) return &sv->slots[k];
                return nullptr;
            };
            auto in_flight = [&] {
                int n = 0;
                for (int k = 0; k < sv->nslots; k++) n += sv->slots[k].phase != 0;
                return n;
            };
            auto any_signal = [&] {
                for (int k = 0; k < sv->nslots; k++)
                    if (sv->slots[k].signaled) return true;
                return false;
            };
            sv->cv_work.wait(lk, [&] {
                return any_signal() || (!sv->pending.empty() && free_slot()) ||
                       (sv->stop && sv->pending.empty() && in_flight() == 0);
            });
            if (sv->stop && sv->pending.empty() && in_flight() == 0) break;
            for (int k = 0; k < sv->nslots; k++)
                if (sv->slots[k].signaled) {
                    sv->slots[k].signaled = false;
                    ready.push_back(&sv->slots[k]);
                }
            ServerSlot *fs = sv->pending.empty() ? nullptr : free_slot();
            if (fs) {
                // Requests are counted in whole 64 KiB windows, as they are
                // laid out in the slab, so a batch never needs more than the
                // slot's pre-sized buffers.  The oldest request always fits.
                uint64_t bytes = 0;
                const double t = now_ms();
                for (auto it = sv->pending.begin(); it != sv->pending.end();) {
                    ServerReq *q = *it;
                    const uint64_t padded = nwin(q->n) * (uint64_t)kW;
                    if (fs->reqs.empty() ||
                        (bytes + padded <= sv->max_batch_bytes && fs->reqs.size() < sv->max_batch_requests)) {
                        q->t_admit = t;
                        q->group = req_group(q);
                        bytes += padded;
                        fs->reqs.push_back(q);
                        it = sv->pending.erase(it);
                    } else {
                        ++it;
                    }
                }
                fs->phase = 1;
                fs->err = GCZ_OK;
                launch = fs;
                sv->max_in_flight = std::max<uint64_t>(sv->max_in_flight, (uint64_t)in_flight());
            }
        }
        for (ServerSlot *s : ready) {
            bool done = true;
            if (s->phase == 1) {
                s->phase = 2;
                done = server_results(sv, *s);
            }
            if (done) server_complete(sv, *s);
        }
        if (launch) {
            int r;
            try {
                r = server_launch(sv, *launch);
            } catch (const std::exception &) {  // host memory: never let it end the worker thread
                r = GCZ_ENOMEM;
            }
            if (r != GCZ_OK) {
                // Nothing signals a batch whose launch failed part-way: drain
                // what it did queue, then complete its requests with the status.
                DeviceGuard dg(sv->c->device);
                cudaStreamSynchronize(launch->st);
                cudaGetLastError();
                launch->err = r;
                server_complete(sv, *launch);
            }
        }
    }
}

}  // namespace

extern "C" int gcz_server_create(gcz_ctx *c, uint64_t hbm_budget, uint64_t max_batch_bytes,
                                 uint32_t max_batch_requests, gcz_server **out) {
    if (!c || !out) return GCZ_EINVAL;
    *out = nullptr;
    // Slot count and batch size from the budget: each slot holds ~23 device
    // bytes per input byte of a max-size batch.  With no batch size given, the
    // budget is split over four slots.
    const uint64_t per_byte_budget = (uint64_t)(hbm_budget / kDeviceBytesPerInputByte);
    if (max_batch_bytes == 0) max_batch_bytes = per_byte_budget / 4;
    max_batch_bytes = std::min<uint64_t>(max_batch_bytes, per_byte_budget) & ~uint64_t(kW - 1);
    if (max_batch_bytes < kW) return fail(c, GCZ_EINVAL, "HBM budget too small for one 64 KiB window per batch");
    const int nslots = (int)std::max<uint64_t>(1, std::min<uint64_t>(kMaxServerSlots, per_byte_budget / max_batch_bytes));
    gcz_server *sv = new (std::nothrow) gcz_server();
    if (!sv) return fail(c, GCZ_ENOMEM, "server allocation failed");
    sv->c = c;
    sv->max_batch_bytes = max_batch_bytes;
    sv->max_batch_requests = max_batch_requests ? max_batch_requests : 65536;
    sv->nslots = nslots;
    int r = GCZ_OK;
    {
        DeviceGuard g(c->device);
        for (int k = 0; k < nslots && r == GCZ_OK; k++) {
            ServerSlot &s = sv->slots[k];
            s.sv = sv;
            s.index = k;
            if (cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking) != cudaSuccess) {
                cudaGetLastError();
                r = fail(c, GCZ_ECUDA, "server stream creation failed");
                break;
            }
            r = slot_alloc(c, s, max_batch_bytes);
        }
        if (r != GCZ_OK) {
            for (int k = 0; k < nslots; k++) slot_release(sv->slots[k]);
            delete sv;
            return r;
        }
        for (int k = 0; k < nslots; k++)
            for (DevBuf *b : {&sv->slots[k].in, &sv->slots[k].wins, &sv->slots[k].status, &sv->slots[k].cand,
                              &sv->slots[k].seg, &sv->slots[k].packed, &sv->slots[k].counts, &sv->slots[k].offsets,
                              &sv->slots[k].seqs, &sv->slots[k].lz_packed, &sv->slots[k].lz_has,
                              &sv->slots[k].frames, &sv->slots[k].foff, &sv->slots[k].zslots, &sv->slots[k].zovs,
                              &sv->slots[k].zaux, &sv->slots[k].zplan})
                sv->device_bytes += b->cap;
    }
    try {
        sv->worker = std::thread(server_loop, sv);
    } catch (const std::exception &) {  // a thread limit: report it, never throw through the C ABI
        DeviceGuard g(c->device);
        for (int k = 0; k < nslots; k++) slot_release(sv->slots[k]);
        delete sv;
        return fail(c, GCZ_ENOMEM, "could not start the request loop's worker thread");
    }
    *out = sv;
    return GCZ_OK;
}

extern "C" void gcz_server_destroy(gcz_server *sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    {
        DeviceGuard g(sv->c->device);
        for (int k = 0; k < sv->nslots; k++) slot_release(sv->slots[k]);
    }
    for (auto &kv : sv->reqs) delete kv.second;
    delete sv;
}

extern "C" uint64_t gcz_server_max_batch_bytes(const gcz_server *sv) { return sv ? sv->max_batch_bytes : 0; }

extern "C" int gcz_server_info(const gcz_server *sv, uint32_t *slots, uint64_t *device_bytes) {
    if (!sv) return GCZ_EINVAL;
    if (slots) *slots = (uint32_t)sv->nslots;
    if (device_bytes) *device_bytes = sv->device_bytes;
    return GCZ_OK;
}

extern "C" int gcz_server_submit(gcz_server *sv, int kind, uint32_t search_depth, const uint8_t *src, size_t n,
                                 void *out_a, size_t cap_a, void *out_b, uint64_t *id) {
    if (!sv || !id || (kind != GCZ_REQ_ZSTD && kind != GCZ_REQ_LZMA2 && kind != GCZ_REQ_ZSTD_FRAMES) || (n && !src))
        return GCZ_EINVAL;
    if (kind == GCZ_REQ_ZSTD && (!out_b || (n && !out_a))) return GCZ_EINVAL;
    if (kind == GCZ_REQ_ZSTD_FRAMES && n && (!out_a || !out_b)) return GCZ_EINVAL;
    if (nwin(n) * (uint64_t)kW > sv->max_batch_bytes) return GCZ_ETOOLARGE;
    ServerReq *q = new (std::nothrow) ServerReq();
    if (!q) return GCZ_ENOMEM;
    q->kind = kind;
    q->depth = search_depth;
    q->src = src;
    q->n = n;
    q->out_a = out_a;
    q->cap_a = cap_a;
    q->out_b = out_b;
    q->t_submit = now_ms();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        q->id = sv->next_id++;
        try {
            sv->reqs[q->id] = q;
            sv->pending.push_back(q);
        } catch (const std::exception &) {  // out of host memory: not thrown through the C ABI
            sv->reqs.erase(q->id);
            delete q;
            return GCZ_ENOMEM;
        }
        *id = q->id;
    }
    sv->cv_work.notify_one();
    return GCZ_OK;
}

extern "C" int gcz_server_selftest_wait_timeout(gcz_server *sv, uint32_t max_iterations, uint64_t *id) {
    if (!sv || !id || max_iterations == 0) return GCZ_EINVAL;
    ServerReq *q = new (std::nothrow) ServerReq();
    if (!q) return GCZ_ENOMEM;
    q->kind = GCZ_REQ_LZMA2;  // no windows: it joins a batch like any request
    q->selftest_iters = max_iterations;
    q->t_submit = now_ms();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        q->id = sv->next_id++;
        try {
            sv->reqs[q->id] = q;
            sv->pending.push_back(q);
        } catch (const std::exception &) {
            sv->reqs.erase(q->id);
            delete q;
            return GCZ_ENOMEM;
        }
        *id = q->id;
    }
    sv->cv_work.notify_one();
    return GCZ_OK;
}

extern "C" int gcz_server_wait(gcz_server *sv, uint64_t id, double timeout_s, double *latency_ms) {
    if (!sv) return GCZ_EINVAL;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return GCZ_EINVAL;
    ServerReq *q = it->second;
    // wait_for releases the lock: submits from other threads may rehash the
    // map (so the id is looked up again, never the iterator kept), and another
    // waiter on the same id may take and free the request first (so q is read
    // only while its id is still present).
    auto gone = [&] { return sv->reqs.find(id) == sv->reqs.end(); };
    const bool ok =
        sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return gone() || q->status != 1; });
    if (gone()) return GCZ_EINVAL;
    if (!ok) return GCZ_ETIMEOUT;  // still queued or running: its buffers stay in use
    const int st = q->status;
    if (latency_ms) *latency_ms = q->t_done - q->t_submit;
    sv->reqs.erase(id);
    delete q;
    return st;
}

extern "C" int gcz_server_stats(gcz_server *sv, uint64_t *completed, uint64_t *bytes, uint64_t *batches,
                                double *p50_ms, double *p99_ms) {
    if (!sv) return GCZ_EINVAL;
    std::vector<double> v;
    int err;
    {
        std::lock_guard<std::mutex> lk(sv->mu);  // copy under the lock, sort outside it (the worker takes it too)
        v = sv->lat_ms;
        if (completed) *completed = sv->completed;
        if (bytes) *bytes = sv->bytes_done;
        if (batches) *batches = sv->batches;
        err = sv->worker_error;
    }
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) { return v.empty() ? 0.0 : v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))]; };
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    return err;
}

// =========================================================================== profiling

extern "C" int gcz_profile_start(gcz_ctx *c) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    c->prof = true;
    c->ev_used = 0;
    c->match_launches = 0;
    c->all_launches = 0;
    return GCZ_OK;
}

extern "C" int gcz_profile_stop(gcz_ctx *c, double *match_kernel_ms, uint64_t *match_kernel_launches,
                                uint64_t *all_kernel_launches) {
    if (!c) return GCZ_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    double total = 0.0;
    for (size_t i = 0; i < c->ev_used; i++) {
        GCZ_CUDA(c, cudaEventSynchronize(c->events[i].b));
        float ms = 0.f;
        GCZ_CUDA(c, cudaEventElapsedTime(&ms, c->events[i].a, c->events[i].b));
        total += ms;
    }
    if (match_kernel_ms) *match_kernel_ms = total;
    if (match_kernel_launches) *match_kernel_launches = c->match_launches;
    if (all_kernel_launches) *all_kernel_launches = c->all_launches;
    c->prof = false;
    c->ev_used = 0;
    return GCZ_OK;
}
