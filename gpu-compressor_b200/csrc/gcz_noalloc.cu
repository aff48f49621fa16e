// gcz_zstd_match_find_device_noalloc: the Zstd match-find step without any
// device allocation, for callers that cannot allocate device memory when they
// call in -- a process whose device memory is already carved up by another
// allocator (a serving engine's or a framework's reserved pool, where one more
// cudaMalloc can fail or fragment it), a latency-bound loop where cudaMalloc /
// cudaFree would stall it (cudaFree synchronises the whole device), or code
// that cannot hold a gcz_ctx at all, since gcz_create itself allocates.
//
// The step's scratch (packed sequences at a per-window stride, per-window
// counts, a status word) lives in the file-scope array below instead.  Every
// GPU that loads this library holds that array until the process exits.  All
// calls on a device share it and it keeps the last call's contents, so two
// calls that overlap on the GPU race; the status word, the only thing that must
// start at zero, is cleared at the start of every call.
#include <mutex>

#include "gcz.h"
#include "gcz_kernels.h"

namespace {

constexpr uint32_t kNaMaxWindows = GCZ_NOALLOC_MAX_INPUT / GCZ_WINDOW;  // 128
constexpr size_t kNaPackedBytes = (size_t)kNaMaxWindows * GCZ_ZSTD_MAX_SEQ_PER_WINDOW * 8;
constexpr size_t kNaCountsOff = kNaPackedBytes;                      // 256-byte aligned
constexpr size_t kNaStatusOff = kNaCountsOff + kNaMaxWindows * 4;    // 256-byte aligned
constexpr size_t kNaScratchBytes = kNaStatusOff + 256;
static_assert(kNaPackedBytes % 256 == 0 && kNaStatusOff % 256 == 0, "scratch sections must stay aligned");

constexpr int kNaMaxDevices = 64;

struct NaDevice {
    unsigned char *scratch = nullptr;  // device address of g_zstd_noalloc_scratch on this device
    int num_sms = 0;
};

std::mutex g_na_mu;
NaDevice g_na_dev[kNaMaxDevices];

}  // namespace

// ~21.3 MiB per GPU: room for GCZ_NOALLOC_MAX_INPUT bytes of input.
static __device__ __align__(256) unsigned char g_zstd_noalloc_scratch[kNaScratchBytes];

namespace {

// Once per device, with that device current: resolve the array's device
// address (the host-side name is only a stand-in) and the SM count.
int na_setup(int device, NaDevice *out) {
    std::lock_guard<std::mutex> lk(g_na_mu);
    NaDevice &d = g_na_dev[device];
    if (!d.scratch) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_zstd_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return GCZ_ECUDA;
        }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess || sms <= 0) {
            cudaGetLastError();
            return GCZ_ECUDA;
        }
        d.num_sms = sms;
        d.scratch = static_cast<unsigned char *>(p);
    }
    *out = d;
    return GCZ_OK;
}

int na_run(int device, const uint8_t *d_src, size_t n, uint32_t search_depth, gcz_zstd_sequence *d_seqs,
           size_t seq_capacity, uint64_t *d_offsets, cudaStream_t st) {
    NaDevice d;
    int r = na_setup(device, &d);
    if (r != GCZ_OK) return r;
    if (n == 0) {
        if (cudaMemsetAsync(d_offsets, 0, 8, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
            return GCZ_ECUDA;
        return GCZ_OK;
    }
    const uint32_t nb = (uint32_t)((n + GCZ_WINDOW - 1) / GCZ_WINDOW);
    uint32_t *counts = reinterpret_cast<uint32_t *>(d.scratch + kNaCountsOff);
    uint32_t *status = reinterpret_cast<uint32_t *>(d.scratch + kNaStatusOff);
    if (cudaMemsetAsync(status, 0, 4, st) != cudaSuccess) return GCZ_ECUDA;
    gcz::ZstdLaunch l{};
    l.src = d_src;
    l.n = n;
    l.window = GCZ_WINDOW;
    l.num_windows = nb;
    l.search_depth = search_depth;
    l.max_seqs = GCZ_ZSTD_MAX_SEQ_PER_WINDOW;
    l.packed = d.scratch;
    l.seq_counts = counts;
    l.status = status;
    l.num_sms = d.num_sms;
    l.staged = 1;
    if (gcz::launch_zstd_match(l, st) != cudaSuccess ||
        gcz::launch_scan_counts(counts, nb, d_offsets, st) != cudaSuccess ||
        gcz::launch_expand_seqs(d.scratch, counts, d_offsets, nb, GCZ_ZSTD_MAX_SEQ_PER_WINDOW, d_seqs, seq_capacity,
                                status, d.num_sms, st) != cudaSuccess)
        return GCZ_ECUDA;
    uint32_t h = 0;
    if (cudaMemcpyAsync(&h, status, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return GCZ_ECUDA;
    if (h & 2u) return GCZ_ECAPACITY;
    if (h) return GCZ_EDEVICE;
    return GCZ_OK;
}

}  // namespace

extern "C" int gcz_zstd_match_find_device_noalloc(int device, const uint8_t *d_src, size_t n, uint32_t search_depth,
                                                  gcz_zstd_sequence *d_seqs, size_t seq_capacity, uint64_t *d_offsets,
                                                  void *stream) {
    if (n > GCZ_NOALLOC_MAX_INPUT) return GCZ_ETOOLARGE;
    if (!d_offsets || (n && (!d_src || !d_seqs))) return GCZ_EINVAL;
    if (reinterpret_cast<uintptr_t>(d_src) & 15u) return GCZ_EINVAL;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return GCZ_ECUDA;
    }
    if (device < 0 || device >= count || device >= kNaMaxDevices) return GCZ_EINVAL;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != device && cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return GCZ_ECUDA;
    }
    const int r = na_run(device, d_src, n, search_depth, d_seqs, seq_capacity, d_offsets,
                         static_cast<cudaStream_t>(stream));
    if (r == GCZ_ECUDA) cudaGetLastError();
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    return r;
}
