// Device-side building blocks shared by the Zstd and LZMA2 match finders.
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

namespace gcz {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kHashLog = 14;              // HASH_LOG, zstd_compress.cu:26 / lzma2_match_find.cu:18
constexpr uint32_t kHashSize = 1u << kHashLog;
constexpr uint32_t kMaxWindow = 65536;         // table entries are u16 positions
constexpr uint32_t kWinPad = 32;               // zeroed bytes kept after a staged window

// Device error codes written to the context's status word.
constexpr uint32_t kErrTmaTimeout = 1;
constexpr uint32_t kErrCapacity = 2;

// Multiplicative 4-byte hash, HASH4 in zstd_compress.cu:228 and lzma2_match_find.cu:92.
__device__ __forceinline__ uint32_t hash4(uint32_t v) { return (v * 2654435761u) >> (32 - kHashLog); }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}
__device__ __forceinline__ uint32_t lanemask_gt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_gt;" : "=r"(m));
    return m;
}
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------------------
// Window byte sources.  Both expose word(i) (the i-th aligned little-endian
// 32-bit word of the window) and u32(q) (the 4 bytes starting at q).  Bytes
// at or past the window size are unspecified; callers bound every comparison
// by the size, exactly like the reference loops.
// ---------------------------------------------------------------------------

// Window staged in shared memory with kWinPad zero bytes after it.
struct SmemWin {
    const uint32_t *w;
    __device__ __forceinline__ uint32_t word(uint32_t i) const { return w[i]; }
    __device__ __forceinline__ uint32_t u32(uint32_t q) const {
        const uint32_t i = q >> 2;
        return __funnelshift_r(w[i], w[i + 1], (q & 3u) * 8u);
    }
    __device__ __forceinline__ uint32_t byte(uint32_t q) const {
        return reinterpret_cast<const uint8_t *>(w)[q];
    }
    // The 8 bytes at q: three aligned words, two funnel shifts.
    __device__ __forceinline__ void u64(uint32_t q, uint32_t &lo, uint32_t &hi) const {
        const uint32_t i = q >> 2, sh = (q & 3u) * 8u;
        const uint32_t w1 = w[i + 1];
        lo = __funnelshift_r(w[i], w1, sh);
        hi = __funnelshift_r(w1, w[i + 2], sh);
    }
};

// Window read in place from global memory (16-byte aligned start).  Only
// aligned words whose first byte lies inside the window are loaded, so a read
// never leaves the 16-byte block of a valid byte.
struct GlobalWin {
    const uint32_t *w;
    uint32_t nwords;  // ceil(size / 4)
    __device__ __forceinline__ uint32_t word(uint32_t i) const { return i < nwords ? __ldg(w + i) : 0u; }
    __device__ __forceinline__ uint32_t u32(uint32_t q) const {
        const uint32_t i = q >> 2, s = q & 3u;
        const uint32_t lo = word(i);
        return s ? __funnelshift_r(lo, word(i + 1), s * 8u) : lo;
    }
    __device__ __forceinline__ uint32_t byte(uint32_t q) const {
        return (word(q >> 2) >> ((q & 3u) * 8u)) & 0xFFu;
    }
};

// One bit per device: the kernel's shared-memory limit is set there.  Atomic,
// because contexts on different host threads launch concurrently.
using SmemOnce = std::atomic<unsigned long long>;

// Sets a kernel's dynamic shared-memory limit once per device (host side), so
// that later launches -- including ones being captured into a CUDA graph --
// make no attribute calls.  (Devices 64 and up set it on every launch.)
template <class Kernel>
inline cudaError_t set_smem_once(Kernel k, uint32_t bytes, SmemOnce &done_mask) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done_mask.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e == cudaSuccess && bit) done_mask.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// ---------------------------------------------------------------------------
// mbarrier + 1-D bulk copy (TMA, no tensor map, no multicast).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// dst (smem) and src (global) 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// Bounded wait on an mbarrier phase: true when the phase completed, false when
// the iteration limit ran out (each try_wait already suspends for a while).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t max_iter = (1u << 24)) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < max_iter; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Stage window bytes [0, size) of `src` into shared memory `dst` followed by
// kWinPad zero bytes.  Called by every lane of one warp; lane 0 issues the
// bulk copies.  Returns false (after recording an error) if the copy did not
// complete within the bounded wait.
__device__ __forceinline__ bool stage_window(uint8_t *dst, const uint8_t *src, uint32_t size, uint64_t *bar,
                                             uint32_t &parity, uint32_t *status) {
    const uint32_t lane = lane_id();
    const uint32_t bulk = size & ~15u;
    __syncwarp();
    fence_proxy_async_smem();  // earlier generic reads of dst precede the async-proxy writes
    if (bulk) {
        if (lane == 0) {
            mbar_arrive_expect_tx(bar, bulk);
            constexpr uint32_t kPiece = 16384;
            for (uint32_t off = 0; off < bulk; off += kPiece) {
                const uint32_t b = bulk - off < kPiece ? bulk - off : kPiece;
                bulk_g2s(dst + off, src + off, b, bar);
            }
        }
    }
    // Tail bytes (< 16) with plain loads, then zero padding; disjoint from the bulk range.
    for (uint32_t i = bulk + lane; i < bulk + 16 + kWinPad; i += 32) dst[i] = i < size ? src[i] : 0;
    bool ok = true;
    if (bulk) {
        ok = mbar_wait(bar, parity);
        parity ^= 1u;
        if (!ok && lane == 0) atomicOr(status, kErrTmaTimeout);
    }
    __syncwarp();
    return ok;
}

}  // namespace gcz
