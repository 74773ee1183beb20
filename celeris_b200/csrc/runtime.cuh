// Runtime support shared by the CELERIS B200 translation units: status/error
// reporting, a per-(device, stream) workspace arena, pinned host staging, the
// launch counter, and the TMA-bulk / mbarrier helpers used by the tiled kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdarg>
#include <cstddef>
#include <string>

#include "../../include/celeris_b200.h"

namespace celeris_rt {

// ---- status / error text --------------------------------------------------
int set_error(int status, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* where);
#define CEL_CUDA(call)                                              \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return celeris_rt::cuda_error(_e, #call); \
    } while (0)
#define CEL_TRY(call)                 \
    do {                              \
        int _s = (call);              \
        if (_s != CELERIS_OK) return _s; \
    } while (0)

// Returns CELERIS_OK when a CUDA device is present (and selects nothing).
int require_device();

// cudaMalloc for every device buffer the library owns (workspace arenas, I/O
// buffers). Fails with CELERIS_ERR_OOM when cudaMalloc fails, and also - for
// failure-path tests - while an injected-failure count is pending
// (celeris_debug_fail_alloc, or the environment variable
// CELERIS_DEBUG_FAIL_ALLOC=<count> read when the library loads): each such call
// consumes one count and allocates nothing.
int device_alloc(void** p, size_t bytes, const char* what);

// ---- launch accounting ----------------------------------------------------
// Kernels launched while the calling thread captures a CUDA graph are not
// counted (set_launch_counting(false)); a graph launch counts its kernels.
void count_launch(uint64_t n = 1);
void set_launch_counting(bool on);

// ---- workspace -------------------------------------------------------------
// A bump allocator over one device buffer that belongs to (current device,
// stream). It only grows; growing synchronizes the stream before the old buffer
// is freed. Calls on the same stream are ordered by the stream, so reusing the
// buffer across calls is safe; different streams get different arenas.
class Workspace {
public:
    // Reserve `bytes` (256-byte aligned chunks) and return device pointers via
    // take(). reserve() must be called with the TOTAL needed before take().
    int reserve(cudaStream_t stream, size_t bytes);
    void* take(size_t bytes);
    void* base() const { return base_; }
    size_t capacity() const { return cap_; }

    static Workspace& for_stream(cudaStream_t stream);
    static void release_all();
    // Free the arenas that belong to `stream` (on any device); the stream must
    // be idle.
    static void release_stream(cudaStream_t stream);

private:
    void* base_ = nullptr;
    size_t cap_ = 0;
    size_t off_ = 0;
};

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// A non-blocking stream owned by the calling thread (declare it thread_local):
// created on first use for the current device and replaced when the device
// changes. When it is replaced, and when the thread exits, the stream is
// synchronized, its workspace arenas are freed and it is destroyed.
class ThreadStream {
public:
    int get(cudaStream_t* out);
    ~ThreadStream() { drop(); }

private:
    void drop();
    cudaStream_t s_ = nullptr;
    int dev_ = -1;
};

// Pinned host staging for the synchronous host-buffer entry points (one per
// calling thread; grows).
void* pinned_staging(size_t bytes);

}  // namespace celeris_rt

// ---- device helpers: bulk async copies with mbarrier completion ------------
// These wrap the sm_90+/sm_100 PTX forms directly. Every wait is bounded: after
// kSpinLimit polls the wait gives up and reports failure to the caller, which
// records CELERIS_ERR_DEVICE_TIMEOUT and leaves the kernel.
namespace celeris_dev {

constexpr uint32_t kSpinLimit = 1u << 26;

// Accuracy model of the MUFU approximations in the precision-form far-field
// terms; the error bound that form states rests on these two figures:
//   kSinCosAbsErr  max |sin.approx.ftz.f32(x) - sin(x)| (and the same for cos)
//                  over every FP32 x in [-pi_f, pi_f], pi_f = 3.14159274f (the
//                  kernel's reduced phase range)
//   kRsqrtRelErr   max |rsqrt.approx.ftz.f32(x) sqrt(x) - 1| over every normal
//                  FP32 x in [2^-10, 2^30)
// celeris_probe_mufu_accuracy measures both exhaustively on the current device
// against FP64 sin / cos / sqrt, and the GPU tests check the measurement stays
// within these figures.
constexpr double kSinCosAbsErr = 6.8e-7;
constexpr double kRsqrtRelErr = 1.3e-7;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
        "r"(bytes)
        : "memory");
}

// 1D bulk copy global -> shared, completion counted on `bar` (transaction bytes).
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Bounded parity wait. Returns true when the phase with parity `parity`
// completed, false when the poll budget (`limit` polls) ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kSpinLimit) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Arrive once on `bar` (no transaction bytes).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar))
                 : "memory");
}

}  // namespace celeris_dev
