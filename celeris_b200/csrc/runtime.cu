// Runtime support: status text, device queries, workspace arenas, pinned
// staging and the launch counter (declared in runtime.cuh).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include "runtime.cuh"

namespace celeris_rt {
namespace {
thread_local std::string t_last_error;
std::atomic<uint64_t> g_launches{0};

std::mutex g_ws_mu;
std::map<std::pair<int, cudaStream_t>, Workspace*>& ws_map() {
    static auto* m = new std::map<std::pair<int, cudaStream_t>, Workspace*>();
    return *m;
}

struct Pinned {
    void* p = nullptr;
    size_t cap = 0;
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};
thread_local Pinned t_pinned;
}  // namespace

int set_error(int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return status;
}

int cuda_error(cudaError_t e, const char* where) {
    if (e == cudaErrorMemoryAllocation)
        return set_error(CELERIS_ERR_OOM, "%s: %s", where, cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return set_error(CELERIS_ERR_NO_DEVICE, "%s: %s", where, cudaGetErrorString(e));
    return set_error(CELERIS_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

int require_device() {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();  // clear the sticky-free error state of the query
        return set_error(CELERIS_ERR_NO_DEVICE, "no CUDA device available (%s)",
                         e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
    }
    return CELERIS_OK;
}

namespace {
// Pending injected allocation failures (failure-path tests only).
std::atomic<int> g_fail_alloc{[] {
    const char* v = std::getenv("CELERIS_DEBUG_FAIL_ALLOC");
    return v ? std::atoi(v) : 0;
}()};
}  // namespace

// Consumes one pending injected failure; true if there was one.
bool take_injected_failure() {
    int pending = g_fail_alloc.load();
    while (pending > 0)
        if (g_fail_alloc.compare_exchange_weak(pending, pending - 1)) return true;
    return false;
}

int device_alloc(void** p, size_t bytes, const char* what) {
    *p = nullptr;
    if (take_injected_failure())
        return set_error(CELERIS_ERR_OOM, "%s: cudaMalloc(%zu) failed (injected failure)", what, bytes);
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return set_error(CELERIS_ERR_OOM, "%s: cudaMalloc(%zu) failed: %s", what, bytes, cudaGetErrorString(e));
    }
    return CELERIS_OK;
}

thread_local bool t_counting = true;

void count_launch(uint64_t n) {
    if (t_counting) g_launches.fetch_add(n, std::memory_order_relaxed);
}

void set_launch_counting(bool on) { t_counting = on; }

int Workspace::reserve(cudaStream_t stream, size_t bytes) {
    off_ = 0;
    if (bytes <= cap_) return CELERIS_OK;
    if (base_) {
        CEL_CUDA(cudaStreamSynchronize(stream));
        CEL_CUDA(cudaFree(base_));
        base_ = nullptr;
        cap_ = 0;
    }
    if (take_injected_failure())
        return set_error(CELERIS_ERR_OOM, "workspace: cudaMalloc(%zu) failed (injected failure)", bytes);
    size_t want = align256(bytes + bytes / 4);
    cudaError_t e = cudaMalloc(&base_, want);
    if (e != cudaSuccess) {
        base_ = nullptr;
        cudaGetLastError();
        // retry with the exact size before giving up
        want = align256(bytes);
        e = cudaMalloc(&base_, want);
        if (e != cudaSuccess) {
            base_ = nullptr;
            cudaGetLastError();
            return set_error(CELERIS_ERR_OOM, "workspace: cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
        }
    }
    cap_ = want;
    return CELERIS_OK;
}

void* Workspace::take(size_t bytes) {
    char* p = static_cast<char*>(base_) + off_;
    off_ += align256(bytes);
    return p;
}

Workspace& Workspace::for_stream(cudaStream_t stream) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_ws_mu);
    auto& m = ws_map();
    auto key = std::make_pair(dev, stream);
    auto it = m.find(key);
    if (it == m.end()) it = m.emplace(key, new Workspace()).first;
    return *it->second;
}

void Workspace::release_stream(cudaStream_t stream) {
    std::lock_guard<std::mutex> lk(g_ws_mu);
    auto& m = ws_map();
    for (auto it = m.begin(); it != m.end();) {
        if (it->first.second != stream) {
            ++it;
            continue;
        }
        if (it->second->base_) {
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(it->first.first);
            cudaFree(it->second->base_);
            cudaSetDevice(cur);
        }
        delete it->second;
        it = m.erase(it);
    }
}

int ThreadStream::get(cudaStream_t* out) {
    int cur = 0;
    CEL_CUDA(cudaGetDevice(&cur));
    if (!s_ || dev_ != cur) {
        drop();
        CEL_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
        dev_ = cur;
    }
    *out = s_;
    return CELERIS_OK;
}

void ThreadStream::drop() {
    if (!s_) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(dev_);
    cudaStreamSynchronize(s_);
    Workspace::release_stream(s_);
    cudaStreamDestroy(s_);
    cudaSetDevice(cur);
    cudaGetLastError();  // a failure here (e.g. the runtime shutting down) is nobody's call's error
    s_ = nullptr;
    dev_ = -1;
}

void Workspace::release_all() {
    std::lock_guard<std::mutex> lk(g_ws_mu);
    for (auto& kv : ws_map()) {
        if (kv.second->base_) {
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(kv.first.first);
            cudaDeviceSynchronize();
            cudaFree(kv.second->base_);
            cudaSetDevice(cur);
        }
        delete kv.second;
    }
    ws_map().clear();
}

void* pinned_staging(size_t bytes) {
    if (bytes <= t_pinned.cap) return t_pinned.p;
    if (t_pinned.p) cudaFreeHost(t_pinned.p);
    t_pinned.p = nullptr;
    t_pinned.cap = 0;
    size_t want = align256(bytes + bytes / 4);
    if (cudaHostAlloc(&t_pinned.p, want, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        t_pinned.p = nullptr;
        return nullptr;
    }
    t_pinned.cap = want;
    return t_pinned.p;
}

}  // namespace celeris_rt

extern "C" {

int celeris_available(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count > 0 ? 1 : 0;
}

const char* celeris_device_name(void) {
    static char name[256] = {0};
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return "";
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "";
    std::strncpy(name, prop.name, sizeof(name) - 1);
    return name;
}

const char* celeris_last_error(void) { return celeris_rt::t_last_error.c_str(); }

int celeris_abi_version(void) { return 10000; }

uint64_t celeris_launch_count(void) { return celeris_rt::g_launches.load(); }

int celeris_release_workspace(void) {
    celeris_rt::Workspace::release_all();
    return CELERIS_OK;
}

int celeris_debug_fail_alloc(int count) {
    if (count < 0) return celeris_rt::set_error(CELERIS_ERR_INVALID_ARG, "count < 0");
    celeris_rt::g_fail_alloc.store(count);
    return CELERIS_OK;
}

}  // extern "C"
