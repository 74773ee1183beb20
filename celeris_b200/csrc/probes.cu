// Throughput probes: measured peaks of the pipes the far-field kernels are
// bound by (MUFU transcendentals, FP32 FMA, FP64 FMA) on the current device.
// Used by bench.py for the roofline denominators; not part of any result path.
#include <cuda_runtime.h>

#include "runtime.cuh"

namespace {

constexpr int kChains = 8;

__global__ void probe_mufu(float seed, int iters, float* sink) {
    float v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = seed + 0.001f * (threadIdx.x + c);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            float y;
            asm volatile("sin.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(v[c]));
            v[c] = y;
        }
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += v[c];
    if (s == 12345.678f) sink[0] = s;
}

__global__ void probe_ffma(float a, int iters, float* sink) {
    float v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = a + threadIdx.x * 1e-3f + c;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) v[c] = fmaf(v[c], 0.9999f, 1e-4f);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += v[c];
    if (s == 12345.678f) sink[0] = s;
}

__global__ void probe_dfma(double a, int iters, double* sink) {
    double v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = a + threadIdx.x * 1e-3 + c;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) v[c] = fma(v[c], 0.9999, 1e-4);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += v[c];
    if (s == 12345.678) sink[0] = s;
}

// FP64 tensor cores: kChains independent m8n8k4 accumulators per warp.
__global__ void probe_dmma(double a, int iters, double* sink) {
    const int lane = threadIdx.x & 31;
    double c0[kChains], c1[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) c0[c] = c1[c] = 0.001 * (lane + c);
    const double x = a + 1e-3 * lane, y = 0.999;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                         : "+d"(c0[c]), "+d"(c1[c])
                         : "d"(x), "d"(y));
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += c0[c] + c1[c];
    if (s == 12345.678) sink[0] = s;
}

// Accuracy of sin.approx / cos.approx against FP64 sin/cos of the same FP32
// argument, for arguments uniform in [-xmax, xmax]: max |error| and the mean
// signed error (bias) of each.
__global__ void probe_sincos_err(float xmax, int npts, double* acc) {
    double ms = 0.0, mc = 0.0, bs = 0.0, bc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += gridDim.x * blockDim.x) {
        const float x = xmax * (2.0f * ((float)i + 0.5f) / (float)npts - 1.0f);
        float s, c;
        asm("sin.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(x));
        asm("cos.approx.ftz.f32 %0, %1;" : "=f"(c) : "f"(x));
        const double es = (double)s - sin((double)x), ec = (double)c - cos((double)x);
        ms = fmax(ms, fabs(es));
        mc = fmax(mc, fabs(ec));
        bs += es;
        bc += ec;
    }
    atomicMax(reinterpret_cast<unsigned long long*>(acc + 0), (unsigned long long)__double_as_longlong(ms));
    atomicMax(reinterpret_cast<unsigned long long*>(acc + 1), (unsigned long long)__double_as_longlong(mc));
    atomicAdd(acc + 2, bs);
    atomicAdd(acc + 3, bc);
}

template <typename F>
int time_probe(F launch, double ops, double* out_per_s) {
    cudaEvent_t a, b;
    CEL_CUDA(cudaEventCreate(&a));
    CEL_CUDA(cudaEventCreate(&b));
    launch();  // warm-up
    CEL_CUDA(cudaEventRecord(a));
    launch();
    CEL_CUDA(cudaEventRecord(b));
    CEL_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    CEL_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *out_per_s = ops / (ms * 1e-3);
    return CELERIS_OK;
}

}  // namespace

// New: accuracy of the MUFU sine/cosine on [-xmax, xmax] (npts samples):
// out = {max |sin err|, max |cos err|, mean sin err, mean cos err}.
extern "C" int celeris_probe_sincos(double xmax, int npts, double* out) {
    CEL_TRY(celeris_rt::require_device());
    if (!out || npts <= 0) return celeris_rt::set_error(CELERIS_ERR_INVALID_ARG, "bad arguments");
    double* d = nullptr;
    CEL_CUDA(cudaMalloc(&d, 4 * sizeof(double)));
    CEL_CUDA(cudaMemset(d, 0, 4 * sizeof(double)));
    probe_sincos_err<<<592, 256>>>((float)xmax, npts, d);
    celeris_rt::count_launch(1);
    double h[4];
    CEL_CUDA(cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost));
    cudaFree(d);
    out[0] = h[0];
    out[1] = h[1];
    out[2] = h[2] / npts;
    out[3] = h[3] / npts;
    return CELERIS_OK;
}

// New: FP64 FMA/s of the tensor cores (mma.sync m8n8k4 f64, 256 FMA per warp op).
extern "C" int celeris_probe_dmma(double* fma_per_s) {
    CEL_TRY(celeris_rt::require_device());
    if (!fma_per_s) return celeris_rt::set_error(CELERIS_ERR_INVALID_ARG, "null output");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void* sink = nullptr;
    CEL_CUDA(cudaMalloc(&sink, 64));
    const int blocks = sms * 8, threads = 256, iters = 2048;
    const double fmas = (double)blocks * (threads / 32) * kChains * iters * 256.0;
    CEL_TRY(time_probe([&] { probe_dmma<<<blocks, threads>>>(0.5, iters, (double*)sink); }, fmas, fma_per_s));
    celeris_rt::count_launch(2);
    cudaFree(sink);
    CEL_CUDA(cudaGetLastError());
    return CELERIS_OK;
}

// New: measured op rates: MUFU sin.approx results/s, FP32 FMA/s, FP64 FMA/s.
extern "C" int celeris_probe_peaks(double* mufu_per_s, double* ffma_per_s, double* dfma_per_s) {
    CEL_TRY(celeris_rt::require_device());
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void* sink = nullptr;
    CEL_CUDA(cudaMalloc(&sink, 64));
    const int blocks = sms * 8, threads = 256;
    const int it_m = 4096, it_f = 16384, it_d = 4096;
    const double thr = (double)blocks * threads * kChains;
    CEL_TRY(time_probe([&] { probe_mufu<<<blocks, threads>>>(0.5f, it_m, (float*)sink); }, thr * it_m, mufu_per_s));
    CEL_TRY(time_probe([&] { probe_ffma<<<blocks, threads>>>(0.5f, it_f, (float*)sink); }, thr * it_f, ffma_per_s));
    CEL_TRY(time_probe([&] { probe_dfma<<<blocks, threads>>>(0.5, it_d, (double*)sink); }, thr * it_d, dfma_per_s));
    celeris_rt::count_launch(6);
    cudaFree(sink);
    CEL_CUDA(cudaGetLastError());
    return CELERIS_OK;
}
