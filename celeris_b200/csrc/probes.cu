// Probes of the current device: measured peaks of the pipes the far-field and
// RCWA kernels are bound by (MUFU transcendentals, FP32 FMA, FP64 FMA, FP64
// tensor cores; bench.py's roofline denominators) and the measured accuracy of
// the MUFU approximations the precision form's stated error bound relies on.
// Not part of any result path.
#include <cuda_runtime.h>

#include <cstring>

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

// Exhaustive accuracy of sin/cos.approx.ftz.f32 over every FP32 x with
// |x| <= the float with bits `hi_bits`, against FP64 sin/cos of the same x:
// out[0] = max |sin err|, out[1] = max |cos err| (as order-preserving bits of
// non-negative doubles, combined by atomicMax).
__global__ void probe_sincos_exhaustive(uint32_t hi_bits, unsigned long long* out) {
    const unsigned long long total = 2ull * ((unsigned long long)hi_bits + 1ull);
    double ms = 0.0, mc = 0.0;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t bits = (uint32_t)(i >> 1) | ((uint32_t)(i & 1ull) << 31);
        const float x = __uint_as_float(bits);
        float s, c;
        asm("sin.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(x));
        asm("cos.approx.ftz.f32 %0, %1;" : "=f"(c) : "f"(x));
        double sr, cr;
        sincos((double)x, &sr, &cr);
        ms = fmax(ms, fabs((double)s - sr));
        mc = fmax(mc, fabs((double)c - cr));
    }
    for (int o = 16; o > 0; o >>= 1) {
        ms = fmax(ms, __shfl_down_sync(0xffffffffu, ms, o));
        mc = fmax(mc, __shfl_down_sync(0xffffffffu, mc, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out + 0, (unsigned long long)__double_as_longlong(ms));
        atomicMax(out + 1, (unsigned long long)__double_as_longlong(mc));
    }
}

// Exhaustive relative accuracy of rsqrt.approx.ftz.f32 over every FP32 x with
// bits in [lo_bits, hi_bits), against 1 / sqrt(x) in FP64: out[0] = max
// |rsqrt.approx(x) * sqrt(x) - 1|.
__global__ void probe_rsqrt_exhaustive(uint32_t lo_bits, uint32_t hi_bits, unsigned long long* out) {
    double m = 0.0;
    const unsigned long long total = (unsigned long long)(hi_bits - lo_bits);
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const float x = __uint_as_float(lo_bits + (uint32_t)i);
        float r;
        asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
        m = fmax(m, fabs((double)r * sqrt((double)x) - 1.0));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
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

// New: measured accuracy of the MUFU approximations used by the precision-form
// far-field, exhaustively over their input ranges (see celeris_dev::kSinCosAbsErr).
extern "C" int celeris_probe_mufu_accuracy(double* measured, double* model) {
    CEL_TRY(celeris_rt::require_device());
    if (!measured || !model) return celeris_rt::set_error(CELERIS_ERR_INVALID_ARG, "null output");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    unsigned long long* d = nullptr;
    CEL_CUDA(cudaMalloc(&d, 4 * sizeof(unsigned long long)));
    CEL_CUDA(cudaMemset(d, 0, 4 * sizeof(unsigned long long)));
    const float pi_f = 3.14159265358979323846f;  // the precision form's reduced angles: |ang| <= pi_f
    uint32_t pi_bits;
    memcpy(&pi_bits, &pi_f, sizeof(pi_bits));
    probe_sincos_exhaustive<<<sms * 16, 256>>>(pi_bits, d);
    const float lo_f = 0x1p-10f, hi_f = 0x1p30f;
    uint32_t lo_bits, hi_bits;
    memcpy(&lo_bits, &lo_f, sizeof(lo_bits));
    memcpy(&hi_bits, &hi_f, sizeof(hi_bits));
    probe_rsqrt_exhaustive<<<sms * 16, 256>>>(lo_bits, hi_bits, d + 2);
    celeris_rt::count_launch(2);
    unsigned long long h[4];
    const cudaError_t e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    CEL_CUDA(e);
    for (int i = 0; i < 3; ++i) memcpy(&measured[i], &h[i], sizeof(double));
    model[0] = model[1] = celeris_dev::kSinCosAbsErr;
    model[2] = celeris_dev::kRsqrtRelErr;
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
