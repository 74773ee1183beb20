// ORACLE - test infrastructure only (the GPU comparator of bench.py).
//
// The REFERENCE's own FP32 far-field kernel, src/celeris/cuda/propagate.cu:36-84
// (psf_kernel) with its host wrapper propagate_psf (propagate.cu:133-193),
// compiled unmodified for sm_100a from the reference tree (included below by
// path; nothing is copied) by oracle/Makefile into oracle/_ref/libref_psf_cuda.so.
// bench.py times it beside the precision-form kernel and reports its error
// against the FP64 form; the product never loads this library.
#include "celeris/cuda/propagate.cu"

#define REF_API extern "C" __attribute__((visibility("default")))

// The reference's public call: host buffers in and out, |E|^2 (double) on the
// n x n grid; its own per-call allocation, float staging and copies.
REF_API int ref_cuda_propagate_psf(const double* px, const double* py, const double* pt, int npil, double cx,
                                   double cy, double z, double k, int n, double half_window, double* out) {
    return celeris::cuda::propagate_psf(px, py, reinterpret_cast<const std::complex<double>*>(pt), npil, cx, cy, z,
                                        k, n, half_window, out)
               ? 0
               : 1;
}

// The reference kernel alone on device buffers (float x, y, Re t, Im t;
// float |E|^2 out), launched with the grid and arguments propagate_psf uses;
// `reps` launches timed with CUDA events on the legacy default stream.
// *ms_per_launch receives the mean launch time.
REF_API int ref_cuda_psf_kernel(const float* dx, const float* dy, const float* dtr, const float* dti, int npil,
                                double cx, double cy, double z, double k, int n, double half_window, float* dout,
                                int reps, float* ms_per_launch) {
    const size_t NN = static_cast<size_t>(n) * n;
    const float step = static_cast<float>(2.0 * half_window / (n - 1));
    const int blocks = static_cast<int>((NN + celeris::cuda::kBlock - 1) / celeris::cuda::kBlock);
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return 2;
    cudaEventRecord(a);
    for (int r = 0; r < reps; ++r)
        celeris::cuda::psf_kernel<<<blocks, celeris::cuda::kBlock>>>(
            dx, dy, dtr, dti, npil, static_cast<float>(cx), static_cast<float>(cy), static_cast<float>(z),
            static_cast<float>(k), n, static_cast<float>(half_window), step, dout);
    cudaEventRecord(b);
    const cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return 3;
    *ms_per_launch = ms / (reps > 0 ? reps : 1);
    return 0;
}
