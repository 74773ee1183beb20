/*
 * celeris_b200.h - C ABI of the B200-native CELERIS hot path.
 *
 * Two data-parallel paths sit behind this boundary:
 *   1. the Rayleigh-Sommerfeld (RS) far-field sum over focal pixels x pillars
 *        E(p) = sum_j t_j exp(i k R_pj) / R_pj,
 *        R_pj = sqrt((fx_p - x_j)^2 + (fy_p - y_j)^2 + z_p^2)
 *      (reference: src/celeris/cuda/propagate.cu:36-130 psf/zx kernels,
 *       src/celeris/analysis/focal.cpp:205-238 propagate_pillars);
 *   2. the 2D vectorial RCWA unit-cell solve (reference:
 *      src/celeris/rcwa/rcwa2d.cpp:209-488 solve_rcwa_2d) and the library sweep
 *      built on it (src/celeris/design/metalens.cpp:122-163).
 *
 * Conventions
 *   - Every entry point returns an int status (CELERIS_OK == 0). On a non-zero
 *     status celeris_last_error() returns a message for the calling thread.
 *     There is no CPU fallback: without a CUDA device the far-field and RCWA
 *     entry points return CELERIS_ERR_NO_DEVICE.
 *   - Complex arrays are interleaved (re, im) doubles: the memory layout of
 *     std::complex<double>[] and of numpy complex128.
 *   - Host-buffer entry points ("drop-in" forms) are synchronous from the
 *     caller's view, like the reference, and thread-safe (each calling thread
 *     gets streams of its own). *_dev entry points take device pointers and a
 *     cudaStream_t (passed as void*, NULL = legacy default stream) and are
 *     asynchronous with respect to the host; their scratch comes from a
 *     workspace arena per (device, stream), so calls on ONE stream from
 *     several host threads at once must be serialised by the caller.
 *   - Focal grid: pixel (i, j), i = column, j = row, row-major index j*n + i,
 *       fx = cx - W + i * step, fy = cy - W + j * step, step = 2W / (n - 1)
 *     (propagate.cu:51-52, focal.cpp:223-226).
 */
#ifndef CELERIS_B200_H
#define CELERIS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define CELERIS_OK 0
#define CELERIS_ERR_NO_DEVICE 1     /* no CUDA device (reference: propagate_psf returns false) */
#define CELERIS_ERR_INVALID_ARG 2   /* bad sizes / NULL pointers (reference: std::invalid_argument) */
#define CELERIS_ERR_OOM 3           /* device or pinned allocation failed */
#define CELERIS_ERR_CUDA 4          /* a CUDA runtime call or kernel failed */
#define CELERIS_ERR_EIG_NOCONV 5    /* QR eigensolve hit its sweep cap (LAPACK info > 0) */
#define CELERIS_ERR_TOO_LARGE 6     /* size beyond a documented limit */
#define CELERIS_ERR_DEVICE_TIMEOUT 7 /* a bounded device-side wait ran out */
#define CELERIS_ERR_SINGULAR 8      /* exactly singular pivot in an LU factorization */

/* Far-field arithmetic forms. */
#define CELERIS_FORM_PLAIN_F64 0 /* FP64 throughout, the reference CPU method (focal.cpp:229-233) */
#define CELERIS_FORM_F32C 1      /* FP32 terms, FP64 k*z phase reduction, compensated accumulation */

/* ---- device / diagnostics -------------------------------------------------- */

/* replaces celeris::cuda::available() (src/celeris/cuda/propagate.hpp:20) */
int celeris_available(void);
/* replaces celeris::cuda::device_name() (src/celeris/cuda/propagate.hpp:21) */
const char* celeris_device_name(void);
/* New: message for the last non-zero status returned on this thread. */
const char* celeris_last_error(void);
/* New: ABI version (major * 10000 + minor * 100 + patch). */
int celeris_abi_version(void);
/* New: number of kernels this library launched since load (all threads). */
uint64_t celeris_launch_count(void);
/* New: free every device workspace arena (all devices, all threads' streams);
 * the next call allocates again. Call it with no call of this library in
 * flight on any thread. A thread's streams, events, pinned staging and device
 * I/O buffer are released when that thread exits. */
int celeris_release_workspace(void);

/* New: measured op rates of the current device (MUFU sin.approx results/s,
 * FP32 FMA/s, FP64 FMA/s) from short probe kernels; roofline denominators. */
int celeris_probe_peaks(double* mufu_per_s, double* ffma_per_s, double* dfma_per_s);
/* New: FP64 FMA/s of the tensor cores (mma.sync m8n8k4 f64) of the current
 * device from a short probe kernel; roofline denominator of the RCWA products. */
int celeris_probe_dmma(double* fma_per_s);
/* New: measured accuracy of the MUFU approximations the precision-form
 * far-field uses, over EVERY FP32 input of their ranges on the current device:
 * measured[0] = max |sin.approx(x) - sin(x)| and measured[1] the same for cos,
 * over all x in [-pi_f, pi_f]; measured[2] = max |rsqrt.approx(x) sqrt(x) - 1|
 * over all x in [2^-10, 2^30) (references in FP64). model[0..2] receive the
 * figures the stated error bound of the precision form assumes for the same
 * three quantities; the bound is valid on a device where measured <= model. */
int celeris_probe_mufu_accuracy(double* measured, double* model);
/* New: when on != 0, the far-field entry points record CUDA events around
 * their main kernel (on the stream it is launched on). */
int celeris_set_kernel_timing(int on);
/* New: duration in ms of the last timed main far-field kernel of this thread
 * (waits for it). Returns CELERIS_ERR_INVALID_ARG if none was recorded. */
int celeris_last_kernel_ms(double* ms);

/* ---- far-field: host-buffer drop-ins --------------------------------------- */

/* Drop-in for celeris::cuda::propagate_psf (src/celeris/cuda/propagate.hpp:27-30,
 * propagate.cu:133-193). Writes |E|^2 on the n x n grid into out (n*n doubles).
 * Computed in the plain FP64 form (the reference kernel is FP32; the plain form
 * reproduces the reference CPU path focal.cpp:224-236 instead). npil == 0
 * writes zeros (the reference then falls back to its CPU path, which returns
 * zeros, focal.cpp:216). */
int celeris_propagate_psf(const double* px, const double* py, const double* pt,
                          int npil, double cx, double cy, double z, double k,
                          int n, double half_window, double* out);

/* Drop-in for celeris::cuda::propagate_zx (src/celeris/cuda/propagate.hpp:35-38,
 * propagate.cu:195-253): |E|^2 on an nz x nx grid in the y = 0 plane, row = z
 * index, fx = xmin + (xmax - xmin) * ix / (nx - 1), z = zmin + (zmax - zmin) *
 * iz / (nz - 1) (the CPU form of throughfocus.cpp:105-118). Plain FP64. */
int celeris_propagate_zx(const double* px, const double* py, const double* pt,
                         int npil, double xmin, double xmax, int nx,
                         double zmin, double zmax, int nz, double k,
                         double* out);

/* New: general far-field on host buffers (the e2e path). form selects
 * CELERIS_FORM_*. field_out (2*n*n doubles, complex E) and intensity_out
 * (n*n doubles, |E|^2) may each be NULL. For CELERIS_FORM_F32C, err_out (may
 * be NULL) receives max_p |E_p - E64_p| / max_p |E_p| over a pixel sample
 * re-evaluated in the FP64 form on the device: the error stated with the
 * result. For the plain form *err_out = 0. */
int celeris_rs_field(int form, const double* px, const double* py,
                     const double* pt, int npil, double cx, double cy,
                     double z, double k, int n, double half_window,
                     double* field_out, double* intensity_out, double* err_out);

/* New: celeris_rs_field with the precision form's error stated two ways.
 * err_out (may be NULL) receives the SAMPLED error: max |E_p - E64_p| over a
 * pixel sample - a 16 x 16 lattice over the grid, the centre pixel and the
 * 21 x 21 pixels around the peak of |E| - recomputed in FP64 on the device, divided by
 * max_p |E_p| over the whole grid. bound_out (may be NULL) receives an UPPER
 * BOUND on max_p |E_p - E64_p| / max_p |E_p| over the whole grid from the error
 * model of the precision-form arithmetic: the MUFU approximation errors
 * (celeris_probe_mufu_accuracy) and the rounding of FP32 constants counted
 * without cancellation, the FP32 rounding errors of the terms and of the tile
 * sums counted as independent and mean zero with 8 standard deviations per
 * pixel (probabilistic rounding-error analysis: exceeded with probability
 * below 1e-13 per pixel under that model). Both are 0 for the plain form, and
 * both cost one pass over the pillars (the bound) or ~700 FP64 pixel sums (the
 * sample), run beside the field's download. */
int celeris_rs_field_bounded(int form, const double* px, const double* py,
                             const double* pt, int npil, double cx, double cy,
                             double z, double k, int n, double half_window,
                             double* field_out, double* intensity_out,
                             double* err_out, double* bound_out);

/* ---- far-field: device-buffer forms ---------------------------------------- */

/* New: far-field with inputs resident on the device. d_field (2*n*n doubles)
 * and d_intensity (n*n) may each be NULL. stream: cudaStream_t or NULL. */
int celeris_rs_field_dev(int form, const double* d_px, const double* d_py,
                         const double* d_pt, int npil, double cx, double cy,
                         double z, double k, int n, double half_window,
                         double* d_field, double* d_intensity, void* stream);

/* New, with no counterpart in the reference: the far-field of
 * celeris_rs_field_dev for callers that cannot allocate device memory - for
 * example a host whose memory pool already owns the GPU's free memory, or a
 * latency-critical loop in which the device-wide synchronisation of
 * cudaMalloc/cudaFree is not acceptable. It allocates nothing: its scratch (the
 * pillar records and the per-chunk partial sums) is a fixed 48 MiB array that
 * every GPU holds from the moment the library's far-field module is loaded on
 * it until the process exits. With CUDA's lazy module loading (the default)
 * that happens at the first far-field call of any kind on the device, so the
 * 48 MiB are taken then, from the device's free memory. Inputs and outputs are
 * the caller's device buffers, as for celeris_rs_field_dev.
 * Limit: (16 B per pillar for CELERIS_FORM_F32C, 32 B for the plain form,
 * rounded up to 256 B) + 16 B per focal pixel must fit in 48 MiB; the pillar
 * axis is cut into fewer, longer chunks until every chunk's partial sums fit
 * (the 785,456-pillar x 1024^2 metalens fits in both forms). Larger requests
 * return CELERIS_ERR_TOO_LARGE. Set-up: the first call on each device (with
 * that device current) loads the module and looks up the array's device
 * address (cudaGetSymbolAddress), which is then cached. A call with n = 0 or
 * npil = 0 does only that, so make one such call on each device before a
 * memory pool takes the free memory and before any stream capture begins.
 * All calls share the one array, which keeps the last call's contents: calls
 * whose kernels overlap on the GPU (different streams, or different host
 * threads without ordering) race on it and must be serialised by the caller. */
int celeris_rs_field_noalloc(int form, const double* d_px, const double* d_py,
                             const double* d_pt, int npil, double cx, double cy,
                             double z, double k, int n, double half_window,
                             double* d_field, double* d_intensity, void* stream);

/* New: rows [row0, row0 + nrows) of the n x n grid of celeris_rs_field_dev
 * (the same pixel positions and arithmetic), for a focal grid split by rows
 * over several devices: d_field holds nrows * n complex values (d_intensity
 * nrows * n), row-major, row i = grid row row0 + i. */
int celeris_rs_field_rows_dev(int form, const double* d_px, const double* d_py,
                              const double* d_pt, int npil, double cx, double cy,
                              double z, double k, int n, double half_window,
                              int row0, int nrows, double* d_field,
                              double* d_intensity, void* stream);

/* New: adjoint (conjugate-transpose, pixel -> pillar) RS sum on the same grid:
 *   d_out[j] = sum_p conj(g_pj) * d_v[p],   g_pj = exp(i k R_pj) / R_pj.
 * d_v: n*n complex, d_out: npil complex. This is the vector-Jacobian product of
 * celeris_rs_field_dev w.r.t. the pillar transmissions t (PyTorch convention).
 * form: CELERIS_FORM_PLAIN_F64, or CELERIS_FORM_F32C (the precision form's
 * arithmetic with pillars as outputs: packed FP32 terms, compensated sums,
 * e^{-ikz} applied in FP64).
 * The reference has no adjoint (its only gradient is central finite differences
 * of RCWA, src/celeris/design/optimize.cpp:60-71). */
int celeris_rs_adjoint_dev(int form, const double* d_px, const double* d_py,
                           int npil, double cx, double cy, double z, double k,
                           int n, double half_window, const double* d_v,
                           double* d_out, void* stream);

/* New: the adjoint over rows [row0, row0 + nrows) of the grid only: d_v holds
 * nrows * n complex pixel values (row i = grid row row0 + i). The adjoint of a
 * field split by rows is the sum of these partial adjoints (one all-reduce). */
int celeris_rs_adjoint_rows_dev(int form, const double* d_px, const double* d_py,
                                int npil, double cx, double cy, double z, double k,
                                int n, double half_window, int row0, int nrows,
                                const double* d_v, double* d_out, void* stream);

/* New: sampled FP64 check of a computed field. For the pixel indices d_idx[0..ns)
 * and the 21 x 21 pixels around the peak of |E| recomputes E in the plain FP64
 * form and writes max|E - E64| over the sample divided by max over all n*n
 * pixels of |E| into *err_out (host). Synchronous. */
int celeris_rs_check_dev(const double* d_px, const double* d_py,
                         const double* d_pt, int npil, double cx, double cy,
                         double z, double k, int n, double half_window,
                         const double* d_field, const int* d_idx, int ns,
                         double* err_out, void* stream);

/* New: the error bound of celeris_rs_field_bounded for a precision-form field
 * d_field (n*n complex) computed on the device from these inputs: an upper
 * bound on max_p |E_p - E64_p| / max_p |E_p|. Synchronous. */
int celeris_rs_error_bound_dev(const double* d_px, const double* d_py,
                               const double* d_pt, int npil, double cx, double cy,
                               double z, double k, int n, double half_window,
                               const double* d_field, double* bound_out,
                               void* stream);

/* New: synchronize `stream` and report a device-side failure recorded by an
 * earlier asynchronous *_dev call on that stream: CELERIS_ERR_DEVICE_TIMEOUT (a
 * bounded wait ran out) or CELERIS_ERR_INVALID_ARG (a pillar input or an
 * adjoint pixel value was NaN or Inf; non-finite values propagate to the
 * outputs). Host-buffer calls report these themselves. */
int celeris_sync_status(void* stream);

/* ---- failure-path diagnostics (tests of the error reporting) -------------- */

/* New: run the bounded device wait of the far-field tile pipeline on a barrier
 * that never completes, limited to `polls` polls: returns
 * CELERIS_ERR_DEVICE_TIMEOUT with the device context intact (no trap). */
int celeris_device_wait_selftest(unsigned polls);
/* New: make the next `count` device allocations of this library fail as if
 * cudaMalloc had (CELERIS_ERR_OOM, nothing allocated); 0 clears. The
 * environment variable CELERIS_DEBUG_FAIL_ALLOC=<count> sets the same count
 * when the library loads. */
int celeris_debug_fail_alloc(int count);
/* New: cap the QR iterations of the RCWA / eigensolver Schur stage at `cap`
 * (0 restores the solver's own cap, 2n + 100), so a test can drive the
 * non-convergence report (CELERIS_ERR_EIG_NOCONV, per-cell info > 0 like
 * LAPACK's). Applies to the current device. */
int celeris_debug_qr_iteration_cap(int cap);

/* ---- RCWA ------------------------------------------------------------------ */

/* Shapes (src/celeris/rcwa/rcwa2d.hpp:26-31). */
#define CELERIS_SHAPE_RECT 0
#define CELERIS_SHAPE_ELLIPSE 1
#define CELERIS_SHAPE_CROSS 2
#define CELERIS_SHAPE_RING 3

/* One unit cell: one patterned layer between two half-spaces, normal or oblique
 * incidence. All permittivities/indices are complex (re, im). Mirrors the
 * arguments solve_rcwa_2d receives for a one-layer Rcwa2DStack
 * (rcwa2d.hpp:114-124, metalens.cpp:141-147). */
typedef struct celeris_rcwa_cell {
    double period_x_um, period_y_um;
    double wavelength_um, theta_rad, phi_rad;
    double n_inc[2];      /* incident half-space index n + i k */
    double n_sub[2];      /* substrate index */
    double eps_pillar[2]; /* pillar permittivity eps = n^2 */
    double eps_bg[2];     /* background permittivity */
    double fill_x, fill_y, thickness_um;
    double shape_param, rotation_rad;
    int shape;            /* CELERIS_SHAPE_* */
    int Mx, My;           /* harmonic half-counts: N = (2Mx+1)(2My+1) */
    int grid;             /* Laurent raster size; <= 0: the reference's max(128, 8(2M+1)) (rcwa2d.cpp:337) */
    int force_laurent;    /* 1: rasterize plain rectangles too (otherwise the analytic Li path, rcwa2d.cpp:280) */
} celeris_rcwa_cell;

/* Per-cell, per-polarization result (Rcwa2DResult, rcwa2d.hpp:84-94). */
typedef struct celeris_rcwa_result {
    double R, T, sum_de, de_t0, de_r0;
    double tx0[2], ty0[2];
} celeris_rcwa_result;

/* Drop-in for celeris::solve_rcwa_2d on a one-layer stack (rcwa2d.cpp:209-488)
 * with incident field (Ex0, Ey0). Synchronous, host buffers. */
int celeris_solve_rcwa_2d(const celeris_rcwa_cell* cell, const double* Ex0,
                          const double* Ey0, celeris_rcwa_result* out);

/* Every real field of a cell must be finite: a NaN or Inf returns
 * CELERIS_ERR_INVALID_ARG (naming the cell in a batch) before any device work. */

/* New: batched uneven cells. Each cell is solved once (one eigensolve, one
 * S-matrix) for BOTH the X (Ex0=1, Ey0=0) and Y (Ex0=0, Ey0=1) excitations;
 * out receives 2*ncell results: out[2c] = X, out[2c+1] = Y. Cells are bucketed
 * by harmonic count internally. info (ncell ints, may be NULL) receives 0 or the
 * failure code per cell: > 0 the QR eigensolve did not converge (LAPACK-style
 * index), < 0 an exactly singular pivot; with info the call returns CELERIS_OK
 * and reports failures there only, without info a failure returns
 * CELERIS_ERR_EIG_NOCONV / CELERIS_ERR_SINGULAR naming the first failing cell.
 * Cells symmetric under both mirrors at normal incidence (every unrotated
 * shape, theta = 0) solve the eigenproblem in its four parity classes (the same
 * eigenpairs at a quarter of the order; CELERIS_RCWA_SYMMETRY=0 turns it off),
 * only the two excited classes, and only one of them when the cell is also
 * symmetric under a 90-degree rotation (square period, Mx = My, fill_x =
 * fill_y). A cell whose Fourier operators are not symmetric to within
 * CELERIS_RCWA_SYM_TOL (default 1e-9) of their largest entry is solved again at
 * full order (0 forces that for every cell). Synchronous, host buffers. */
int celeris_rcwa_batch(const celeris_rcwa_cell* cells, int ncell,
                       celeris_rcwa_result* out, int* info);

/* Drop-in for celeris::solve_rcwa_2d on a multi-layer stack (rcwa2d.cpp:209-488;
 * the S-matrix recursion of rcwa2d.cpp:376-401 over nlayers + 1 interfaces).
 * layers[0] is next to the incident half-space, layers[nlayers-1] next to the
 * substrate. Orders, periods, wavelength, angles and both half-space indices
 * must agree across the layers (the reference's Rcwa2DStack holds them once);
 * each layer carries its own pattern, materials and thickness. Synchronous,
 * host buffers. */
int celeris_solve_rcwa_2d_stack(const celeris_rcwa_cell* layers, int nlayers,
                                const double* Ex0, const double* Ey0,
                                celeris_rcwa_result* out);

/* Drop-in for celeris::eig_general (eig.hpp:25; eig.cpp:52-92): right
 * eigenpairs of a general complex n x n matrix, A * v_i = lambda_i * v_i. A and
 * evecs are column-major complex (Eigen::MatrixXcd / LAPACK layout, n*n
 * interleaved (re, im) pairs), evals n complex. Each eigenvector has unit
 * 2-norm and its largest-magnitude component real and positive (zgeev's
 * normalisation); the order of the eigenvalues is the QR's. The device path is
 * the RCWA eigen-stages (Hessenberg, multishift QR with early deflation,
 * back substitution). n <= 2048. Synchronous, host buffers. */
int celeris_eig_general(const double* A, int n, double* evals, double* evecs);

/* New: `count` matrices of order n at once (one CTA per matrix), stored one
 * after another; info (count ints, may be NULL) receives 0 or the QR failure
 * code per matrix (without info a failure is CELERIS_ERR_EIG_NOCONV). */
int celeris_eig_general_batch(const double* A, int n, int count, double* evals,
                              double* evecs, int* info);

/* Per-order efficiency (OrderEfficiency, rcwa2d.hpp:101-107). */
typedef struct celeris_rcwa_order {
    int p, q;          /* diffraction order */
    double de_t, de_r; /* transmitted / reflected efficiency of the order */
    int prop_t, prop_r; /* 1 if the order propagates in the substrate / incident medium */
} celeris_rcwa_order;

/* Drop-in for celeris::solve_rcwa_2d with its orders_out argument
 * (rcwa2d.cpp:464-485): as celeris_solve_rcwa_2d_stack (one layer or several),
 * and orders[i] for every order i = (p + Mx)(2 My + 1) + (q + My), in the
 * reference's loop order. orders holds max_orders >= (2Mx+1)(2My+1) records. */
int celeris_solve_rcwa_2d_orders(const celeris_rcwa_cell* layers, int nlayers,
                                 const double* Ex0, const double* Ey0,
                                 celeris_rcwa_result* out, celeris_rcwa_order* orders,
                                 int max_orders);

/* New: batched multi-layer stacks. Stack s is layers[layer_start[s] ..
 * layer_start[s+1]) (layer_start holds nstack + 1 offsets). Like
 * celeris_rcwa_batch, each stack is solved once for both excitations:
 * out[2s] = X (Ex0=1), out[2s+1] = Y (Ey0=1). info (nstack ints, may be NULL)
 * receives 0, the eigensolve failure code of a layer (> 0), or minus the
 * singular pivot of an interface system (< 0) per stack. */
int celeris_rcwa_stack_batch(const celeris_rcwa_cell* layers, const int* layer_start,
                             int nstack, celeris_rcwa_result* out, int* info);

/* New: the autotuner's table (one line per bucket shape Mx, My, raster: the
 * threads per CTA it chose for each RCWA stage), NUL-terminated into buf. The
 * batch runs all buckets as one CUDA graph (one stream per bucket), captured on
 * the first call for a given set of bucket shapes and replayed afterwards. */
int celeris_rcwa_tuning_report(char* buf, int len);

#ifdef __cplusplus
}
#endif

#endif /* CELERIS_B200_H */
