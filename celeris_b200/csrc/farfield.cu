// Rayleigh-Sommerfeld far-field sum on sm_100a.
//
//   E(p) = sum_j t_j exp(i k R_pj) / R_pj
//
// Reference: src/celeris/cuda/propagate.cu:36-130 (FP32 psf/zx kernels, one
// thread per pixel, 256-pillar shared tiles), src/celeris/analysis/focal.cpp:
// 205-238 (CPU FP64 loop that the plain form reproduces) and
// throughfocus.cpp:105-118 (CPU caustic loop).
//
// Layout in HBM
//   pillar records  f64 form: double4 {x, y, Re t, Im t}            32 B/pillar
//                   f32 form: float4  {x - ox, y - oy, |t|, arg t/2pi} 16 B/pillar
//   partial sums    double2 [nchunk][npix] (pillar-chunk split of the sum)
//   outputs         double2 field [npix] and/or double |E|^2 [npix]
//
// Kernels
//   ff_pack_*        FP64 inputs -> pillar records (one pass over the pillars)
//   rs_f64_kernel    plain form: FP64 terms exactly as focal.cpp:229-233
//   rs_f32c_kernel   precision form: FP32 terms; R - z refined by one Newton
//                    step on (R - z)(R + z) = dx^2 + dy^2 so the large k*z part
//                    of the phase never enters FP32; phase reduced in turns;
//                    MUFU rsqrt/sin/cos; per-tile FP32 partial sums folded into
//                    TwoSum-compensated (hi, lo) pairs.
//   rs_reduce_kernel ordered FP64 sum over chunks; f32 form multiplies by the
//                    FP64 global phase exp(i k z).
//   rs_adj_f64_kernel conjugate-transpose (pixel -> pillar) sum for the adjoint.
// Every main kernel stages its tiles in shared memory with cp.async.bulk
// (TMA bulk copies) completing on an mbarrier, 3-4 stages deep, so each record
// is read from HBM once per CTA.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "runtime.cuh"

namespace {

using celeris_rt::count_launch;
using celeris_rt::set_error;
using celeris_rt::Workspace;
using namespace celeris_dev;

// Device-side failure flags of the far-field kernels, read and cleared by the
// host after a synchronous call (or by celeris_sync_status).
constexpr int kFlagTimeout = 1;    // a bounded device wait ran out
constexpr int kFlagNonFinite = 2;  // a pillar coordinate / transmission or an adjoint input was NaN or Inf
// One status word per stream (hashed into kStatusSlots slots, the legacy
// default stream in slot 0), so a flag raised by an asynchronous call on one
// stream is reported by the call or celeris_sync_status on that stream, not by
// an unrelated call on another.
constexpr int kStatusSlots = 1024;
__device__ int g_ff_status[kStatusSlots];

constexpr int kThreads = 256;
constexpr int kTile64 = 256;  // pillars (or pixels) per stage, 32 B records -> 8 KB
constexpr int kTile32 = 512;  // pillars per stage, 16 B records -> 8 KB
constexpr int kStages = 4;
constexpr int kPPT64 = 2;     // pixels per thread, plain form
constexpr int kPPT32 = 6;     // pixels per thread, precision form: 3 packed pixel pairs share each pillar record
constexpr int kAdjPPT = 2;    // pillars per thread, adjoint
constexpr int kAdjPPT32 = 6;  // pillars per thread, precision-form adjoint (3 packed pairs)

enum { GEOM_PSF = 0, GEOM_ZX = 1 };

// Pixel grid. GEOM_PSF: fx = (cx - W) + i*step, fy = (cy - W) + j*step, z const
// (focal.cpp:223-227). GEOM_ZX: fx = xmin + (xmax - xmin)*i/(nx-1), fy = 0,
// z = zmin + (zmax - zmin)*j/(nz-1) (throughfocus.cpp:108-110).
struct Geom {
    int mode;
    int nx, ny;
    double a0, a1;  // PSF: cx - W, step      ZX: xmin, xmax
    double b0, b1;  // PSF: cy - W, step      ZX: zmin, zmax
    double z;       // PSF: z
    double ox, oy;  // origin subtracted from pillars and pixels in the f32 form
    int row0;       // PSF: first row of a row block (pixel row j is grid row row0 + j)
    int slot;       // status word of the launching stream (g_ff_status)
};

__device__ __forceinline__ void pixel_pos(const Geom& g, int i, int j, double& fx,
                                          double& fy, double& fz) {
    if (g.mode == GEOM_PSF) {
        fx = g.a0 + i * g.a1;
        fy = g.b0 + (j + g.row0) * g.b1;
        fz = g.z;
    } else {
        fx = g.a0 + (g.a1 - g.a0) * i / (g.nx - 1);
        fy = 0.0;
        fz = g.b0 + (g.b1 - g.b0) * j / (g.ny - 1);
    }
}

__device__ __forceinline__ void record_timeout(int slot) { atomicOr(&g_ff_status[slot], kFlagTimeout); }

// Non-finite inputs are not screened on the host (that would cost a pass over
// the caller's arrays and a synchronisation); the packing pass, which reads
// every input once anyway, flags them and the call reports
// CELERIS_ERR_INVALID_ARG. Non-finite values propagate to the outputs.
__device__ __forceinline__ void flag_nonfinite(int slot, double a, double b, double c, double d) {
    if (!(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(d))) atomicOr(&g_ff_status[slot], kFlagNonFinite);
}

// ---- packing ----------------------------------------------------------------
__global__ void ff_pack_f64(const double* __restrict__ px, const double* __restrict__ py,
                            const double2* __restrict__ pt, int npil, int slot,
                            double4* __restrict__ rec) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= npil) return;
    double2 t = pt[j];
    flag_nonfinite(slot, px[j], py[j], t.x, t.y);
    rec[j] = make_double4(px[j], py[j], t.x, t.y);
}

// ---- pixel grid of the precision form ----------------------------------------------
// Pillar coordinates are rounded to FP32 relative to the FP32 origin (ulp <=
// G below). A pixel is split into a base on the grid of step G = 2^(ilogb(L) -
// 23), the ulp of L = the largest |x - ox|, |y - oy| of a pillar plus the
// largest pixel offset, and a small offset c from it: base - x then rounds (if
// at all) only bits of x, never bits of the pixel, and the offset enters rho^2
// through c (2 (base - x) + c), a product with the pillar. Rounding fx - x
// directly would snap fx to the grid of x's exponent - the same shift for
// every pillar of that exponent - and adding a pixel-only value to an FP32
// number likewise rounds it the same way for every pillar of one exponent:
// errors that add up coherently near a focus.
__host__ __device__ __forceinline__ double grid_step(double L) {
    L = fmax(L, 1e-30);
    return ldexp(1.0, ilogb(L) - 23);
}

// ext[0] = bits of max_j max(|x_j - ox|, |y_j - oy|)
__global__ void ff_extent_kernel(const double* __restrict__ px, const double* __restrict__ py, int npil, double ox,
                                 double oy, unsigned long long* __restrict__ ext) {
    double m = 0.0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npil; j += gridDim.x * blockDim.x)
        m = fmax(m, fmax(fabs(px[j] - ox), fabs(py[j] - oy)));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(ext, (unsigned long long)__double_as_longlong(m));
}

__device__ __forceinline__ double ext_grid(const unsigned long long* ext, double wmax) {
    return grid_step(__longlong_as_double((long long)*ext) + wmax);
}

__global__ void ff_pack_f32(const double* __restrict__ px, const double* __restrict__ py,
                            const double2* __restrict__ pt, int npil, double ox, double oy, int slot,
                            float4* __restrict__ rec) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= npil) return;
    double2 t = pt[j];
    flag_nonfinite(slot, px[j], py[j], t.x, t.y);
    double A = hypot(t.x, t.y);
    double psi = atan2(t.y, t.x) * 0.15915494309189533577;  // turns
    rec[j] = make_float4((float)(px[j] - ox), (float)(py[j] - oy), (float)A, (float)psi);
}

// pixel records for the adjoint: {fx, fy, Re v, Im v}
__global__ void ff_pack_pix(Geom g, const double2* __restrict__ v, double4* __restrict__ rec) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    int npix = g.nx * g.ny;
    if (p >= npix) return;
    int j = p / g.nx, i = p - j * g.nx;
    double fx, fy, fz;
    pixel_pos(g, i, j, fx, fy, fz);
    double2 vv = v[p];
    flag_nonfinite(g.slot, vv.x, vv.y, 0.0, 0.0);
    rec[p] = make_double4(fx, fy, vv.x, vv.y);
}

// precision-form adjoint: float4 {fx - ox, fy - oy, Re v, Im v} per pixel
__global__ void ff_pack_pix_f32(Geom g, const double2* __restrict__ v, float4* __restrict__ rec) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    int npix = g.nx * g.ny;
    if (p >= npix) return;
    int j = p / g.nx, i = p - j * g.nx;
    double fx, fy, fz;
    pixel_pos(g, i, j, fx, fy, fz);
    double2 vv = v[p];
    flag_nonfinite(g.slot, vv.x, vv.y, 0.0, 0.0);
    rec[p] = make_float4((float)(fx - g.ox), (float)(fy - g.oy), (float)vv.x, (float)vv.y);
}

// ---- tile pipeline (shared by all main kernels) ----------------------------
// Thread 0 owns the producer role: it arms stage s's mbarrier with the byte
// count and issues one bulk copy. All threads consume. A stage is refilled only
// after a __syncthreads that follows its last read.
template <typename Rec, int TILE>
struct TilePipe {
    Rec (*buf)[TILE];
    uint64_t* full;
    const Rec* src;
    int c0, c1, ntiles, slot;

    __device__ void init(Rec (*b)[TILE], uint64_t* f, const Rec* s, int lo, int hi, int status_slot) {
        slot = status_slot;
        buf = b;
        full = f;
        src = s;
        c0 = lo;
        c1 = hi;
        ntiles = hi > lo ? (hi - lo + TILE - 1) / TILE : 0;
        if (threadIdx.x == 0) {
            for (int st = 0; st < kStages; ++st) mbar_init(&full[st], 1);
            fence_barrier_init();
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int t = 0; t < kStages && t < ntiles; ++t) issue(t);
    }
    __device__ int count(int t) const { return min(TILE, c1 - (c0 + t * TILE)); }
    __device__ void issue(int t) {
        const int st = t % kStages;
        const int base = c0 + t * TILE;
        const uint32_t bytes = (uint32_t)(count(t) * sizeof(Rec));
        mbar_arrive_expect_tx(&full[st], bytes);
        bulk_g2s(&buf[st][0], src + base, bytes, &full[st]);
    }
    __device__ bool wait(int t) { return mbar_wait(&full[t % kStages], (t / kStages) & 1); }
    // call after every thread finished reading tile t; returns false on timeout
    __device__ bool release(int t, bool got) {
        if (!__syncthreads_and(got)) {
            if (threadIdx.x == 0) record_timeout(slot);
            return false;
        }
        if (threadIdx.x == 0 && t + kStages < ntiles) {
            fence_proxy_async_smem();
            issue(t + kStages);
        }
        return true;
    }
};

// ---- plain FP64 form ----------------------------------------------------------
__global__ void __launch_bounds__(kThreads) rs_f64_kernel(const double4* __restrict__ rec,
                                                          int npil, int chunk_len, Geom g,
                                                          double k, double2* __restrict__ partial) {
    __shared__ __align__(128) double4 buf[kStages][kTile64];
    __shared__ __align__(8) uint64_t full[kStages];

    const int npix = g.nx * g.ny;
    const int spr = (g.nx + kPPT64 - 1) / kPPT64;
    const int strip = blockIdx.x * kThreads + threadIdx.x;
    const int j = strip / spr;
    const int i0 = (strip - j * spr) * kPPT64;
    const int jj = min(j, g.ny - 1);

    double fx[kPPT64], fy = 0.0, fz = 0.0;
#pragma unroll
    for (int q = 0; q < kPPT64; ++q) pixel_pos(g, min(i0 + q, g.nx - 1), jj, fx[q], fy, fz);
    const double z2 = fz * fz;

    TilePipe<double4, kTile64> pipe;
    const int lo = blockIdx.y * chunk_len;
    pipe.init(buf, full, rec, lo, min(npil, lo + chunk_len), g.slot);

    double er[kPPT64], ei[kPPT64];
#pragma unroll
    for (int q = 0; q < kPPT64; ++q) er[q] = ei[q] = 0.0;

    for (int t = 0; t < pipe.ntiles; ++t) {
        const bool got = pipe.wait(t);
        if (got) {
            const double4* tile = buf[t % kStages];
            const int cnt = pipe.count(t);
            for (int p = 0; p < cnt; ++p) {
                const double4 r = tile[p];
                const double dy = fy - r.y;
                const double dy2 = dy * dy;
#pragma unroll
                for (int q = 0; q < kPPT64; ++q) {
                    const double dx = fx[q] - r.x;
                    const double R = sqrt(dx * dx + dy2 + z2);
                    double s, c;
                    sincos(k * R, &s, &c);
                    const double inv = 1.0 / R;
                    const double pr = inv * c, pim = inv * s;  // std::polar(1/R, kR)
                    er[q] += r.z * pr - r.w * pim;             // t * polar
                    ei[q] += r.z * pim + r.w * pr;
                }
            }
        }
        if (!pipe.release(t, got)) return;
    }
    if (j < g.ny) {
#pragma unroll
        for (int q = 0; q < kPPT64; ++q)
            if (i0 + q < g.nx)
                partial[(size_t)blockIdx.y * npix + (size_t)j * g.nx + i0 + q] =
                    make_double2(er[q], ei[q]);
    }
}

// ---- precision form: FP32 terms, compensated accumulation -------------------
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sin_approx(float x) {
    float y;
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float cos_approx(float x) {
    float y;
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// Packed FP32 pairs (add / mul / fma .rn.f32x2, sm_100): one instruction does the
// same IEEE-rounded operation on two pixels, halving the issue slots of the
// term arithmetic. A pair lives in a 64-bit register, low half = first pixel.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk2(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ f32x2 dup2(float a) { return pk2(a, a); }
__device__ __forceinline__ void upk2(f32x2 r, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Knuth TwoSum: s + c += x with the rounding error of s + x kept in c.
__device__ __forceinline__ void two_sum_acc(float& s, float& c, float x) {
    const float t = s + x;
    const float bp = t - s;
    const float ap = t - bp;
    c += (s - ap) + (x - bp);
    s = t;
}

template <bool ZLO>
__global__ void __launch_bounds__(kThreads, 3) rs_f32c_kernel(const float4* __restrict__ rec,
                                                           int npil, int chunk_len, Geom g,
                                                           float il_hi, float il_lo,
                                                           const unsigned long long* __restrict__ ext,
                                                           double wmax, double2* __restrict__ partial) {
    __shared__ __align__(128) float4 buf[kStages][kTile32];
    __shared__ __align__(8) uint64_t full[kStages];

    const int npix = g.nx * g.ny;
    const int spr = (g.nx + kPPT32 - 1) / kPPT32;
    const int strip = blockIdx.x * kThreads + threadIdx.x;
    const int j = strip / spr;
    const int i0 = (strip - j * spr) * kPPT32;
    const int jj = min(j, g.ny - 1);

    // pixel coordinates relative to the FP32 origin (see grid_step): the row's
    // y as a grid value and its offset fr_y (|fr_y| <= G/2); the thread's x as
    // a base on the grid plus per-pixel offsets c_q (|c_q| <= G/2 + 5 steps):
    // dx_q = s0 + c_q with s0 = base - x
    const double G = ext_grid(ext, wmax);
    float bx = 0.f, cq[kPPT32], fyq = 0.f, fyo = 0.f, nfr2 = 0.f, z = 0.f, zl = 0.f;
    {
        double fx, fy, fz;
        pixel_pos(g, min(i0, g.nx - 1), jj, fx, fy, fz);
        const double xb = rint((fx - g.ox) / G) * G, yq = rint((fy - g.oy) / G) * G, fr = (fy - g.oy) - yq;
        bx = (float)xb;
        fyq = (float)yq;
        fyo = (float)(-2.0 * fr);
        nfr2 = (float)(-fr * fr);
        z = (float)fz;
        zl = (float)(fz - (double)z);  // z = z + zl to ~u^2 |z|
#pragma unroll
        for (int q = 0; q < kPPT32; ++q) {
            pixel_pos(g, min(i0 + q, g.nx - 1), jj, fx, fy, fz);
            cq[q] = (float)((fx - g.ox) - xb);
        }
    }
    const float z2 = z * z;
    const float kMagic = 12582912.0f;  // 1.5 * 2^23: x + M - M rounds x to an integer
    // pixel pairs and the constants of the packed term arithmetic
    constexpr int kPairs = kPPT32 / 2;
    f32x2 c2[kPairs];
#pragma unroll
    for (int h = 0; h < kPairs; ++h) c2[h] = pk2(cq[2 * h], cq[2 * h + 1]);
    const f32x2 Z2P = dup2(z2);
    const f32x2 NZ = dup2(-z), Z2X = dup2(2.0f * z), NHALF = dup2(-0.5f);
    const f32x2 Z2L = dup2(2.0f * zl);
    const f32x2 ILHI = dup2(il_hi), ILLO = dup2(il_lo), MAGIC = dup2(kMagic);
    const f32x2 TWOPI = dup2(6.28318530717958647692f);

    TilePipe<float4, kTile32> pipe;
    const int lo = blockIdx.y * chunk_len;
    pipe.init(buf, full, rec, lo, min(npil, lo + chunk_len), g.slot);

    float sr[kPPT32], cr[kPPT32], si[kPPT32], ci[kPPT32];
#pragma unroll
    for (int q = 0; q < kPPT32; ++q) sr[q] = cr[q] = si[q] = ci[q] = 0.f;

    for (int t = 0; t < pipe.ntiles; ++t) {
        const bool got = pipe.wait(t);
        if (got) {
            const float4* tile = buf[t % kStages];
            const int cnt = pipe.count(t);
            f32x2 er[kPairs], ei[kPairs];
#pragma unroll
            for (int h = 0; h < kPairs; ++h) er[h] = ei[h] = 0ull;
#pragma unroll 2
            for (int p = 0; p < cnt; ++p) {
                const float4 r = tile[p];  // {x, y, |t|, arg t / 2pi}
                // s0 = base - x, sy = fy - y (grid values: only bits of x, y
                // can round off); -(s0^2 + dy^2), dy = sy + fr_y
                const float s0 = bx - r.x, sy = fyq - r.y;
                const f32x2 RW = dup2(r.w), RZ = dup2(r.z), NS02 = dup2(-2.0f * s0);
                const f32x2 NB = dup2(fmaf(s0, -s0, fmaf(sy, -sy, fmaf(sy, fyo, nfr2))));
#pragma unroll
                for (int h = 0; h < kPairs; ++h) {
                    // -rho^2 = -(s0^2 + dy^2) - c (2 s0 + c)
                    const f32x2 ns = fma2(sub2(NS02, c2[h]), c2[h], NB);
                    const f32x2 u = sub2(Z2P, ns);                        // R^2 (seed, amplitude)
                    float ua, ub;
                    upk2(u, ua, ub);
                    const f32x2 ri = pk2(rsqrt_approx(ua), rsqrt_approx(ub));  // ~1/R
                    const f32x2 d0 = fma2(u, ri, NZ);          // ~R - z
                    // Newton on f(d) = d^2 + 2 (z + zl) d - rho^2 (root R - z for
                    // the FP64 z, so the FP64 phase k z applied later matches)
                    const f32x2 gg = ZLO ? fma2(d0, d0, fma2(Z2X, d0, fma2(Z2L, d0, ns)))
                                         : fma2(d0, d0, fma2(Z2X, d0, ns));
                    const f32x2 d = fma2(mul2(gg, ri), NHALF, d0);
                    // phase in turns: (R - z)/lambda + arg(t)/2pi; k z is added in FP64
                    const f32x2 th = fma2(d, ILHI, fma2(d, ILLO, RW));
                    const f32x2 w = sub2(MAGIC, add2(th, MAGIC));         // -(th rounded to an integer)
                    const f32x2 ang = mul2(add2(th, w), TWOPI);           // in [-pi, pi]
                    const f32x2 a = mul2(RZ, ri);                         // |t| / R
                    float aa, ab;
                    upk2(ang, aa, ab);
                    er[h] = fma2(a, pk2(cos_approx(aa), cos_approx(ab)), er[h]);
                    ei[h] = fma2(a, pk2(sin_approx(aa), sin_approx(ab)), ei[h]);
                }
            }
#pragma unroll
            for (int h = 0; h < kPairs; ++h) {
                float e0, e1, f0, f1;
                upk2(er[h], e0, e1);
                upk2(ei[h], f0, f1);
                two_sum_acc(sr[2 * h], cr[2 * h], e0);
                two_sum_acc(sr[2 * h + 1], cr[2 * h + 1], e1);
                two_sum_acc(si[2 * h], ci[2 * h], f0);
                two_sum_acc(si[2 * h + 1], ci[2 * h + 1], f1);
            }
        }
        if (!pipe.release(t, got)) return;
    }
    if (j < g.ny) {
#pragma unroll
        for (int q = 0; q < kPPT32; ++q)
            if (i0 + q < g.nx)
                partial[(size_t)blockIdx.y * npix + (size_t)j * g.nx + i0 + q] =
                    make_double2((double)sr[q] + (double)cr[q], (double)si[q] + (double)ci[q]);
    }
}

// ---- precision-form adjoint: out_j = e^{-ikz} sum_p (1/R) e^{-2 pi i (R - z)/lambda} v_p
// The forward kernel's arithmetic with the roles swapped: each thread owns
// kAdjPPT32 pillars (packed pairs), pixel records stream through the tiles; the
// product with v is conj(g) v = (1/R) [(c vr + s vi) + i (c vi - s vr)].
__global__ void __launch_bounds__(kThreads, 3) rs_adj_f32c_kernel(const float4* __restrict__ pix, int npix,
                                                                  int chunk_len, const double* __restrict__ px,
                                                                  const double* __restrict__ py, int npil, Geom g,
                                                                  float z, float il_hi, float il_lo,
                                                                  double2* __restrict__ partial) {
    __shared__ __align__(128) float4 buf[kStages][kTile32];
    __shared__ __align__(8) uint64_t full[kStages];
    constexpr int kPairs = kAdjPPT32 / 2;
    const int j0 = (blockIdx.x * kThreads + threadIdx.x) * kAdjPPT32;
    f32x2 xj[kPairs], yj[kPairs];
#pragma unroll
    for (int h = 0; h < kPairs; ++h) {
        const int a = min(j0 + 2 * h, npil - 1), b = min(j0 + 2 * h + 1, npil - 1);
        xj[h] = pk2((float)(px[a] - g.ox), (float)(px[b] - g.ox));
        yj[h] = pk2((float)(py[a] - g.oy), (float)(py[b] - g.oy));
    }
    const f32x2 NEG1 = dup2(-1.0f), NZ = dup2(-z), Z2X = dup2(2.0f * z), NHALF = dup2(-0.5f);
    const f32x2 Z2 = dup2(z * z), ILHI = dup2(il_hi), NILHI = dup2(-il_hi), ILLO = dup2(il_lo);
    const f32x2 MAGIC = dup2(12582912.0f);
    const f32x2 TWOPI = dup2(6.28318530717958647692f);

    TilePipe<float4, kTile32> pipe;
    const int lo = blockIdx.y * chunk_len;
    pipe.init(buf, full, pix, lo, min(npix, lo + chunk_len), g.slot);

    float sr[kAdjPPT32], cr[kAdjPPT32], si[kAdjPPT32], ci[kAdjPPT32];
#pragma unroll
    for (int q = 0; q < kAdjPPT32; ++q) sr[q] = cr[q] = si[q] = ci[q] = 0.f;

    for (int t = 0; t < pipe.ntiles; ++t) {
        const bool got = pipe.wait(t);
        if (got) {
            const float4* tile = buf[t % kStages];
            const int cnt = pipe.count(t);
            f32x2 er[kPairs], ei[kPairs];
#pragma unroll
            for (int h = 0; h < kPairs; ++h) er[h] = ei[h] = 0ull;
#pragma unroll 2
            for (int p = 0; p < cnt; ++p) {
                const float4 r = tile[p];  // {fx, fy, Re v, Im v}
                const f32x2 FX = dup2(r.x), FY = dup2(r.y), VR = dup2(r.z), VI = dup2(r.w), NVR = dup2(-r.z);
#pragma unroll
                for (int h = 0; h < kPairs; ++h) {
                    const f32x2 dx = fma2(xj[h], NEG1, FX), ndx = fma2(FX, NEG1, xj[h]);
                    const f32x2 dy = fma2(yj[h], NEG1, FY), ndy = fma2(FY, NEG1, yj[h]);
                    const f32x2 u = fma2(dx, dx, fma2(dy, dy, Z2));         // R^2 (seed only)
                    const f32x2 ns = fma2(dx, ndx, mul2(dy, ndy));          // -rho^2
                    float ua, ub;
                    upk2(u, ua, ub);
                    const f32x2 ri = pk2(rsqrt_approx(ua), rsqrt_approx(ub));  // ~1/R
                    const f32x2 d0 = fma2(u, ri, NZ);
                    const f32x2 gg = fma2(d0, d0, fma2(Z2X, d0, ns));
                    const f32x2 d = fma2(mul2(gg, ri), NHALF, d0);           // R - z
                    // (R - z)/lambda in turns, reduced exactly as in the forward kernel
                    const f32x2 np = mul2(d, NILHI);
                    const f32x2 rp = fma2(d, ILHI, np);
                    const f32x2 t = fma2(d, ILLO, rp);
                    const f32x2 w = fma2(add2(np, MAGIC), NEG1, MAGIC);
                    const f32x2 ang = mul2(fma2(add2(np, w), NEG1, t), TWOPI);
                    float aa, ab;
                    upk2(ang, aa, ab);
                    const f32x2 pr = mul2(ri, pk2(cos_approx(aa), cos_approx(ab)));
                    const f32x2 pi = mul2(ri, pk2(sin_approx(aa), sin_approx(ab)));
                    er[h] = fma2(pi, VI, fma2(pr, VR, er[h]));
                    ei[h] = fma2(pi, NVR, fma2(pr, VI, ei[h]));
                }
            }
#pragma unroll
            for (int h = 0; h < kPairs; ++h) {
                float e0, e1, f0, f1;
                upk2(er[h], e0, e1);
                upk2(ei[h], f0, f1);
                two_sum_acc(sr[2 * h], cr[2 * h], e0);
                two_sum_acc(sr[2 * h + 1], cr[2 * h + 1], e1);
                two_sum_acc(si[2 * h], ci[2 * h], f0);
                two_sum_acc(si[2 * h + 1], ci[2 * h + 1], f1);
            }
        }
        if (!pipe.release(t, got)) return;
    }
#pragma unroll
    for (int q = 0; q < kAdjPPT32; ++q)
        if (j0 + q < npil)
            partial[(size_t)blockIdx.y * npil + j0 + q] =
                make_double2((double)sr[q] + (double)cr[q], (double)si[q] + (double)ci[q]);
}

// chunk sums of the precision-form adjoint, then the factor e^{-ikz} in FP64
__global__ void adj_f32c_reduce(const double2* __restrict__ partial, int nchunk, int n, double kz,
                                double2* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double r = 0.0, i = 0.0;
    for (int c = 0; c < nchunk; ++c) {
        const double2 v = partial[(size_t)c * n + j];
        r += v.x;
        i += v.y;
    }
    double sn, cs;
    sincos(kz, &sn, &cs);
    out[j] = make_double2(r * cs + i * sn, i * cs - r * sn);
}

// ---- chunk reduction + epilogue ---------------------------------------------
__global__ void rs_reduce_kernel(const double2* __restrict__ partial, int nchunk, Geom g,
                                 double k, int apply_phase, double2* __restrict__ field,
                                 double* __restrict__ intensity) {
    const int npix = g.nx * g.ny;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    double er = 0.0, ei = 0.0;
    for (int c = 0; c < nchunk; ++c) {
        const double2 v = partial[(size_t)c * npix + p];
        er += v.x;
        ei += v.y;
    }
    if (apply_phase) {
        const int j = p / g.nx;
        double fx, fy, fz;
        pixel_pos(g, 0, j, fx, fy, fz);
        // the FP32 terms hold the phase of R - z for z carried as a float pair
        // (the precision forward) or R - z_f, z_f = (float)z (the adjoint); the
        // global phase k z uses the FP64 z
        double s, c;
        sincos(k * fz, &s, &c);
        const double r = er * c - ei * s;
        ei = er * s + ei * c;
        er = r;
    }
    if (field) field[p] = make_double2(er, ei);
    if (intensity) intensity[p] = er * er + ei * ei;  // std::norm(E)
}

// ---- adjoint: out_j = sum_p conj(g_pj) v_p ----------------------------------
__global__ void __launch_bounds__(kThreads) rs_adj_f64_kernel(const double4* __restrict__ pix,
                                                              int npix, int chunk_len,
                                                              const double* __restrict__ px,
                                                              const double* __restrict__ py,
                                                              int npil, double z, double k, int slot,
                                                              double2* __restrict__ partial) {
    __shared__ __align__(128) double4 buf[kStages][kTile64];
    __shared__ __align__(8) uint64_t full[kStages];

    const int j0 = (blockIdx.x * kThreads + threadIdx.x) * kAdjPPT;
    double x[kAdjPPT], y[kAdjPPT];
#pragma unroll
    for (int q = 0; q < kAdjPPT; ++q) {
        const int jq = min(j0 + q, npil - 1);
        x[q] = px[jq];
        y[q] = py[jq];
    }
    const double z2 = z * z;

    TilePipe<double4, kTile64> pipe;
    const int lo = blockIdx.y * chunk_len;
    pipe.init(buf, full, pix, lo, min(npix, lo + chunk_len), slot);

    double gr[kAdjPPT], gi[kAdjPPT];
#pragma unroll
    for (int q = 0; q < kAdjPPT; ++q) gr[q] = gi[q] = 0.0;

    for (int t = 0; t < pipe.ntiles; ++t) {
        const bool got = pipe.wait(t);
        if (got) {
            const double4* tile = buf[t % kStages];
            const int cnt = pipe.count(t);
            for (int p = 0; p < cnt; ++p) {
                const double4 r = tile[p];  // {fx, fy, Re v, Im v}
#pragma unroll
                for (int q = 0; q < kAdjPPT; ++q) {
                    const double dx = r.x - x[q];
                    const double dy = r.y - y[q];
                    const double R = sqrt(dx * dx + dy * dy + z2);
                    double s, c;
                    sincos(k * R, &s, &c);
                    const double inv = 1.0 / R;
                    const double pr = inv * c, pim = inv * s;
                    gr[q] += pr * r.z + pim * r.w;  // conj(g) * v
                    gi[q] += pr * r.w - pim * r.z;
                }
            }
        }
        if (!pipe.release(t, got)) return;
    }
#pragma unroll
    for (int q = 0; q < kAdjPPT; ++q)
        if (j0 + q < npil)
            partial[(size_t)blockIdx.y * npil + j0 + q] = make_double2(gr[q], gi[q]);
}

__global__ void chunk_sum_kernel(const double2* __restrict__ partial, int nchunk, int n,
                                 double2* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double r = 0.0, i = 0.0;
    for (int c = 0; c < nchunk; ++c) {
        const double2 v = partial[(size_t)c * n + j];
        r += v.x;
        i += v.y;
    }
    out[j] = make_double2(r, i);
}

// ---- stated error of the precision form ------------------------------------------
// (1) Sampled: the field recomputed in FP64 at a set of pixels - a strided
//     lattice, the centre pixel and the 21 x 21 pixels around the peak of |E|
//     (where errors that add coherently are largest) - against the computed
//     field there.
// (2) Bound: an upper bound on max_p |E_p - E64_p| from the error model of the
//     precision-form arithmetic (ff_bound_kernel).
constexpr int kPeakHalf = 10;  // the peak neighbourhood is (2 kPeakHalf + 1)^2 pixels

// acc[0]: bits of max_p |E_p| (FP64); acc[1]: (bits of (float)|E_p| << 32) | p,
// so that atomicMax leaves the index of a peak pixel in the low word.
__global__ void abs_max_kernel(const double2* __restrict__ field, int npix,
                               unsigned long long* __restrict__ acc) {
    double m = 0.0;
    unsigned long long arg = 0ull;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const double2 v = field[p];
        const double a = hypot(v.x, v.y);
        m = fmax(m, a);
        const unsigned long long key =
            ((unsigned long long)__float_as_uint((float)a) << 32) | (unsigned long long)(unsigned)p;
        arg = key > arg ? key : arg;
    }
    for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        const unsigned long long other = __shfl_down_sync(0xffffffffu, arg, o);
        arg = other > arg ? other : arg;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(acc + 0, (unsigned long long)__double_as_longlong(m));
        atomicMax(acc + 1, arg);
    }
}

// One block per sampled pixel: blocks [0, ns) take idx[b]; blocks [ns, ns +
// (2 kPeakHalf + 1)^2) the neighbourhood of the peak pixel found by
// abs_max_kernel (clamped to the grid). acc[2] receives the bits of max |E - E64|.
__global__ void rs_check_kernel(const double4* __restrict__ rec, int npil, Geom g, double k,
                                const double2* __restrict__ field, const int* __restrict__ idx,
                                int ns, unsigned long long* __restrict__ acc) {
    __shared__ double red[2][32];
    const int b = blockIdx.x;
    const int npix = g.nx * g.ny;
    int p;
    if (b < ns) {
        p = idx[b];
    } else {
        const int q = b - ns, side = 2 * kPeakHalf + 1;
        const int peak = (int)(unsigned)(acc[1] & 0xffffffffull);
        const int pj = peak / g.nx, pi = peak - pj * g.nx;
        const int i = min(max(pi + q % side - kPeakHalf, 0), g.nx - 1);
        const int j = min(max(pj + q / side - kPeakHalf, 0), g.ny - 1);
        p = j * g.nx + i;
    }
    if (p < 0 || p >= npix) return;
    const int j = p / g.nx, i = p - j * g.nx;
    double fx, fy, fz;
    pixel_pos(g, i, j, fx, fy, fz);
    const double z2 = fz * fz;
    double er = 0.0, ei = 0.0;
    for (int q = threadIdx.x; q < npil; q += blockDim.x) {
        const double4 r = rec[q];
        const double dx = fx - r.x, dy = fy - r.y;
        const double R = sqrt(dx * dx + dy * dy + z2);
        double s, c;
        sincos(k * R, &s, &c);
        const double inv = 1.0 / R;
        er += r.z * inv * c - r.w * inv * s;
        ei += r.z * inv * s + r.w * inv * c;
    }
    for (int o = 16; o > 0; o >>= 1) {
        er += __shfl_down_sync(0xffffffffu, er, o);
        ei += __shfl_down_sync(0xffffffffu, ei, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        red[0][w] = er;
        red[1][w] = ei;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sr = 0.0, si = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            sr += red[0][q];
            si += red[1][q];
        }
        const double2 f = field[p];
        const double err = hypot(f.x - sr, f.y - si);
        atomicMax(acc + 2, (unsigned long long)__double_as_longlong(err));
    }
}

// Error model of one precision-form term (rs_f32c_kernel), per pillar j, for
// every pixel of the window. u = 2^-24 (FP32 round to nearest), G the pixel
// grid step (grid_step), cmax = G/2 + 5 pixel steps the largest offset of a
// pixel from its thread's base. With the pillar's offset (xo, yo) from the
// FP32 origin and the window's largest pixel offset w, dxm = xo + w and dym =
// yo + w bound |dx|, |dy|, rho^2 <= dxm^2 + dym^2 and delta = R - z <= dmax.
// Random part (roundings whose error depends on each pillar's own data): the
// FP32 rounding of the pillar's x, y (u xo, u yo) and of base - x, fy - y
// (which can only drop bits of x, y: u dxm, u dym) moves rho^2 by at most
// 4u (dxm^2 + dym^2), its assembly rounds by at most 4u (dxm^2 + dym^2) more;
// R - z moves by that / (2|z|); the Newton step adds u dmax (1 + dmax / 2|z|)
// and the quadratic remainder of its seed (rsqrt.approx); the phase in turns
// th = d hi + (d lo + psi) rounds with u (dmax/lambda + 1/2) plus u for psi and
// the inner sum (its low bits come from d, i.e. from the pillar's own R - z),
// the reduced angle with u pi; the amplitude |t|/R rounds with 6u:
//   e_R(j)  = 2 pi (dDelta/lambda + u (dmax/lambda + 1/2) + u) + u pi + 6u
// Systematic part (the same for many pillars, so it can add up coherently near
// a focus where the phases of all terms agree), summed without cancellation:
// the MUFU approximations, the 2 pi_f constant (|2 pi_f - 2 pi| / 2 on a
// fraction <= 1/2), the FP32 rounding of the pixel's offsets (u cmax in x, u G
// in y: a shift of the pixel), and what is left of the rounding of z once it is
// carried as a float pair z_f + z_l (dz = |z - z_f - z_l|, ~u^2 |z|):
//   e_D(j)  = kRsqrtRelErr + sqrt(2) kSinCosAbsErr + |2 pi_f - 2 pi| / 2
//             + k u (cmax dxm + G dym) / |z| + dz / |z| + k dz rho_max^2 / (2 z^2)
// Every term has magnitude a_j = |t_j| / R <= |t_j| / |z|. acc (doubles):
// [0] sum_j a_j e_D(j), [1] sum_j (a_j e_R(j))^2, [2] bits of max_j a_j,
// [3] sum_j a_j; ext: the coordinate extent word of ff_extent_kernel.
__global__ void ff_bound_kernel(const double* __restrict__ px, const double* __restrict__ py,
                                const double2* __restrict__ pt, int npil, Geom g, double k,
                                const unsigned long long* __restrict__ ext, double wmax,
                                double* __restrict__ acc) {
    const double u = 5.9604644775390625e-08;  // 2^-24
    const double pi = 3.14159265358979323846;
    // the terms use z as the float pair z_f + z_l; what remains of its rounding
    const double zf = (double)(float)g.z, zl = (double)(float)(g.z - zf);
    const double z = fabs(g.z), dz = fabs(g.z - zf - zl);
    const double lam = 2.0 * pi / k;
    const double G = ext_grid(ext, wmax);
    const double pstep = g.mode == GEOM_PSF ? fabs(g.a1) : fabs(g.a1 - g.a0) / fmax(1.0, (double)(g.nx - 1));
    const double cmax = 0.5 * G + (kPPT32 - 1) * pstep;
    const double two_pi_f = (double)6.28318530717958647692f;
    const double eD0 = celeris_dev::kRsqrtRelErr + 1.4142135623730951 * celeris_dev::kSinCosAbsErr +
                       0.5 * fabs(two_pi_f - 2.0 * pi) + dz / z;
    double sD = 0.0, sR = 0.0, sA = 0.0, amax = 0.0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npil; j += gridDim.x * blockDim.x) {
        const double2 t = pt[j];
        const double a = hypot(t.x, t.y) / z;
        const double dxm = fabs(px[j] - g.ox) + wmax, dym = fabs(py[j] - g.oy) + wmax;
        const double rho2 = dxm * dxm + dym * dym;
        const double R = sqrt(rho2 + z * z);
        const double dmax = rho2 / (R + z);
        const double seed = R * (celeris_dev::kRsqrtRelErr + 4.0 * u);
        const double dDelta = 8.0 * u * rho2 / (2.0 * z) + u * dmax * (1.0 + dmax / (2.0 * z)) + seed * seed / z;
        const double eR = 2.0 * pi * (dDelta / lam + u * (dmax / lam + 0.5) + u) + u * pi + 6.0 * u;
        const double eD = eD0 + k * u * (cmax * dxm + G * dym) / z + k * dz * rho2 / (2.0 * z * z);
        sD += a * eD;
        sR += (a * eR) * (a * eR);
        sA += a;
        amax = fmax(amax, a);
    }
    for (int o = 16; o > 0; o >>= 1) {
        sD += __shfl_down_sync(0xffffffffu, sD, o);
        sR += __shfl_down_sync(0xffffffffu, sR, o);
        sA += __shfl_down_sync(0xffffffffu, sA, o);
        amax = fmax(amax, __shfl_down_sync(0xffffffffu, amax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc + 0, sD);
        atomicAdd(acc + 1, sR);
        atomicMax(reinterpret_cast<unsigned long long*>(acc + 2), (unsigned long long)__double_as_longlong(amax));
        atomicAdd(acc + 3, sA);
    }
}

// Failure-path self-test of the bounded device waits: one warp arms an
// mbarrier that expects two arrivals, arrives once, and waits on it with the
// same bounded poll loop the tile pipeline uses, limited to `polls`. Nothing
// else arrives and no copy is issued, so the wait always runs out; the kernel
// records the timeout in the stream's status word (the path a stalled TMA tile
// takes) and returns.
__global__ void ff_wait_selftest_kernel(unsigned polls, int slot) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 2);
        fence_barrier_init();
        mbar_arrive(&bar);
    }
    __syncwarp();
    const bool done = mbar_wait(&bar, 0, polls);
    if (!__all_sync(0xffffffffu, done) && threadIdx.x == 0) record_timeout(slot);
}

// ---- host-side planning -----------------------------------------------------
int g_sm_count = 0;

int sm_count() {
    if (g_sm_count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (g_sm_count <= 0) g_sm_count = 148;
    }
    return g_sm_count;
}

// Split the pillar (or pixel) axis into chunks so the grid holds about eight
// CTAs per SM-slot while every chunk keeps whole tiles.
void plan_chunks(int ctas_other, int nrec, int tile, int resident_per_sm, int* nchunk,
                 int* chunk_len) {
    const int ntiles = std::max(1, (nrec + tile - 1) / tile);
    const long slots = (long)sm_count() * resident_per_sm;  // CTAs resident at once
    const long target = slots * 8;
    long want = (target + ctas_other - 1) / std::max(1, ctas_other);
    want = std::max(1L, std::min<long>(want, ntiles));
    // Among want .. 2 want chunks pick the count whose grid fills its last wave
    // of resident CTAs best (CTAs of one launch take about equally long).
    long best_c = want;
    double best_fill = -1.0;
    for (long c = want; c <= std::min<long>(2 * want, ntiles); ++c) {
        const int tiles_per = (int)((ntiles + c - 1) / c);
        const long chunks = (ntiles + tiles_per - 1) / tiles_per;
        const double waves = (double)(ctas_other * chunks) / (double)slots;
        const double fill = waves / std::ceil(waves);
        if (fill > best_fill + 1e-9) {
            best_fill = fill;
            best_c = c;
        }
    }
    const int tiles_per = (int)((ntiles + best_c - 1) / best_c);
    *chunk_len = tiles_per * tile;
    *nchunk = (nrec + *chunk_len - 1) / *chunk_len;
    if (*nchunk < 1) *nchunk = 1;
}

// Status word of a stream: the legacy default stream in slot 0, other streams
// hashed over the remaining slots.
int status_slot(cudaStream_t st) {
    if (!st) return 0;
    const uint64_t h = (uint64_t)(uintptr_t)st * 0x9E3779B97F4A7C15ull;
    return 1 + (int)((h >> 33) % (uint64_t)(kStatusSlots - 1));
}

// Read and clear the status word of `st` (the stream's work must be complete).
int check_status_and_reset(cudaStream_t stream) {
    const size_t off = sizeof(int) * (size_t)status_slot(stream);
    int st = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&st, g_ff_status, sizeof(int), off);
    if (e != cudaSuccess) return celeris_rt::cuda_error(e, "read far-field status");
    if (st != 0) {
        int zero = 0;
        cudaMemcpyToSymbol(g_ff_status, &zero, sizeof(int), off);
        if (st & kFlagTimeout)
            return set_error(CELERIS_ERR_DEVICE_TIMEOUT, "far-field kernel: a bounded device wait ran out");
        return set_error(CELERIS_ERR_INVALID_ARG,
                         "far-field input holds NaN or Inf (pillar positions / transmissions, or the adjoint's "
                         "pixel values); the outputs hold non-finite values where it reached them");
    }
    return CELERIS_OK;
}

Geom psf_geom(double cx, double cy, double z, int n, double W) {
    Geom g;
    g.mode = GEOM_PSF;
    g.nx = g.ny = n;
    const double step = 2.0 * W / (n - 1);  // focal.cpp:223 (n == 1 gives inf, as the reference)
    g.a0 = cx - W;
    g.a1 = step;
    g.b0 = cy - W;
    g.b1 = step;
    g.z = z;
    g.ox = cx;
    g.oy = cy;
    g.row0 = 0;
    g.slot = 0;
    return g;
}

// Rows [row0, row0 + nrows) of the n x n grid of psf_geom (the same pixel
// positions and the same FP32 origin), for a focal grid split by rows.
Geom psf_rows_geom(double cx, double cy, double z, int n, double W, int row0, int nrows) {
    Geom g = psf_geom(cx, cy, z, n, W);
    g.ny = nrows;
    g.row0 = row0;
    return g;
}

Geom zx_geom(double xmin, double xmax, int nx, double zmin, double zmax, int nz) {
    Geom g;
    g.mode = GEOM_ZX;
    g.nx = nx;
    g.ny = nz;
    g.a0 = xmin;
    g.a1 = xmax;
    g.b0 = zmin;
    g.b1 = zmax;
    g.z = 0.0;
    g.ox = 0.0;
    g.oy = 0.0;
    g.row0 = 0;
    g.slot = 0;
    return g;
}

// Largest pixel offset from the FP32 origin over the grid (either axis).
double window_extent(const Geom& g) {
    if (g.mode == GEOM_ZX) return std::max(std::fabs(g.a0), std::fabs(g.a1));  // x only; y = 0
    const double x0 = g.a0 - g.ox, x1 = g.a0 + (g.nx - 1) * g.a1 - g.ox;
    const double y0 = g.b0 + g.row0 * g.b1 - g.oy, y1 = g.b0 + (g.row0 + g.ny - 1) * g.b1 - g.oy;
    return std::max(std::max(std::fabs(x0), std::fabs(x1)), std::max(std::fabs(y0), std::fabs(y1)));
}

// Whether z needs its FP32 lo part (z not exactly a float): every row of a
// PSF grid shares z; a ZX grid's rows differ and always carry it.
bool needs_zlo(const Geom& g) { return g.mode == GEOM_ZX || (double)(float)g.z != g.z; }

// The precision-form kernel launch (the two z variants).
void launch_f32c(dim3 grid, cudaStream_t st, const float4* rec, int npil, int chunk_len, const Geom& g, float hi,
                 float lo, const unsigned long long* ext, double wmax, double2* partial) {
    if (needs_zlo(g))
        rs_f32c_kernel<true><<<grid, kThreads, 0, st>>>(rec, npil, chunk_len, g, hi, lo, ext, wmax, partial);
    else
        rs_f32c_kernel<false><<<grid, kThreads, 0, st>>>(rec, npil, chunk_len, g, hi, lo, ext, wmax, partial);
}

// Optional CUDA-event timing of the main kernel (bench instrumentation).
std::atomic<int> g_time_kernels{0};
struct KernelTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    bool pending = false;
    ~KernelTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        cudaGetLastError();
    }
};
thread_local KernelTimer t_timer;

void timer_begin(cudaStream_t st) {
    if (!g_time_kernels.load()) return;
    if (!t_timer.a) {
        cudaEventCreate(&t_timer.a);
        cudaEventCreate(&t_timer.b);
    }
    cudaEventRecord(t_timer.a, st);
}
void timer_end(cudaStream_t st) {
    if (!g_time_kernels.load()) return;
    cudaEventRecord(t_timer.b, st);
    t_timer.pending = true;
}

// Full far-field on device buffers (inputs SoA px, py + interleaved complex pt).
int ff_run(int form, const double* d_px, const double* d_py, const double* d_pt, int npil,
           const Geom& g0, double k, double* d_field, double* d_int, cudaStream_t st) {
    Geom g = g0;
    g.slot = status_slot(st);
    const long npix = (long)g.nx * g.ny;
    if (npix <= 0) return CELERIS_OK;
    if (npix > (1L << 30)) return set_error(CELERIS_ERR_TOO_LARGE, "grid too large (%ld pixels)", npix);
    if (npil == 0) {
        if (d_field) CEL_CUDA(cudaMemsetAsync(d_field, 0, npix * 2 * sizeof(double), st));
        if (d_int) CEL_CUDA(cudaMemsetAsync(d_int, 0, npix * sizeof(double), st));
        return CELERIS_OK;
    }
    const bool f32 = (form == CELERIS_FORM_F32C);
    const int ppt = f32 ? kPPT32 : kPPT64;
    const int tile = f32 ? kTile32 : kTile64;
    const long spr = (g.nx + ppt - 1) / ppt;
    const long strips = spr * g.ny;
    const int ctas_pix = (int)((strips + kThreads - 1) / kThreads);
    int nchunk = 1, chunk_len = npil;
    plan_chunks(ctas_pix, npil, tile, f32 ? 3 : 2, &nchunk, &chunk_len);

    Workspace& ws = Workspace::for_stream(st);
    const size_t rec_bytes = (size_t)npil * (f32 ? sizeof(float4) : sizeof(double4));
    const size_t part_bytes = (size_t)nchunk * npix * sizeof(double2);
    CEL_TRY(ws.reserve(st, celeris_rt::align256(rec_bytes) + celeris_rt::align256(part_bytes) + 256));
    void* rec = ws.take(rec_bytes);
    double2* partial = static_cast<double2*>(ws.take(part_bytes));
    unsigned long long* ext = static_cast<unsigned long long*>(ws.take(sizeof(unsigned long long)));
    const double wmax = window_extent(g);

    const int pb = (npil + 255) / 256;
    if (f32) {
        CEL_CUDA(cudaMemsetAsync(ext, 0, sizeof(unsigned long long), st));
        ff_extent_kernel<<<std::min(pb, 4 * sm_count()), 256, 0, st>>>(d_px, d_py, npil, g.ox, g.oy, ext);
        ff_pack_f32<<<pb, 256, 0, st>>>(d_px, d_py, reinterpret_cast<const double2*>(d_pt), npil,
                                        g.ox, g.oy, g.slot, static_cast<float4*>(rec));
        count_launch(1);
    } else {
        ff_pack_f64<<<pb, 256, 0, st>>>(d_px, d_py, reinterpret_cast<const double2*>(d_pt), npil,
                                        g.slot, static_cast<double4*>(rec));
    }
    dim3 grid(ctas_pix, nchunk);
    timer_begin(st);
    if (f32) {
        const double il = k / (2.0 * 3.14159265358979323846);  // 1/lambda in turns per micron
        const float hi = (float)il;
        const float lo = (float)(il - (double)hi);
        launch_f32c(grid, st, static_cast<const float4*>(rec), npil, chunk_len, g, hi, lo, ext, wmax, partial);
    } else {
        rs_f64_kernel<<<grid, kThreads, 0, st>>>(static_cast<const double4*>(rec), npil,
                                                 chunk_len, g, k, partial);
    }
    timer_end(st);
    rs_reduce_kernel<<<(int)((npix + 255) / 256), 256, 0, st>>>(
        partial, nchunk, g, k, f32 ? 1 : 0, reinterpret_cast<double2*>(d_field), d_int);
    count_launch(3);
    CEL_CUDA(cudaGetLastError());
    return CELERIS_OK;
}

int ff_adjoint(const double* d_px, const double* d_py, int npil, const Geom& g0, double k,
               const double* d_v, double* d_out, cudaStream_t st, int form = CELERIS_FORM_PLAIN_F64) {
    Geom g = g0;
    g.slot = status_slot(st);
    const long npix = (long)g.nx * g.ny;
    if (npil <= 0) return CELERIS_OK;
    if (npix <= 0) {
        CEL_CUDA(cudaMemsetAsync(d_out, 0, (size_t)npil * 2 * sizeof(double), st));
        return CELERIS_OK;
    }
    if (form == CELERIS_FORM_F32C) {
        const int ctas = (int)(((long)npil + kThreads * kAdjPPT32 - 1) / (kThreads * kAdjPPT32));
        int nchunk = 1, chunk_len = (int)npix;
        plan_chunks(ctas, (int)npix, kTile32, 3, &nchunk, &chunk_len);
        Workspace& ws = Workspace::for_stream(st);
        const size_t rec_bytes = (size_t)npix * sizeof(float4);
        const size_t part_bytes = (size_t)nchunk * npil * sizeof(double2);
        CEL_TRY(ws.reserve(st, celeris_rt::align256(rec_bytes) + celeris_rt::align256(part_bytes)));
        float4* rec = static_cast<float4*>(ws.take(rec_bytes));
        double2* partial = static_cast<double2*>(ws.take(part_bytes));
        ff_pack_pix_f32<<<(int)((npix + 255) / 256), 256, 0, st>>>(g, reinterpret_cast<const double2*>(d_v), rec);
        const double il = k / (2.0 * 3.14159265358979323846);
        const float hi = (float)il, lo = (float)(il - (double)hi);
        const float zf = (float)g.z;
        dim3 grid(ctas, nchunk);
        timer_begin(st);
        rs_adj_f32c_kernel<<<grid, kThreads, 0, st>>>(rec, (int)npix, chunk_len, d_px, d_py, npil, g, zf, hi, lo,
                                                      partial);
        timer_end(st);
        adj_f32c_reduce<<<(npil + 255) / 256, 256, 0, st>>>(partial, nchunk, npil, k * g.z,
                                                           reinterpret_cast<double2*>(d_out));
        count_launch(3);
        CEL_CUDA(cudaGetLastError());
        return CELERIS_OK;
    }
    const int ctas = (int)(((long)npil + kThreads * kAdjPPT - 1) / (kThreads * kAdjPPT));
    int nchunk = 1, chunk_len = (int)npix;
    plan_chunks(ctas, (int)npix, kTile64, 2, &nchunk, &chunk_len);
    Workspace& ws = Workspace::for_stream(st);
    const size_t rec_bytes = (size_t)npix * sizeof(double4);
    const size_t part_bytes = (size_t)nchunk * npil * sizeof(double2);
    CEL_TRY(ws.reserve(st, celeris_rt::align256(rec_bytes) + celeris_rt::align256(part_bytes)));
    double4* rec = static_cast<double4*>(ws.take(rec_bytes));
    double2* partial = static_cast<double2*>(ws.take(part_bytes));
    ff_pack_pix<<<(int)((npix + 255) / 256), 256, 0, st>>>(g, reinterpret_cast<const double2*>(d_v), rec);
    dim3 grid(ctas, nchunk);
    timer_begin(st);
    rs_adj_f64_kernel<<<grid, kThreads, 0, st>>>(rec, (int)npix, chunk_len, d_px, d_py, npil, g.z, k, g.slot,
                                                 partial);
    timer_end(st);
    chunk_sum_kernel<<<(npil + 255) / 256, 256, 0, st>>>(partial, nchunk, npil,
                                                         reinterpret_cast<double2*>(d_out));
    count_launch(3);
    CEL_CUDA(cudaGetLastError());
    return CELERIS_OK;
}

// Accumulator words of the stated-error evaluation (device and host copies):
// [0] bits of max |E|, [1] peak key, [2] bits of max sampled |E - E64|,
// [3..6] the sums of ff_bound_kernel, [7] the coordinate extent.
constexpr int kAccWords = 8;

// Enqueue the stated-error evaluation of the field d_field on st: the sampled
// FP64 check when ns > 0 (d_idx: ns pixel indices; the peak neighbourhood is
// added) and the model bound when want_bound. When st reaches the end, h_acc
// (host memory, kAccWords words; pinned keeps the copy asynchronous) holds the
// accumulators.
int ff_check_enqueue(const double* d_px, const double* d_py, const double* d_pt, int npil, const Geom& g0,
                     double k, const double* d_field, const int* d_idx, int ns, bool want_bound,
                     unsigned long long* h_acc, cudaStream_t st) {
    Geom g = g0;
    g.slot = status_slot(st);
    const long npix = (long)g.nx * g.ny;
    Workspace& ws = Workspace::for_stream(st);
    const size_t rec_bytes = ns > 0 ? (size_t)npil * sizeof(double4) : 0;
    CEL_TRY(ws.reserve(st, celeris_rt::align256(rec_bytes) + 256));
    double4* rec = static_cast<double4*>(ws.take(rec_bytes));
    unsigned long long* acc = static_cast<unsigned long long*>(ws.take(kAccWords * sizeof(unsigned long long)));
    CEL_CUDA(cudaMemsetAsync(acc, 0, kAccWords * sizeof(unsigned long long), st));
    abs_max_kernel<<<4 * sm_count(), 256, 0, st>>>(reinterpret_cast<const double2*>(d_field), (int)npix, acc);
    int launches = 1;
    if (ns > 0) {
        ff_pack_f64<<<(npil + 255) / 256, 256, 0, st>>>(d_px, d_py, reinterpret_cast<const double2*>(d_pt), npil,
                                                        g.slot, rec);
        const int side = 2 * kPeakHalf + 1;
        rs_check_kernel<<<ns + side * side, 256, 0, st>>>(rec, npil, g, k, reinterpret_cast<const double2*>(d_field),
                                                          d_idx, ns, acc);
        launches += 2;
    }
    if (want_bound) {
        const double wmax = window_extent(g);
        ff_extent_kernel<<<2 * sm_count(), 256, 0, st>>>(d_px, d_py, npil, g.ox, g.oy, acc + 7);
        ff_bound_kernel<<<2 * sm_count(), 256, 0, st>>>(d_px, d_py, reinterpret_cast<const double2*>(d_pt), npil, g,
                                                        k, acc + 7, wmax, reinterpret_cast<double*>(acc + 3));
        launches += 2;
    }
    count_launch(launches);
    CEL_CUDA(cudaGetLastError());
    CEL_CUDA(cudaMemcpyAsync(h_acc, acc, kAccWords * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    return CELERIS_OK;
}

double acc_double(const unsigned long long* h, int i) {
    double v;
    std::memcpy(&v, &h[i], sizeof(double));
    return v;
}

// The sampled error from the accumulators: max sampled |E - E64| / max |E|.
double check_ratio(const unsigned long long* h) {
    const double e = acc_double(h, 2), m = acc_double(h, 0);
    return m > 0.0 ? e / m : e;
}

// The stated bound from the accumulators, relative to max |E|:
//   B = sum_j a_j e_D(j)                                   (systematic parts)
//     + sqrt(2) lambda sqrt(sum_j (a_j e_R(j))^2 + T (u a_max C)^2)
//     + sum_j a_j ((u T)^2 + 64 eps64)
// The middle line bounds the FP32 rounding errors, modelled as independent and
// mean zero (the probabilistic rounding-error analysis of Higham and Mary,
// SIAM J. Sci. Comput. 41 (2019)): per component, a sum of independent terms
// bounded by c_i exceeds lambda sqrt(sum c_i^2) with probability at most
// 2 exp(-lambda^2 / 2) (Hoeffding); lambda = 8 makes that 2.5e-14 per pixel and
// component. It holds the per-term rounding (e_R) and the FP32 accumulation of
// each tile of kTile32 terms (fma into a running sum: each step errs by at most
// u |S_k| <= u k a_max, so C = sqrt(sum_{k<=K} k^2), K = kTile32) over at most T
// = 2 ceil(npil / K) tiles per pixel. The last line covers the compensated
// (TwoSum) tile folding and the FP64 chunk sums and global phase.
double bound_ratio(const unsigned long long* h, int npil) {
    const double u = 5.9604644775390625e-08, eps64 = 1.1102230246251565e-16, lambda = 8.0;
    const double K = kTile32;
    const double C = std::sqrt(K * (K + 1.0) * (2.0 * K + 1.0) / 6.0);
    const double T = 2.0 * std::ceil((double)npil / K);
    const double sD = acc_double(h, 3), sR = acc_double(h, 4), amax = acc_double(h, 5), sA = acc_double(h, 6);
    const double rnd = std::sqrt(2.0) * lambda * std::sqrt(sR + T * (u * amax * C) * (u * amax * C));
    const double B = sD + rnd + sA * ((u * T) * (u * T) + 64.0 * eps64);
    const double m = acc_double(h, 0);
    return m > 0.0 ? B / m : B;
}

// Synchronous stated-error evaluation of a field on the device (sampled error
// and/or bound), on st.
int ff_stated(const double* d_px, const double* d_py, const double* d_pt, int npil, const Geom& g, double k,
              const double* d_field, const int* d_idx, int ns, double* err_out, double* bound_out,
              cudaStream_t st) {
    if (err_out) *err_out = 0.0;
    if (bound_out) *bound_out = 0.0;
    if (npil <= 0 || (long)g.nx * g.ny <= 0 || (ns <= 0 && !bound_out)) return CELERIS_OK;
    unsigned long long h[kAccWords] = {0};
    CEL_TRY(ff_check_enqueue(d_px, d_py, d_pt, npil, g, k, d_field, d_idx, err_out ? ns : 0, bound_out != nullptr,
                             h, st));
    CEL_CUDA(cudaStreamSynchronize(st));
    if (err_out) *err_out = check_ratio(h);
    if (bound_out) *bound_out = bound_ratio(h, npil);
    return check_status_and_reset(st);
}

// Non-blocking streams per host thread for the synchronous host-buffer calls:
// which = 0 carries the call, which = 1 the stated-error check beside it.
thread_local celeris_rt::ThreadStream t_streams[2];

int thread_stream(cudaStream_t* out, int which = 0) { return t_streams[which].get(out); }

// Per-thread events without timing, created on first use, destroyed with the
// thread (and when the thread moves to another device).
struct ThreadEvents {
    std::vector<cudaEvent_t> ev;
    int dev = -1;
    void clear() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        ev.clear();
        cudaGetLastError();
    }
    ~ThreadEvents() { clear(); }
};
thread_local ThreadEvents t_events;

cudaEvent_t thread_event(size_t i) {
    int cur = 0;
    cudaGetDevice(&cur);
    if (t_events.dev != cur) {
        t_events.clear();
        t_events.dev = cur;
    }
    while (t_events.ev.size() <= i) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
        t_events.ev.push_back(e);
    }
    return t_events.ev[i];
}

// Device I/O buffers of the host-buffer calls, one per thread (separate from
// the scratch arena the kernels use on the same stream); freed with the thread.
struct ThreadIo {
    void* p = nullptr;
    size_t cap = 0;
    int dev = -1;
    void release() {
        if (p) {
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(dev);
            cudaFree(p);
            cudaSetDevice(cur);
            cudaGetLastError();
        }
        p = nullptr;
        cap = 0;
        dev = -1;
    }
    ~ThreadIo() { release(); }
};
thread_local ThreadIo t_io;

// Host <-> device copies through pinned staging go in pieces of this size, so
// the host copy of one piece overlaps the transfer of the next.
constexpr size_t kPiece = (size_t)4 << 20;

// D2H of `bytes` from src into the caller's dst through pinned `stage`
// (per-thread events 1, 2, ...).
int download(void* dst, char* stage, const void* src, size_t bytes, cudaStream_t st) {
    if (!dst || bytes == 0) return CELERIS_OK;
    const size_t np = (bytes + kPiece - 1) / kPiece;
    for (size_t i = 0; i < np; ++i) {
        const size_t o = i * kPiece, b = std::min(kPiece, bytes - o);
        cudaEvent_t e = thread_event(1 + i);
        if (!e) return set_error(CELERIS_ERR_CUDA, "cudaEventCreate failed");
        CEL_CUDA(cudaMemcpyAsync(stage + o, static_cast<const char*>(src) + o, b, cudaMemcpyDeviceToHost, st));
        CEL_CUDA(cudaEventRecord(e, st));
    }
    for (size_t i = 0; i < np; ++i) {
        const size_t o = i * kPiece, b = std::min(kPiece, bytes - o);
        CEL_CUDA(cudaEventSynchronize(thread_event(1 + i)));
        std::memcpy(static_cast<char*>(dst) + o, stage + o, b);
    }
    return CELERIS_OK;
}

// Sample of pixel indices for the stated error: a side x side lattice spread
// over both axes of the grid, plus the centre pixel (the kernel adds the
// neighbourhood of the peak).
std::vector<int> sample_pixels(int nx, int ny, int side) {
    std::vector<int> idx;
    const long npix = (long)nx * ny;
    if (npix <= (long)side * side) {
        for (int p = 0; p < npix; ++p) idx.push_back(p);
        return idx;
    }
    for (int a = 0; a < side; ++a)
        for (int b = 0; b < side; ++b) {
            const int j = (int)(((long)(2 * a + 1) * ny) / (2 * side));
            const int i = (int)(((long)(2 * b + 1) * nx) / (2 * side));
            idx.push_back(j * nx + i);
        }
    idx.push_back((ny / 2) * nx + nx / 2);
    return idx;
}

// Host-buffer wrapper: stage inputs through pinned memory, run, copy back.
int ff_host(int form, const double* px, const double* py, const double* pt, int npil,
            const Geom& g, double k, double* field_out, double* int_out, double* err_out,
            double* bound_out = nullptr) {
    CEL_TRY(celeris_rt::require_device());
    const long npix = (long)g.nx * g.ny;
    if (err_out) *err_out = 0.0;
    if (bound_out) *bound_out = 0.0;
    if (npix <= 0) return CELERIS_OK;
    if (npil < 0) return set_error(CELERIS_ERR_INVALID_ARG, "npil < 0");
    if (npil > 0 && (!px || !py || !pt)) return set_error(CELERIS_ERR_INVALID_ARG, "NULL pillar arrays");
    cudaStream_t st = nullptr;
    CEL_TRY(thread_stream(&st));
    const bool want_err = (form == CELERIS_FORM_F32C) && err_out && npil > 0;
    const bool want_bound = (form == CELERIS_FORM_F32C) && bound_out && npil > 0;
    std::vector<int> sidx;
    if (want_err) sidx = sample_pixels(g.nx, g.ny, 16);

    const size_t in_bytes = (size_t)npil * 4 * sizeof(double);
    const size_t fld_bytes = (size_t)npix * 2 * sizeof(double);
    const size_t int_bytes = (size_t)npix * sizeof(double);
    const size_t idx_bytes = sidx.size() * sizeof(int);
    const size_t pin_bytes = celeris_rt::align256(in_bytes) + celeris_rt::align256(fld_bytes) +
                             celeris_rt::align256(int_bytes) + celeris_rt::align256(idx_bytes);
    // pinned: the device I/O layout, then the accumulator words of the error check
    char* pin = static_cast<char*>(celeris_rt::pinned_staging(pin_bytes + 256));
    if (!pin) return set_error(CELERIS_ERR_OOM, "pinned staging of %zu bytes failed", pin_bytes);

    int dev = 0;
    CEL_CUDA(cudaGetDevice(&dev));
    if (t_io.cap < pin_bytes || t_io.dev != dev) {
        CEL_CUDA(cudaStreamSynchronize(st));
        t_io.release();
        CEL_TRY(celeris_rt::device_alloc(&t_io.p, pin_bytes, "far-field I/O buffer"));
        t_io.cap = pin_bytes;
        t_io.dev = dev;
    }
    char* d = static_cast<char*>(t_io.p);
    double* d_px = reinterpret_cast<double*>(d);
    double* d_py = d_px + npil;
    double* d_pt = d_py + npil;
    double* d_fld = reinterpret_cast<double*>(d + celeris_rt::align256(in_bytes));
    double* d_int = reinterpret_cast<double*>(d + celeris_rt::align256(in_bytes) +
                                              celeris_rt::align256(fld_bytes));
    int* d_idx = reinterpret_cast<int*>(d + celeris_rt::align256(in_bytes) +
                                        celeris_rt::align256(fld_bytes) + celeris_rt::align256(int_bytes));
    if (npil > 0) {
        // px | py | pt, each piece sent while the next one is staged
        const char* src[3] = {reinterpret_cast<const char*>(px), reinterpret_cast<const char*>(py),
                              reinterpret_cast<const char*>(pt)};
        const size_t len[3] = {npil * sizeof(double), npil * sizeof(double), npil * 2 * sizeof(double)};
        size_t off = 0;
        for (int a = 0; a < 3; ++a) {
            for (size_t o = 0; o < len[a]; o += kPiece) {
                const size_t b = std::min(kPiece, len[a] - o);
                std::memcpy(pin + off + o, src[a] + o, b);
                CEL_CUDA(cudaMemcpyAsync(d + off + o, pin + off + o, b, cudaMemcpyHostToDevice, st));
            }
            off += len[a];
        }
    }
    if (want_err) {
        int* h_idx = reinterpret_cast<int*>(pin + celeris_rt::align256(in_bytes) +
                                            celeris_rt::align256(fld_bytes) + celeris_rt::align256(int_bytes));
        std::memcpy(h_idx, sidx.data(), idx_bytes);
        CEL_CUDA(cudaMemcpyAsync(d_idx, h_idx, idx_bytes, cudaMemcpyHostToDevice, st));
    }
    const bool need_field = field_out || want_err || want_bound;
    CEL_TRY(ff_run(form, d_px, d_py, d_pt, npil, g, k, need_field ? d_fld : nullptr,
                   int_out ? d_int : nullptr, st));
    char* h_fld = pin + celeris_rt::align256(in_bytes);
    char* h_int = h_fld + celeris_rt::align256(fld_bytes);
    unsigned long long* h_acc = reinterpret_cast<unsigned long long*>(pin + pin_bytes);
    // the stated-error evaluation runs on the second stream while the field downloads
    cudaStream_t st2 = nullptr;
    const bool stated = want_err || want_bound;
    if (stated) {
        CEL_TRY(thread_stream(&st2, 1));
        for (int i = 0; i < kAccWords; ++i) h_acc[i] = 0;
        cudaEvent_t done = thread_event(0);
        if (!done) return set_error(CELERIS_ERR_CUDA, "cudaEventCreate failed");
        CEL_CUDA(cudaEventRecord(done, st));
        CEL_CUDA(cudaStreamWaitEvent(st2, done, 0));
        CEL_TRY(ff_check_enqueue(d_px, d_py, d_pt, npil, g, k, d_fld, d_idx, want_err ? (int)sidx.size() : 0,
                                 want_bound, h_acc, st2));
    }
    const int rd = download(field_out, h_fld, d_fld, field_out ? fld_bytes : 0, st);
    const int ri = rd == CELERIS_OK ? download(int_out, h_int, d_int, int_out ? int_bytes : 0, st) : rd;
    cudaError_t e1 = cudaStreamSynchronize(st);
    cudaError_t e2 = stated ? cudaStreamSynchronize(st2) : cudaSuccess;
    CEL_TRY(ri);
    CEL_CUDA(e1);
    CEL_CUDA(e2);
    if (want_err) *err_out = check_ratio(h_acc);
    if (want_bound) *bound_out = bound_ratio(h_acc, npil);
    const int s1 = check_status_and_reset(st);
    const int s2 = stated ? check_status_and_reset(st2) : CELERIS_OK;
    return s1 != CELERIS_OK ? s1 : s2;
}

bool valid_form(int form) { return form == CELERIS_FORM_PLAIN_F64 || form == CELERIS_FORM_F32C; }

// ---- far-field without allocation ----------------------------------------------
// Scratch for callers that cannot allocate device memory: the pillar records
// and the per-chunk partial sums live in this fixed module-scope array. The
// CUDA runtime creates it on a device when it loads this file's module there -
// with lazy module loading (the default), at the first use of any far-field
// kernel or of the array on that device - and keeps it until the process exits.
// Host code must not pass the symbol itself to a kernel (on the host it names a
// shadow variable, not device memory); it passes the device address obtained
// with cudaGetSymbolAddress below.
constexpr size_t kNoAllocScratchBytes = (size_t)48 << 20;  // 48 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device; resolved on the
// first call per device (with that device current) and cached.
int noalloc_scratch(void** out) {
    int dev = 0;
    CEL_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(CELERIS_ERR_TOO_LARGE, "device index %d", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return celeris_rt::cuda_error(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return CELERIS_OK;
}

int ff_run_noalloc(int form, const double* d_px, const double* d_py, const double* d_pt, int npil, const Geom& g0,
                   double k, double* d_field, double* d_int, cudaStream_t st) {
    Geom g = g0;
    g.slot = status_slot(st);
    // Resolve the scratch first, so that a call with nothing to compute (n = 0
    // or no pillars) serves as the set-up call: it loads this module on the
    // device (creating the array) and caches the array's device address.
    void* base = nullptr;
    CEL_TRY(noalloc_scratch(&base));
    const long npix = (long)g.nx * g.ny;
    if (npix <= 0) return CELERIS_OK;
    if (npix > (1L << 30)) return set_error(CELERIS_ERR_TOO_LARGE, "grid too large (%ld pixels)", npix);
    if (npil == 0) {
        if (d_field) CEL_CUDA(cudaMemsetAsync(d_field, 0, npix * 2 * sizeof(double), st));
        if (d_int) CEL_CUDA(cudaMemsetAsync(d_int, 0, npix * sizeof(double), st));
        return CELERIS_OK;
    }
    const bool f32 = (form == CELERIS_FORM_F32C);
    const int ppt = f32 ? kPPT32 : kPPT64;
    const int tile = f32 ? kTile32 : kTile64;
    const long spr = (g.nx + ppt - 1) / ppt;
    const int ctas_pix = (int)((spr * g.ny + kThreads - 1) / kThreads);
    // scratch: pillar records | the coordinate extent word (256 B) | partial sums
    const size_t rec_bytes =
        celeris_rt::align256((size_t)npil * (f32 ? sizeof(float4) : sizeof(double4))) + 256;
    const size_t part_one = (size_t)npix * sizeof(double2);
    if (rec_bytes + part_one > kNoAllocScratchBytes)
        return set_error(CELERIS_ERR_TOO_LARGE,
                         "no-alloc far-field: %d pillars x %ld pixels need %zu bytes of scratch, limit %zu",
                         npil, npix, rec_bytes + part_one, kNoAllocScratchBytes);
    int nchunk = 1, chunk_len = npil;
    plan_chunks(ctas_pix, npil, tile, f32 ? 3 : 2, &nchunk, &chunk_len);
    // fewer chunks (longer ones) until the partial sums fit beside the records
    const int ntiles = (npil + tile - 1) / tile;
    while ((size_t)nchunk * part_one + rec_bytes > kNoAllocScratchBytes) {
        const int tiles_per = (chunk_len / tile) + 1;
        chunk_len = tiles_per * tile;
        nchunk = (ntiles + tiles_per - 1) / tiles_per;
    }
    void* rec = base;
    unsigned long long* ext = reinterpret_cast<unsigned long long*>(static_cast<char*>(base) + rec_bytes - 256);
    double2* partial = reinterpret_cast<double2*>(static_cast<char*>(base) + rec_bytes);
    const double wmax = window_extent(g);
    const int pb = (npil + 255) / 256;
    if (f32) {
        CEL_CUDA(cudaMemsetAsync(ext, 0, sizeof(unsigned long long), st));
        ff_extent_kernel<<<std::min(pb, 4 * sm_count()), 256, 0, st>>>(d_px, d_py, npil, g.ox, g.oy, ext);
        ff_pack_f32<<<pb, 256, 0, st>>>(d_px, d_py, reinterpret_cast<const double2*>(d_pt), npil, g.ox, g.oy,
                                        g.slot, static_cast<float4*>(rec));
        count_launch(1);
    } else
        ff_pack_f64<<<pb, 256, 0, st>>>(d_px, d_py, reinterpret_cast<const double2*>(d_pt), npil, g.slot,
                                        static_cast<double4*>(rec));
    dim3 grid(ctas_pix, nchunk);
    if (f32) {
        const double il = k / (2.0 * 3.14159265358979323846);
        const float hi = (float)il;
        const float lo = (float)(il - (double)hi);
        launch_f32c(grid, st, static_cast<const float4*>(rec), npil, chunk_len, g, hi, lo, ext, wmax, partial);
    } else {
        rs_f64_kernel<<<grid, kThreads, 0, st>>>(static_cast<const double4*>(rec), npil, chunk_len, g, k, partial);
    }
    rs_reduce_kernel<<<(int)((npix + 255) / 256), 256, 0, st>>>(partial, nchunk, g, k, f32 ? 1 : 0,
                                                                 reinterpret_cast<double2*>(d_field), d_int);
    count_launch(3);
    CEL_CUDA(cudaGetLastError());
    return CELERIS_OK;
}

}  // namespace

extern "C" {

int celeris_propagate_psf(const double* px, const double* py, const double* pt, int npil,
                          double cx, double cy, double z, double k, int n, double half_window,
                          double* out) {
    if (n < 0) return set_error(CELERIS_ERR_INVALID_ARG, "n < 0");
    if (n == 0) return CELERIS_OK;
    if (!out) return set_error(CELERIS_ERR_INVALID_ARG, "out is NULL");
    return ff_host(CELERIS_FORM_PLAIN_F64, px, py, pt, npil, psf_geom(cx, cy, z, n, half_window), k,
                   nullptr, out, nullptr);
}

int celeris_propagate_zx(const double* px, const double* py, const double* pt, int npil,
                         double xmin, double xmax, int nx, double zmin, double zmax, int nz,
                         double k, double* out) {
    if (nx <= 1 || nz <= 1) return set_error(CELERIS_ERR_INVALID_ARG, "nx, nz must be > 1");
    if (!out) return set_error(CELERIS_ERR_INVALID_ARG, "out is NULL");
    return ff_host(CELERIS_FORM_PLAIN_F64, px, py, pt, npil, zx_geom(xmin, xmax, nx, zmin, zmax, nz),
                   k, nullptr, out, nullptr);
}

int celeris_rs_field(int form, const double* px, const double* py, const double* pt, int npil,
                     double cx, double cy, double z, double k, int n, double half_window,
                     double* field_out, double* intensity_out, double* err_out) {
    if (!valid_form(form)) return set_error(CELERIS_ERR_INVALID_ARG, "unknown form %d", form);
    if (n < 0) return set_error(CELERIS_ERR_INVALID_ARG, "n < 0");
    if (n == 0) {
        if (err_out) *err_out = 0.0;
        return CELERIS_OK;
    }
    return ff_host(form, px, py, pt, npil, psf_geom(cx, cy, z, n, half_window), k, field_out,
                   intensity_out, err_out);
}

int celeris_rs_field_dev(int form, const double* d_px, const double* d_py, const double* d_pt,
                         int npil, double cx, double cy, double z, double k, int n,
                         double half_window, double* d_field, double* d_intensity, void* stream) {
    if (!valid_form(form)) return set_error(CELERIS_ERR_INVALID_ARG, "unknown form %d", form);
    if (n < 0 || npil < 0) return set_error(CELERIS_ERR_INVALID_ARG, "negative size");
    if (npil > 0 && (!d_px || !d_py || !d_pt)) return set_error(CELERIS_ERR_INVALID_ARG, "NULL pillar arrays");
    CEL_TRY(celeris_rt::require_device());
    return ff_run(form, d_px, d_py, d_pt, npil, psf_geom(cx, cy, z, n, half_window), k, d_field,
                  d_intensity, static_cast<cudaStream_t>(stream));
}

int celeris_rs_adjoint_dev(int form, const double* d_px, const double* d_py, int npil, double cx,
                           double cy, double z, double k, int n, double half_window,
                           const double* d_v, double* d_out, void* stream) {
    if (!valid_form(form)) return set_error(CELERIS_ERR_INVALID_ARG, "unknown form %d", form);
    if (n < 0 || npil < 0) return set_error(CELERIS_ERR_INVALID_ARG, "negative size");
    if (npil > 0 && (!d_px || !d_py || !d_out)) return set_error(CELERIS_ERR_INVALID_ARG, "NULL arrays");
    if ((long)n * n > 0 && !d_v) return set_error(CELERIS_ERR_INVALID_ARG, "d_v is NULL");
    CEL_TRY(celeris_rt::require_device());
    return ff_adjoint(d_px, d_py, npil, psf_geom(cx, cy, z, n, half_window), k, d_v, d_out,
                      static_cast<cudaStream_t>(stream), form);
}

int celeris_rs_check_dev(const double* d_px, const double* d_py, const double* d_pt, int npil,
                         double cx, double cy, double z, double k, int n, double half_window,
                         const double* d_field, const int* d_idx, int ns, double* err_out,
                         void* stream) {
    if (!err_out) return set_error(CELERIS_ERR_INVALID_ARG, "err_out is NULL");
    if (n < 0 || npil < 0 || ns < 0) return set_error(CELERIS_ERR_INVALID_ARG, "negative size");
    CEL_TRY(celeris_rt::require_device());
    return ff_stated(d_px, d_py, d_pt, npil, psf_geom(cx, cy, z, n, half_window), k, d_field, d_idx, ns, err_out,
                     nullptr, static_cast<cudaStream_t>(stream));
}

int celeris_rs_field_noalloc(int form, const double* d_px, const double* d_py, const double* d_pt, int npil,
                             double cx, double cy, double z, double k, int n, double half_window, double* d_field,
                             double* d_intensity, void* stream) {
    if (!valid_form(form)) return set_error(CELERIS_ERR_INVALID_ARG, "unknown form %d", form);
    if (n < 0 || npil < 0) return set_error(CELERIS_ERR_INVALID_ARG, "negative size");
    if (npil > 0 && (!d_px || !d_py || !d_pt)) return set_error(CELERIS_ERR_INVALID_ARG, "NULL pillar arrays");
    CEL_TRY(celeris_rt::require_device());
    return ff_run_noalloc(form, d_px, d_py, d_pt, npil, psf_geom(cx, cy, z, n, half_window), k, d_field,
                          d_intensity, static_cast<cudaStream_t>(stream));
}

int celeris_set_kernel_timing(int on) {
    g_time_kernels.store(on ? 1 : 0);
    return CELERIS_OK;
}

int celeris_last_kernel_ms(double* ms) {
    if (!ms) return set_error(CELERIS_ERR_INVALID_ARG, "ms is NULL");
    if (!t_timer.pending) return set_error(CELERIS_ERR_INVALID_ARG, "no timed kernel recorded");
    CEL_CUDA(cudaEventSynchronize(t_timer.b));
    float v = 0.f;
    CEL_CUDA(cudaEventElapsedTime(&v, t_timer.a, t_timer.b));
    *ms = v;
    return CELERIS_OK;
}

int celeris_sync_status(void* stream) {
    CEL_TRY(celeris_rt::require_device());
    CEL_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    return check_status_and_reset(static_cast<cudaStream_t>(stream));
}

int celeris_rs_field_bounded(int form, const double* px, const double* py, const double* pt, int npil, double cx,
                             double cy, double z, double k, int n, double half_window, double* field_out,
                             double* intensity_out, double* err_out, double* bound_out) {
    if (!valid_form(form)) return set_error(CELERIS_ERR_INVALID_ARG, "unknown form %d", form);
    if (n < 0) return set_error(CELERIS_ERR_INVALID_ARG, "n < 0");
    if (n == 0) {
        if (err_out) *err_out = 0.0;
        if (bound_out) *bound_out = 0.0;
        return CELERIS_OK;
    }
    return ff_host(form, px, py, pt, npil, psf_geom(cx, cy, z, n, half_window), k, field_out, intensity_out,
                   err_out, bound_out);
}

int celeris_rs_error_bound_dev(const double* d_px, const double* d_py, const double* d_pt, int npil, double cx,
                               double cy, double z, double k, int n, double half_window, const double* d_field,
                               double* bound_out, void* stream) {
    if (!bound_out) return set_error(CELERIS_ERR_INVALID_ARG, "bound_out is NULL");
    if (n < 0 || npil < 0) return set_error(CELERIS_ERR_INVALID_ARG, "negative size");
    if (npil > 0 && (!d_px || !d_py || !d_pt)) return set_error(CELERIS_ERR_INVALID_ARG, "NULL pillar arrays");
    if (n > 0 && !d_field) return set_error(CELERIS_ERR_INVALID_ARG, "d_field is NULL");
    CEL_TRY(celeris_rt::require_device());
    return ff_stated(d_px, d_py, d_pt, npil, psf_geom(cx, cy, z, n, half_window), k, d_field, nullptr, 0, nullptr,
                     bound_out, static_cast<cudaStream_t>(stream));
}

int celeris_rs_field_rows_dev(int form, const double* d_px, const double* d_py, const double* d_pt, int npil,
                              double cx, double cy, double z, double k, int n, double half_window, int row0,
                              int nrows, double* d_field, double* d_intensity, void* stream) {
    if (!valid_form(form)) return set_error(CELERIS_ERR_INVALID_ARG, "unknown form %d", form);
    if (n < 0 || npil < 0 || nrows < 0) return set_error(CELERIS_ERR_INVALID_ARG, "negative size");
    if (row0 < 0 || (long)row0 + nrows > (long)n)
        return set_error(CELERIS_ERR_INVALID_ARG, "rows [%d, %d) outside the %d-row grid", row0, row0 + nrows, n);
    if (npil > 0 && (!d_px || !d_py || !d_pt)) return set_error(CELERIS_ERR_INVALID_ARG, "NULL pillar arrays");
    CEL_TRY(celeris_rt::require_device());
    return ff_run(form, d_px, d_py, d_pt, npil, psf_rows_geom(cx, cy, z, n, half_window, row0, nrows), k,
                  d_field, d_intensity, static_cast<cudaStream_t>(stream));
}

int celeris_rs_adjoint_rows_dev(int form, const double* d_px, const double* d_py, int npil, double cx, double cy,
                                double z, double k, int n, double half_window, int row0, int nrows,
                                const double* d_v, double* d_out, void* stream) {
    if (!valid_form(form)) return set_error(CELERIS_ERR_INVALID_ARG, "unknown form %d", form);
    if (n < 0 || npil < 0 || nrows < 0) return set_error(CELERIS_ERR_INVALID_ARG, "negative size");
    if (row0 < 0 || (long)row0 + nrows > (long)n)
        return set_error(CELERIS_ERR_INVALID_ARG, "rows [%d, %d) outside the %d-row grid", row0, row0 + nrows, n);
    if (npil > 0 && (!d_px || !d_py || !d_out)) return set_error(CELERIS_ERR_INVALID_ARG, "NULL arrays");
    if ((long)n * nrows > 0 && !d_v) return set_error(CELERIS_ERR_INVALID_ARG, "d_v is NULL");
    CEL_TRY(celeris_rt::require_device());
    return ff_adjoint(d_px, d_py, npil, psf_rows_geom(cx, cy, z, n, half_window, row0, nrows), k, d_v, d_out,
                      static_cast<cudaStream_t>(stream), form);
}

int celeris_device_wait_selftest(unsigned polls) {
    CEL_TRY(celeris_rt::require_device());
    cudaStream_t st = nullptr;
    CEL_TRY(thread_stream(&st));
    const int slot = status_slot(st);
    ff_wait_selftest_kernel<<<1, 32, 0, st>>>(polls, slot);
    count_launch(1);
    CEL_CUDA(cudaGetLastError());
    CEL_CUDA(cudaStreamSynchronize(st));
    return check_status_and_reset(st);
}

}  // extern "C"
