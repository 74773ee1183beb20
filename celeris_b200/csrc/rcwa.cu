// Batched 2D vectorial RCWA on sm_100a (FP64 throughout).
//
// Reference: src/celeris/rcwa/rcwa2d.cpp:209-488 (solve_rcwa_2d), 147-205
// (shape_operators), 74-95 (rasterize_eps), src/celeris/design/metalens.cpp:
// 122-163 (library sweep), src/celeris/rcwa/eig.cpp (eig_general).
//
// One unit cell = one patterned layer between the incident and substrate
// half-spaces (the library-sweep stack). Cells are bucketed by (Mx, My, raster
// size); a bucket runs as a fixed sequence of kernels with one CTA per cell:
//   rcwa_fourier_rect / rcwa_fourier_laurent  eps operators (analytic Li rule,
//                 or 4x4-supersampled raster -> centred DFT -> Laurent Toeplitz)
//                 and Einv (LU inverse for the Laurent path)
//   rcwa_build_M  M = ep2 kp - kkT using the diagonal Kx, Ky (two N^3 GEMMs)
//   rcwa_hess     Householder reduction to Hessenberg form H = Q^H M Q (in
//                 shared memory for n <= 112, blocked compact-WY panels above)
//   rcwa_schur    multishift QR with aggressive early deflation: Schur form
//                 T = Z^H M Z (schur_aed.cuh)
//   rcwa_vec      triangular back substitution for the eigenvectors of T;
//                 W = Z X; q = branch(sqrt(lambda))
//   rcwa_smat1    A = kp W, T11/T12 of interface 0, S12 and u = T11^{-1} a0
//   rcwa_smat2    W^{-1}, A^{-1}, T11'/T12' of interface 1, B = T11' - D S12 T12',
//                 aN = B^{-1} D u, b0 = T12 u + S22 T12' aN
//   rcwa_epilogue Poynting flux and order-0 field for each requested excitation
// The algebra is that of the reference's grcwa recursion specialised to
// phi = I in the half-spaces and to the two excitation columns actually read
// (a0 has two non-zeros), so only 2 columns of the global S11/S21 are formed.
#include <cuda_runtime.h>
#include <math.h>

#include <cmath>

#include <algorithm>
#include <chrono>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "cblas_block.cuh"
#include "schur_aed.cuh"
#include "runtime.cuh"

namespace {

using namespace cb;
using celeris_rt::count_launch;
using celeris_rt::set_error;
using celeris_rt::Workspace;

constexpr double PI = 3.14159265358979323846;
constexpr int kRT = 256;            // threads per CTA
constexpr int kDbgSlots = 24;       // diagnostic counters per cell
constexpr int kSmemEigMaxN = 116;   // Hessenberg reduction in shared memory up to this n ((n^2 + 2n) 16 B <= 227 KB)

struct CellDev {
    double omega;  // k0 = 2 pi / lambda (c = 1 units, omega = k0)
    double px, py, h, theta;
    double fill_x, fill_y, shape_param, rot;
    cplx kx0, ky0;
    cplx eps_p, eps_b;
    cplx n_inc, n_sub;
    cplx ex0, ey0;  // excitation of result slot 0 (batch: X = (1, 0))
    int shape, nexc;
    int pad0, pad1;
};

struct Bucket {
    int Mx, My, N, n, ng, ncell;
    const CellDev* cells;
    cplx *H, *Z, *X, *W, *A, *T11, *T11lu, *T12, *S12;
    cplx *Einv, *Exx, *Eyy;
    cplx* q1;
    int* piv;
    cplx* vec;  // per cell [10n]: aN_X, aN_Y, b0_X, b0_Y | x [n x 2] | y [n x 2] | z [n x 2]
    int* info;
    celeris_rcwa_result* res;  // per cell: nexc results
    size_t s_nn, s_ns, s_NN, s_n;
    const cplx* phx;  // [(4Mx+1) x ng] centred DFT phase table (x)
    const cplx* phy;  // [(4My+1) x ng]
    long long* dbg;   // optional per-cell counters, kDbgSlots each (CELERIS_RCWA_STAGE_CLOCKS=1), else NULL
    double* ord;      // optional per-order efficiencies: per cell and excitation [N][2] = (de_t, de_r), else NULL
    // mirror-symmetric cells (sym != 0): the eigenproblem solved in its four
    // parity classes; size class k (0: classes (+,+) and (-,-), 1: (+,-) and
    // (-,+)) holds two m[k] x m[k] matrices per cell, matrix 2 cell + j
    int sym;         // 0: full path; 1: both excited classes; 2: also C4-symmetric (one class)
    int ncls, cls0;  // excited classes solved per cell (2, or 1 = class 1 only) and the first one
    double sym_tol;  // largest asymmetry of M (relative to max |M|) the class split accepts
    int m[2];
    cplx *sH[2], *sZ[2], *sX[2], *sW[2], *sA[2], *sq[2];
    int* sinfo[2];
    // S-matrix in the two excited classes, matrix 2 cell + c (c = 0: (+,+), the
    // Y excitation; c = 1: (-,-), the X excitation), order m[0]: layer kp,
    // incident diag(kz) kp^-1, substrate kp diag(1/kz), and the work matrices
    cplx *cKp, *cC0, *cKs, *cA, *cT11, *cT11lu, *cT12, *cS12, *cQ, *cSQ, *cCm, *cvec;
    int* cpiv;
};

__device__ __forceinline__ cplx* at(cplx* base, size_t stride, int c) { return base + stride * c; }

// Mirror-symmetric cells (Bucket::sym != 0): per-cell info code of a cell found
// not symmetric to the tolerance, which is solved again by the full path.
constexpr int kInfoAsym = 1 << 29;

// Parity classes under the two mirrors p -> -p, q -> -q.
// class c: 0 = (+,+), 1 = (-,-), 2 = (+,-), 3 = (-,+)
__host__ __device__ __forceinline__ int sym_class_a(int c) { return (c == 0 || c == 2) ? 1 : -1; }
__host__ __device__ __forceinline__ int sym_class_b(int c) { return (c == 0 || c == 3) ? 1 : -1; }
__host__ __device__ __forceinline__ int sym_count(int M, int parity) { return parity > 0 ? M + 1 : M; }

__device__ __forceinline__ void order_pq(const Bucket& b, int i, int& p, int& q) {
    const int ny = 2 * b.My + 1;
    p = i / ny - b.Mx;
    q = i % ny - b.My;
}
__device__ __forceinline__ cplx kx_of(const Bucket& b, const CellDev& c, int i) {
    int p, q;
    order_pq(b, i, p, q);
    return csub(c.kx0, C(2.0 * PI * (double)p / c.px, 0.0));  // rcwa2d.cpp:240
}
__device__ __forceinline__ cplx ky_of(const Bucket& b, const CellDev& c, int i) {
    int p, q;
    order_pq(b, i, p, q);
    return csub(c.ky0, C(2.0 * PI * (double)q / c.py, 0.0));  // rcwa2d.cpp:241
}
__device__ __forceinline__ double rect1d(int m, double fill) {
    return m == 0 ? fill : sin(PI * m * fill) / (PI * m);  // rcwa2d.cpp:108-110
}
// kz of a homogeneous region (rcwa2d.cpp:259-261): grazing guard, then branch
__device__ __forceinline__ cplx kz_uniform(cplx er, double omega, cplx kx, cplx ky) {
    cplx v = csub(csub(cscale(er, omega * omega), cmul(kx, kx)), cmul(ky, ky));
    cplx kz = csqrt_p(v);
    if (cabs(kz) < 1e-8) kz = C(0.0, 1e-8);
    if (kz.y < 0.0) kz = cneg(kz);
    return kz;
}
// kp block of a homogeneous region for order i (rcwa2d.cpp:265-269)
__device__ __forceinline__ void kp_uniform(cplx ier, double omega, cplx kx, cplx ky, cplx& a, cplx& b, cplx& c,
                                           cplx& d) {
    const cplx w2 = C(omega * omega, 0.0);
    a = csub(w2, cmul(ier, cmul(ky, ky)));
    b = cmul(ier, cmul(ky, kx));
    c = cmul(ier, cmul(kx, ky));
    d = csub(w2, cmul(ier, cmul(kx, kx)));
}

// ---- Fourier operators: analytic rectangle (Li inverse rule) ------------------
// dynamic smem: hx [nx*nx] | ax [nx*nx] | hy [ny*ny] | ay [ny*ny]
__global__ void __launch_bounds__(kRT) rcwa_fourier_rect(Bucket b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int pv[32];
    __shared__ RedScratch rs;
    const int cell = blockIdx.x;
    const CellDev c = b.cells[cell];
    const int nx = 2 * b.Mx + 1, ny = 2 * b.My + 1, N = b.N;
    cplx* hx = reinterpret_cast<cplx*>(smem);
    cplx* ax = hx + nx * nx;
    cplx* hy = ax + nx * nx;
    cplx* ay = hy + ny * ny;
    cplx* stg = ay + ny * ny;  // LU staging: 2 * max(nx, ny)
    const int tid = threadIdx.x, nt = blockDim.x;
    const cplx ep = c.eps_p, eb = c.eps_b;
    const cplx ipe = cinv(ep), ibe = cinv(eb);
    const cplx dI = csub(ipe, ibe);
    // Hx, Hy: in-band 1D reciprocal Toeplitz (rcwa2d.cpp:299-303, 317-321)
    for (int e = tid; e < nx * nx; e += nt) {
        const int a = e / nx, bb = e % nx;
        cplx v = cscale(dI, rect1d(a - bb, c.fill_x));
        if (a == bb) v = cadd(v, ibe);
        hx[e] = v;
        ax[e] = C(a == bb ? 1.0 : 0.0, 0.0);
    }
    for (int e = tid; e < ny * ny; e += nt) {
        const int a = e / ny, bb = e % ny;
        cplx v = cscale(dI, rect1d(a - bb, c.fill_y));
        if (a == bb) v = cadd(v, ibe);
        hy[e] = v;
        ay[e] = C(a == bb ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    blk_lu(nx, hx, nx, pv, &rs, stg);
    blk_lu_solve(nx, hx, nx, pv, nx, ax, nx, stg);  // ax = Hx^{-1}
    blk_lu(ny, hy, ny, pv, &rs, stg);
    blk_lu_solve(ny, hy, ny, pv, ny, ay, ny, stg);  // ay = Hy^{-1}
    cplx* Einv = at(b.Einv, b.s_NN, cell);
    cplx* Exx = at(b.Exx, b.s_NN, cell);
    cplx* Eyy = at(b.Eyy, b.s_NN, cell);
    for (int e = tid; e < N * N; e += nt) {
        const int r = e / N, col = e % N;
        int p, q, pp, qq;
        order_pq(b, r, p, q);
        order_pq(b, col, pp, qq);
        const double sx = rect1d(p - pp, c.fill_x), sy = rect1d(q - qq, c.fill_y);
        // (1/eps)_{pq} (rcwa2d.cpp:25-35, 288-295)
        cplx ei = cscale(dI, sx * sy);
        if (p == pp && q == qq) ei = cadd(ei, ibe);
        Einv[e] = ei;
        // Exx (rcwa2d.cpp:305-315): inverse rule in x, Laurent in y
        cplx vx = cscale(ax[(p + b.Mx) * nx + (pp + b.Mx)], sy);
        if (p == pp) vx = cadd(vx, cscale(eb, (q == qq ? 1.0 : 0.0) - sy));
        Exx[e] = vx;
        // Eyy (rcwa2d.cpp:323-333)
        cplx vy = cscale(ay[(q + b.My) * ny + (qq + b.My)], sx);
        if (q == qq) vy = cadd(vy, cscale(eb, (p == pp ? 1.0 : 0.0) - sx));
        Eyy[e] = vy;
    }
}

// ---- Fourier operators: rasterised shape, Laurent rule --------------------------
__device__ bool inside_shape(const CellDev& c, double xf, double yf) {
    if (c.rot != 0.0) {  // rcwa2d.cpp:41-47
        const double co = cos(c.rot), si = sin(c.rot);
        const double xr = co * xf + si * yf;
        const double yr = -si * xf + co * yf;
        xf = xr;
        yf = yr;
    }
    const double ax = c.fill_x * 0.5, ay = c.fill_y * 0.5;
    switch (c.shape) {
        case CELERIS_SHAPE_RECT:
            return fabs(xf) <= ax && fabs(yf) <= ay;
        case CELERIS_SHAPE_ELLIPSE: {
            if (ax <= 0.0 || ay <= 0.0) return false;
            const double u = xf / ax, v = yf / ay;
            return u * u + v * v <= 1.0;
        }
        case CELERIS_SHAPE_CROSS: {
            const double hx = ax * c.shape_param, hy = ay * c.shape_param;
            const bool vbar = fabs(xf) <= hx && fabs(yf) <= ay;
            const bool hbar = fabs(yf) <= hy && fabs(xf) <= ax;
            return vbar || hbar;
        }
        case CELERIS_SHAPE_RING: {
            if (ax <= 0.0 || ay <= 0.0) return false;
            const double u = xf / ax, v = yf / ay;
            const double r2 = u * u + v * v;
            const double ri = c.shape_param;
            return r2 <= 1.0 && r2 >= ri * ri;
        }
    }
    return false;
}

// phase tables: ph[(m + mmax) * ng + i] = exp(-2 pi i m xf_i) / ng, xf = (i+0.5)/ng - 0.5
__global__ void rcwa_phase_table(int ng, int mmax, cplx* ph) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (2 * mmax + 1) * ng) return;
    const int m = e / ng - mmax, i = e % ng;
    const double xf = (i + 0.5) / ng - 0.5;
    double s, co;
    sincos(-2.0 * PI * m * xf, &s, &co);
    ph[e] = C(co / ng, s / ng);
}

// 1 / sqrt(cnt) for cnt = 2^e, e in 0..4: the product of two orbit-vector
// weights (1, 1/sqrt2 or 1/2 each) with no rounding beyond the one constant.
__device__ __forceinline__ double orbit_weight(int e) {
    return (e & 1) ? ldexp(0.70710678118654752440, -(e >> 1)) : ldexp(1.0, -(e >> 1));
}

// Position of order (p, q) in scalar parity class c: its index in the class
// basis (orbit vectors of (|p|, |q|)) and the sign of its entry there, or
// -1 when the orbit has no vector in that class (p = 0 in an odd-x class, or
// q = 0 in an odd-y class). *e gains log2 of the orbit size.
__device__ __forceinline__ int scalar_class_index(int My, int c, int p, int q, double* sgn, int* e) {
    const int a = sym_class_a(c), bb = sym_class_b(c);
    if ((p == 0 && a < 0) || (q == 0 && bb < 0)) return -1;
    const int ap = abs(p), aq = abs(q);
    *sgn = (p < 0 && a < 0 ? -1.0 : 1.0) * (q < 0 && bb < 0 ? -1.0 : 1.0);
    *e += (ap > 0) + (aq > 0);
    return (ap - (a > 0 ? 0 : 1)) * sym_count(My, bb) + (aq - (bb > 0 ? 0 : 1));
}

// Einv = epsT^-1 of a mirror-symmetric cell (Bucket::sym != 0). The Laurent
// matrix epsT[(p,q)][(p',q')] = Ge[p-p'][q-q'] commutes with both mirrors when
// Ge is even in dp and in dq, so in the scalar parity basis (unit orbit vectors
// of (|p|, |q|) with signs a^[p<0] b^[q<0]) it is block diagonal with four blocks
// of orders (Mx + [a>0]) (My + [b>0]). Each block is inverted on its own, in
// place in shared memory by Gauss-Jordan with partial pivoting (about N^3/16 of
// the work of the full inverse, and no triangular solves), and Einv assembled:
//   Einv[k][l] = sum_c s_c(k) s_c(l) B_c^-1[i_c(k)][i_c(l)].
// A Ge that is not even to the symmetry tolerance flags the cell kInfoAsym (it
// is solved again by the full path). work: 2 N^2 complex (blocks, then their
// inverses); smem: the kernel's dynamic shared memory, Ge's region included.
__device__ void laurent_inverse_by_class(const Bucket& b, int cell, const cplx* Ge, cplx* work, cplx* Einv,
                                         unsigned char* smem, RedScratch* rs) {
    const int Mx = b.Mx, My = b.My, N = b.N, my4 = 4 * My + 1, mx4 = 4 * Mx + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    double dev = 0.0, mag = 0.0;
    for (int e = tid; e < mx4 * my4; e += nt) {
        const int pi = e / my4, qi = e % my4;
        const cplx v = Ge[e];
        dev = fmax(dev, fmax(cabs(csub(v, Ge[(mx4 - 1 - pi) * my4 + qi])), cabs(csub(v, Ge[pi * my4 + (my4 - 1 - qi)]))));
        mag = fmax(mag, cabs(v));
    }
    for (int o = 16; o > 0; o >>= 1) {
        dev = fmax(dev, __shfl_down_sync(0xffffffffu, dev, o));
        mag = fmax(mag, __shfl_down_sync(0xffffffffu, mag, o));
    }
    if ((tid & 31) == 0) {
        rs->d[tid >> 5] = dev;
        rs->d[32 + (tid >> 5)] = mag;
    }
    // assemble the four blocks B_c = S_c^T epsT S_c and identity right-hand sides
    size_t off = 0;
    for (int c = 0; c < 4; ++c) {
        const int a = sym_class_a(c), bb = sym_class_b(c);
        const int nb = sym_count(My, bb), s = sym_count(Mx, a) * nb;
        cplx* B = work + off;
        for (int e = tid; e < s * s; e += nt) {
            const int i = e / s, j = e % s;
            const int pi = i / nb + (a > 0 ? 0 : 1), qi = i % nb + (bb > 0 ? 0 : 1);
            const int pj = j / nb + (a > 0 ? 0 : 1), qj = j % nb + (bb > 0 ? 0 : 1);
            const double w = orbit_weight((pi > 0) + (qi > 0) + (pj > 0) + (qj > 0));
            cplx v = C(0.0, 0.0);
            for (int sp = 1; sp >= (pi > 0 ? -1 : 1); sp -= 2)
                for (int sq = 1; sq >= (qi > 0 ? -1 : 1); sq -= 2)
                    for (int tp = 1; tp >= (pj > 0 ? -1 : 1); tp -= 2)
                        for (int tq = 1; tq >= (qj > 0 ? -1 : 1); tq -= 2) {
                            const double sg = (sp < 0 ? a : 1) * (sq < 0 ? bb : 1) * (tp < 0 ? a : 1) * (tq < 0 ? bb : 1);
                            const cplx g = Ge[(sp * pi - tp * pj + 2 * Mx) * my4 + (sq * qi - tq * qj + 2 * My)];
                            v = cadd(v, cscale(g, sg));
                        }
            B[e] = cscale(v, w);
        }
        off += (size_t)s * s;
    }
    __syncthreads();
    if (tid == 0) {
        double d = 0.0, m = 0.0;
        for (int w = 0; w < nt / 32; ++w) {
            d = fmax(d, rs->d[w]);
            m = fmax(m, rs->d[32 + w]);
        }
        if (!(d < b.sym_tol * m) && b.info[cell] == 0) b.info[cell] = kInfoAsym;  // strict: tolerance 0 flags all
    }
    // Ge is dead: each block is inverted in place in shared memory over the
    // raster region (Gauss-Jordan, laurent_smem() reserves the largest block)
    off = 0;
    for (int c = 0; c < 4; ++c) {
        const int s = sym_count(Mx, sym_class_a(c)) * sym_count(My, sym_class_b(c));
        if (s == 0) continue;
        const int ld = s | 1;  // odd: the pivot search's column walk spreads over the banks
        cplx* Ms = reinterpret_cast<cplx*>(smem);
        cplx* scr = Ms + (size_t)s * ld;
        int* gpiv = reinterpret_cast<int*>(scr + 2 * s + 1);
        int* sp = gpiv + s;
        const cplx* B = work + off;
        for (int e = tid; e < s * s; e += nt) Ms[(e / s) * ld + e % s] = B[e];
        const int info = blk_gj_inverse_smem(s, Ms, ld, scr, gpiv, sp);
        if (info != 0 && tid == 0 && b.info[cell] == 0) b.info[cell] = -info;
        cplx* R = work + (size_t)N * N + off;
        for (int e = tid; e < s * s; e += nt) R[e] = Ms[(e / s) * ld + e % s];
        __syncthreads();
        off += (size_t)s * s;
    }
    size_t offs[4];
    off = 0;
    for (int c = 0; c < 4; ++c) {
        offs[c] = off;
        const int s = sym_count(Mx, sym_class_a(c)) * sym_count(My, sym_class_b(c));
        off += (size_t)s * s;
    }
    for (int e = tid; e < N * N; e += nt) {
        int p, q, pp, qq;
        order_pq(b, e / N, p, q);
        order_pq(b, e % N, pp, qq);
        cplx v = C(0.0, 0.0);
        for (int c = 0; c < 4; ++c) {
            double si, sj;
            int ex = 0;
            const int i = scalar_class_index(My, c, p, q, &si, &ex);
            const int j = scalar_class_index(My, c, pp, qq, &sj, &ex);
            if (i < 0 || j < 0) continue;
            const int s = sym_count(Mx, sym_class_a(c)) * sym_count(My, sym_class_b(c));
            const cplx r = work[(size_t)N * N + offs[c] + (size_t)i * s + j];
            v = cadd(v, cscale(r, si * sj * orbit_weight(ex)));
        }
        Einv[e] = v;
    }
}

// Rows of G1 in shared memory: at least 4, so that the per-axis sample tables
// of the raster (2 x 4 ng doubles) fit in the same region.
__host__ __device__ __forceinline__ int laurent_g1_rows(int Mx) { return 4 * Mx + 1 > 4 ? 4 * Mx + 1 : 4; }

// The sample coordinate (rcwa2d.cpp:88-89) of subsample s of pixel i.
__device__ __forceinline__ double raster_coord(int i, int s, int ng) { return (i + (s + 0.5) / 4) / ng - 0.5; }

// dynamic smem: G1 [laurent_g1_rows(Mx) * ng] | Ge [(4Mx+1)(4My+1)] | counts [ng*ng] u8,
// counts stored column-major (cnt[ix * ng + iy]) so that the row sums of G1 read
// consecutive bytes across a warp.
__global__ void __launch_bounds__(kRT) rcwa_fourier_laurent(Bucket b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ RedScratch rs;
    const int cell = blockIdx.x;
    const CellDev c = b.cells[cell];
    const int ng = b.ng, N = b.N;
    const int mx4 = 4 * b.Mx + 1, my4 = 4 * b.My + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    cplx* G1 = reinterpret_cast<cplx*>(smem);
    cplx* Ge = G1 + (size_t)laurent_g1_rows(b.Mx) * ng;
    unsigned char* cnt = reinterpret_cast<unsigned char*>(Ge + (size_t)mx4 * my4);
    // 4x4 supersampled inside counts (rcwa2d.cpp:74-95). Unrotated, every shape
    // test factors into per-axis terms: the sample coordinates (or their scaled
    // squares) are tabulated once per axis in the G1 region, and each of a
    // pixel's 16 samples combines one entry of each table with the reference's
    // own roundings (u*u and v*v rounded separately, then added).
    const double ax = c.fill_x * 0.5, ay = c.fill_y * 0.5;
    const bool round_shape = c.shape == CELERIS_SHAPE_ELLIPSE || c.shape == CELERIS_SHAPE_RING;
    if (c.rot != 0.0 || (round_shape && (ax <= 0.0 || ay <= 0.0))) {
        for (int e = tid; e < ng * ng; e += nt) {
            const int ix = e / ng, iy = e % ng;
            int hit = 0;
            for (int sy = 0; sy < 4; ++sy)
                for (int sx = 0; sx < 4; ++sx)
                    if (inside_shape(c, raster_coord(ix, sx, ng), raster_coord(iy, sy, ng))) ++hit;
            cnt[e] = (unsigned char)hit;
        }
    } else {
        double* tx = reinterpret_cast<double*>(G1);
        double* ty = tx + 4 * ng;
        const double hx = ax * c.shape_param, hy = ay * c.shape_param;
        for (int t = tid; t < 4 * ng; t += nt) {
            const double xf = raster_coord(t >> 2, t & 3, ng), yf = xf;  // square raster: one coordinate set
            if (round_shape) {
                const double u = xf / ax, v = yf / ay;
                tx[t] = __dmul_rn(u, u);
                ty[t] = __dmul_rn(v, v);
            } else {  // bit 0: within the main half-width, bit 1: within the cross arm's
                tx[t] = (fabs(xf) <= ax ? 1.0 : 0.0) + (fabs(xf) <= hx ? 2.0 : 0.0);
                ty[t] = (fabs(yf) <= ay ? 1.0 : 0.0) + (fabs(yf) <= hy ? 2.0 : 0.0);
            }
        }
        __syncthreads();
        const double ri2 = __dmul_rn(c.shape_param, c.shape_param);
        for (int e = tid; e < ng * ng; e += nt) {
            const int ix = e / ng, iy = e % ng;
            double X[4], Y[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                X[s] = tx[4 * ix + s];
                Y[s] = ty[4 * iy + s];
            }
            int hit = 0;
#pragma unroll
            for (int sy = 0; sy < 4; ++sy)
#pragma unroll
                for (int sx = 0; sx < 4; ++sx) {
                    bool in;
                    if (round_shape) {
                        const double r2 = __dadd_rn(X[sx], Y[sy]);
                        in = r2 <= 1.0 && (c.shape == CELERIS_SHAPE_ELLIPSE || r2 >= ri2);
                    } else {
                        const int bx = (int)X[sx], by = (int)Y[sy];
                        in = c.shape == CELERIS_SHAPE_RECT ? ((bx & by & 1) != 0)
                                                           : (((bx >> 1) & by & 1) != 0 || ((by >> 1) & bx & 1) != 0);
                    }
                    hit += in ? 1 : 0;
                }
            cnt[e] = (unsigned char)hit;
        }
        __syncthreads();  // the tables are dead: G1 overwrites them
    }
    __syncthreads();
    const cplx dE = csub(c.eps_p, c.eps_b);
    // G1[dp][iy] = sum_ix eps[iy][ix] PX[dp][ix]   (rcwa2d.cpp:170-177); four
    // rows dp per thread share the raster reads and give four independent chains
    for (int e = tid; e < ((mx4 + 3) >> 2) * ng; e += nt) {
        const int dp0 = 4 * (e / ng), iy = e % ng;
        const int nd = min(4, mx4 - dp0);
        cplx s[4] = {C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0)};
        for (int ix = 0; ix < ng; ++ix) {
            const cplx eps = cadd(c.eps_b, cscale(dE, cnt[ix * ng + iy] / 16.0));
#pragma unroll
            for (int d = 0; d < 4; ++d)
                if (d < nd) s[d] = cfma(eps, b.phx[(size_t)(dp0 + d) * ng + ix], s[d]);
        }
        for (int d = 0; d < nd; ++d) G1[(size_t)(dp0 + d) * ng + iy] = s[d];
    }
    __syncthreads();
    // Ge[dp][dq] = sum_iy G1[dp][iy] PY[dq][iy]   (rcwa2d.cpp:179-185)
    for (int e = tid; e < mx4 * my4; e += nt) {
        const int dpi = e / my4, dqi = e % my4;
        const cplx* ph = b.phy + (size_t)dqi * ng;
        cplx s = C(0.0, 0.0);
        for (int iy = 0; iy < ng; ++iy) s = cfma(G1[dpi * ng + iy], ph[iy], s);
        Ge[e] = s;
    }
    __syncthreads();
    // Laurent Toeplitz (rcwa2d.cpp:191-198); Exx = Eyy = epsT
    cplx* Exx = at(b.Exx, b.s_NN, cell);
    cplx* lu = at(b.H, b.s_nn, cell);  // scratch for the LU of epsT
    cplx* Einv = at(b.Einv, b.s_NN, cell);
    for (int e = tid; e < N * N; e += nt) {
        const int r = e / N, col = e % N;
        int p, q, pp, qq;
        order_pq(b, r, p, q);
        order_pq(b, col, pp, qq);
        const cplx v = Ge[(p - pp + 2 * b.Mx) * my4 + (q - qq + 2 * b.My)];
        Exx[e] = v;
        if (!b.sym) {
            lu[e] = v;
            Einv[e] = C(r == col ? 1.0 : 0.0, 0.0);
        }
    }
    if (b.sym) {
        laurent_inverse_by_class(b, cell, Ge, lu, Einv, smem, &rs);
        return;
    }
    __syncthreads();
    // the raster, G1 and Ge are dead: the LU staging and GEMM tiles overlay them
    cplx* stg = reinterpret_cast<cplx*>(smem);
    GemmSmem* gs = reinterpret_cast<GemmSmem*>(stg + 2 * N + LNB * LNB);
    int* piv = b.piv + b.s_n * cell;
    const int info = blk_lu_blocked(N, lu, N, piv, &rs, stg, gs);
    if (info != 0 && tid == 0 && b.info[cell] == 0) b.info[cell] = -info;  // keep an earlier stage's code
    blk_lu_solve_blocked(N, lu, N, piv, N, Einv, N, stg, gs);  // Einv = epsT^{-1} (rcwa2d.cpp:203)
}

// ---- M = ep2 kp - kkT -------------------------------------------------------------
__global__ void __launch_bounds__(kRT) rcwa_build_M(Bucket b, int laurent) {
    __shared__ GemmSmem gs;
    const int cell = blockIdx.x;
    const CellDev c = b.cells[cell];
    const int N = b.N, n = b.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    const cplx* Einv = at(b.Einv, b.s_NN, cell);
    const cplx* Exx = at(b.Exx, b.s_NN, cell);
    const cplx* Eyy = laurent ? Exx : at(b.Eyy, b.s_NN, cell);
    cplx* tmp = at(b.Z, b.s_nn, cell);  // [2N x N]: Eyy diag(-ky) ; Exx diag(kx)
    cplx* Y = at(b.X, b.s_nn, cell);    // [2N x N]: Ytop ; Ybot
    for (int e = tid; e < N * N; e += nt) {
        const int col = e % N;
        tmp[e] = cmul(Eyy[e], cneg(ky_of(b, c, col)));
        tmp[N * N + e] = cmul(Exx[e], kx_of(b, c, col));
    }
    blk_gemm(2 * N, N, N, C(1.0, 0.0), tmp, N, Einv, N, C(0.0, 0.0), Y, N, &gs);
    cplx* H = at(b.H, b.s_nn, cell);
    const double w2 = c.omega * c.omega;
    for (int e = tid; e < n * n; e += nt) {
        const int i = e / n, j = e % n;
        cplx v;
        if (i < N && j < N) {
            v = cfma(Y[i * N + j], ky_of(b, c, j), cscale(Eyy[i * N + j], w2));
            if (i == j) v = csub(v, cmul(kx_of(b, c, i), kx_of(b, c, i)));
        } else if (i < N) {
            const int m = j - N;
            v = cneg(cmul(Y[i * N + m], kx_of(b, c, m)));
            if (i == m) v = csub(v, cmul(kx_of(b, c, i), ky_of(b, c, i)));
        } else if (j < N) {
            const int l = i - N;
            v = cmul(Y[(N + l) * N + j], ky_of(b, c, j));
            if (l == j) v = csub(v, cmul(ky_of(b, c, l), kx_of(b, c, l)));
        } else {
            const int l = i - N, m = j - N;
            v = cfms(Y[(N + l) * N + m], kx_of(b, c, m), cscale(Exx[l * N + m], w2));
            if (l == m) v = csub(v, cmul(ky_of(b, c, l), ky_of(b, c, l)));
        }
        H[e] = v;
    }
}

// ---- eigensolve -----------------------------------------------------------------------
// Three kernels so that each gets its own register budget (the bulge chase
// keeps 16-element row/column segments in registers). SMEM variants (n <= 112)
// stage H in shared memory for the duration of the kernel.
// dynamic smem: SMEM: H [n*n] | v [n] | w [n] (rank-1 updates on the shared
// copy); otherwise the staging of blk_hessenberg_blocked (scratch in X, which
// is free until the eigenvectors).
// The shared-memory variant may run 512 threads: for the larger orders its
// shared block leaves one CTA per SM, and the column steps are latency-bound.
constexpr int kHessBigThreads = 512;
template <bool SMEM>
__global__ void __launch_bounds__(SMEM ? kHessBigThreads : kRT) rcwa_hess(Bucket b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ RedScratch rs;
    const int cell = blockIdx.x;
    const int n = b.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    cplx* Hg = at(b.H, b.s_nn, cell);
    if constexpr (SMEM) {
        // reduce H in shared memory recording the reflectors in X (free until
        // the eigenvectors), write H back, then form Z = Q in the same shared
        // buffer
        cplx* H = reinterpret_cast<cplx*>(smem);
        cplx* v = H + (size_t)n * n;
        cplx* refl = at(b.X, b.s_nn, cell);
        for (int e = tid; e < n * n; e += nt) H[e] = Hg[e];
        __syncthreads();
        blk_hessenberg_refl(n, H, n, refl, v, v + n, &rs);
        __syncthreads();
        for (int e = tid; e < n * n; e += nt) Hg[e] = H[e];
        __syncthreads();
        blk_form_q(n, H, n, refl, v, v + n);
        __syncthreads();
        cplx* Zg = at(b.Z, b.s_nn, cell);
        for (int e = tid; e < n * n; e += nt) Zg[e] = H[e];
    } else {
        __shared__ GemmSmem gs;
        blk_hessenberg_blocked(n, Hg, n, at(b.Z, b.s_nn, cell), n, at(b.X, b.s_nn, cell),
                               reinterpret_cast<cplx*>(smem), &rs, &gs,
                               b.dbg ? b.dbg + kDbgSlots * (size_t)cell + 9 : nullptr);
    }
}

// Schur form by multishift QR with aggressive early deflation (schur_aed.cuh).
// dynamic smem: AedShared.
// QR iteration cap for failure-path tests (0: the solver's own cap); set by
// celeris_debug_qr_iteration_cap.
__device__ int g_qr_iter_cap;

__global__ void __launch_bounds__(kSchurThreads, 2) rcwa_schur(Bucket b) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int cell = blockIdx.x;
    const int n = b.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    cplx* H = at(b.H, b.s_nn, cell);
    AedShared* sh = reinterpret_cast<AedShared*>(smem);
    const int info = blk_schur_aed(n, H, n, at(b.Z, b.s_nn, cell), n, sh,
                                   b.dbg ? b.dbg + kDbgSlots * (size_t)cell : nullptr, g_qr_iter_cap);
    if (tid == 0) {
        if (info != 0) b.info[cell] = info;
        if (b.dbg) b.dbg[kDbgSlots * (size_t)cell + 6] = sh->nsweep;
    }
    // eigenvalues -> q = branch(sqrt(lambda)) (rcwa2d.cpp:364)
    cplx* q1 = at(b.q1, b.s_n, cell);
    for (int i = tid; i < n; i += nt) {
        cplx q = csqrt_p(H[(size_t)i * n + i]);
        if (q.y < 0.0) q = cneg(q);
        q1[i] = q;
    }
}

// eigenvectors of T, then W = Z X
__global__ void __launch_bounds__(kRT) rcwa_vec(Bucket b) {
    __shared__ GemmSmem gs;
    const int cell = blockIdx.x;
    const int n = b.n;
    cplx* X = at(b.X, b.s_nn, cell);
    blk_trevc(n, at(b.H, b.s_nn, cell), n, X, n, at(b.A, b.s_nn, cell), &gs);  // A is free until smat1
    blk_gemm(n, n, n, C(1.0, 0.0), at(b.Z, b.s_nn, cell), n, X, n, C(0.0, 0.0), at(b.W, b.s_nn, cell), n, &gs);
}

// ---- S-matrix, interface 0 --------------------------------------------------------------
// dynamic smem: LU staging (2n + LNB^2 complex)
__global__ void __launch_bounds__(kRT) rcwa_smat1(Bucket b) {
    extern __shared__ __align__(16) unsigned char smem[];
    cplx* stg = reinterpret_cast<cplx*>(smem);
    __shared__ GemmSmem gs;
    __shared__ RedScratch rs;
    const int cell = blockIdx.x;
    const CellDev c = b.cells[cell];
    const int N = b.N, n = b.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    const double w2 = c.omega * c.omega;
    const cplx* W = at(b.W, b.s_nn, cell);
    const cplx* Einv = at(b.Einv, b.s_NN, cell);
    const cplx* q1 = at(b.q1, b.s_n, cell);
    cplx* V = at(b.Z, b.s_nn, cell);  // [N x n]
    cplx* U = at(b.X, b.s_nn, cell);  // [N x n]
    cplx* A = at(b.A, b.s_nn, cell);
    // A = kp W = w^2 W - Jk Einv (Jk^T W), Jk = [-Ky; Kx]
    for (int e = tid; e < N * n; e += nt) {
        const int i = e / n, j = e % n;
        V[e] = cfma(kx_of(b, c, i), W[(size_t)(N + i) * n + j], cneg(cmul(ky_of(b, c, i), W[(size_t)i * n + j])));
    }
    blk_gemm(N, n, N, C(1.0, 0.0), Einv, N, V, n, C(0.0, 0.0), U, n, &gs);
    for (int e = tid; e < N * n; e += nt) {
        const int i = e / n;
        A[e] = cfma(ky_of(b, c, i), U[e], cscale(W[e], w2));
        A[(size_t)N * n + e] = cfms(kx_of(b, c, i), U[e], cscale(W[(size_t)N * n + e], w2));
    }
    __syncthreads();
    // P = diag(q0) kp0^{-1} A diag(1/q1); T11 = (W + P)/2, T12 = (W - P)/2
    cplx* T11 = at(b.T11, b.s_nn, cell);
    cplx* T11lu = at(b.T11lu, b.s_nn, cell);
    cplx* T12 = at(b.T12, b.s_nn, cell);
    const cplx ier = cinv(cmul(c.n_inc, c.n_inc));
    const cplx er = cmul(c.n_inc, c.n_inc);
    for (int e = tid; e < N * n; e += nt) {
        const int i = e / n, j = e % n;
        const cplx kx = kx_of(b, c, i), ky = ky_of(b, c, i);
        cplx ka, kb, kc, kd;
        kp_uniform(ier, c.omega, kx, ky, ka, kb, kc, kd);
        const cplx kz = kz_uniform(er, c.omega, kx, ky);
        const cplx idet = cinv(csub(cmul(ka, kd), cmul(kb, kc)));
        const cplx c00 = cmul(kz, cmul(kd, idet)), c01 = cneg(cmul(kz, cmul(kb, idet)));
        const cplx c10 = cneg(cmul(kz, cmul(kc, idet))), c11 = cmul(kz, cmul(ka, idet));
        const cplx iq = cinv(q1[j]);
        const cplx a0 = A[(size_t)i * n + j], a1 = A[(size_t)(N + i) * n + j];
        const cplx p0 = cmul(cfma(c00, a0, cmul(c01, a1)), iq);
        const cplx p1 = cmul(cfma(c10, a0, cmul(c11, a1)), iq);
        const cplx w0 = W[(size_t)i * n + j], w1 = W[(size_t)(N + i) * n + j];
        const cplx t0 = cscale(cadd(w0, p0), 0.5), t1 = cscale(cadd(w1, p1), 0.5);
        T11[(size_t)i * n + j] = t0;
        T11[(size_t)(N + i) * n + j] = t1;
        T11lu[(size_t)i * n + j] = t0;
        T11lu[(size_t)(N + i) * n + j] = t1;
        T12[(size_t)i * n + j] = cscale(csub(w0, p0), 0.5);
        T12[(size_t)(N + i) * n + j] = cscale(csub(w1, p1), 0.5);
    }
    __syncthreads();
    // RHS [ -T12 D | a0_X | a0_Y ], D = diag(exp(i q1 h))
    cplx* S = at(b.S12, b.s_ns, cell);
    const int ld = n + 2;
    const int i0 = b.Mx * (2 * b.My + 1) + b.My;  // order (0, 0)
    for (int e = tid; e < n * ld; e += nt) {
        const int i = e / ld, j = e % ld;
        cplx v;
        if (j < n)
            v = cneg(cmul(T12[(size_t)i * n + j], cexpi(cscale(q1[j], c.h))));
        else if (j == n)
            v = C(i == N + i0 ? 1.0 : 0.0, 0.0);  // X: Ex0 = 1
        else
            v = C(i == i0 ? -1.0 : 0.0, 0.0);     // Y: Ey0 = 1 -> a0[i0] = -1
        S[e] = v;
    }
    __syncthreads();
    int* piv = b.piv + b.s_n * cell;
    const int info = blk_lu_blocked(n, T11lu, n, piv, &rs, stg, &gs);
    if (info != 0 && tid == 0 && b.info[cell] == 0) b.info[cell] = -info;  // keep an earlier stage's code
    blk_lu_solve_blocked(n, T11lu, n, piv, ld, S, ld, stg, &gs);  // [S12 | u_X | u_Y]
}

// ---- S-matrix, interface 1 + exterior amplitudes --------------------------------------------
// The layer -> substrate interface in the reference's form (rcwa2d.cpp:394-410) is
// T11' = (W^-1 + P')/2, T12' = (W^-1 - P')/2 with P' = diag(q1) A^-1 K, K the
// substrate kp diag(1/kz) blocks; the exterior amplitudes solve
// (T11' - D S12 T12') aN = D u, D = diag(exp(i q1 h)). With aN = W y the
// inverse of W drops out: T11' aN = (y + Q y)/2, T12' aN = (y - Q y)/2 with
// Q = diag(q1) A^-1 K W, so
//     (I + Q - D S12 + D S12 Q) y = 2 D u,   aN = W y,   y2 = T12' aN = (y - Q y)/2,
//     b0 = T12 (u + S12 y2) + T11 D y2.
// One LU of A with n right-hand sides, one GEMM and one LU of the combined
// matrix (instead of two inverses, a GEMM and an LU).
// dynamic smem: staging (2n + LNB^2 complex)
__global__ void __launch_bounds__(kRT) rcwa_smat2(Bucket b) {
    extern __shared__ __align__(16) unsigned char smem[];
    cplx* stg = reinterpret_cast<cplx*>(smem);
    __shared__ GemmSmem gs;
    __shared__ RedScratch rs;
    const int cell = blockIdx.x;
    const CellDev c = b.cells[cell];
    const int N = b.N, n = b.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    const cplx* W = at(b.W, b.s_nn, cell);
    cplx* A = at(b.A, b.s_nn, cell);
    cplx* Q = at(b.H, b.s_nn, cell);   // K W, then Q (H, Z, X are dead after the eigenvectors)
    cplx* SQ = at(b.Z, b.s_nn, cell);  // S12 Q
    cplx* Cm = at(b.X, b.s_nn, cell);  // I + Q - D S12 + D S12 Q, then its LU
    const cplx* q1 = at(b.q1, b.s_n, cell);
    int* piv = b.piv + b.s_n * cell;
    // K W: rows m and N+m mix through the substrate kp block of order m over kz_m
    const cplx ier = cinv(cmul(c.n_sub, c.n_sub));
    const cplx er = cmul(c.n_sub, c.n_sub);
    for (int e = tid; e < N * n; e += nt) {
        const int m = e / n, j = e % n;
        const cplx kx = kx_of(b, c, m), ky = ky_of(b, c, m);
        cplx ka, kb, kc, kd;
        kp_uniform(ier, c.omega, kx, ky, ka, kb, kc, kd);
        const cplx iq2 = cinv(kz_uniform(er, c.omega, kx, ky));
        const cplx w0 = W[(size_t)m * n + j], w1 = W[(size_t)(N + m) * n + j];
        Q[(size_t)m * n + j] = cmul(cfma(ka, w0, cmul(kb, w1)), iq2);
        Q[(size_t)(N + m) * n + j] = cmul(cfma(kc, w0, cmul(kd, w1)), iq2);
    }
    int info = blk_lu_blocked(n, A, n, piv, &rs, stg, &gs);
    blk_lu_solve_blocked(n, A, n, piv, n, Q, n, stg, &gs);  // A^-1 K W
    if (tid == 0 && info && b.info[cell] == 0) b.info[cell] = -info;
    for (int e = tid; e < n * n; e += nt) Q[e] = cmul(q1[e / n], Q[e]);
    cplx* S = at(b.S12, b.s_ns, cell);
    const int ld = n + 2;
    blk_gemm(n, n, n, C(1.0, 0.0), S, ld, Q, n, C(0.0, 0.0), SQ, n, &gs);
    for (int e = tid; e < n * n; e += nt) {
        const int i = e / n, j = e % n;
        const cplx d = cexpi(cscale(q1[i], c.h));
        cplx v = cadd(Q[e], cmul(d, csub(SQ[e], S[(size_t)i * ld + j])));
        if (i == j) v.x += 1.0;
        Cm[e] = v;
    }
    // rhs = 2 D u (2 columns) into vec scratch [n x 2]
    cplx* vec = at(b.vec, 10 * b.s_n, cell);
    cplx* x = vec + 4 * (size_t)b.s_n;    // [n x 2] row-major: y
    cplx* y2 = vec + 6 * (size_t)b.s_n;   // [n x 2]: Q y, then y2
    cplx* zz = vec + 8 * (size_t)b.s_n;   // [n x 2]: u + S12 y2
    for (int e = tid; e < 2 * n; e += nt) {
        const int i = e / 2, r = e % 2;
        x[e] = cscale(cmul(cexpi(cscale(q1[i], c.h)), S[(size_t)i * ld + n + r]), 2.0);
    }
    info = blk_lu_blocked(n, Cm, n, piv, &rs, stg, &gs);
    if (tid == 0 && info && b.info[cell] == 0) b.info[cell] = -info;
    blk_lu_solve_blocked(n, Cm, n, piv, 2, x, 2, stg, &gs);  // x = y (X, Y)
    cplx* aN = vec;                      // [2][n]
    cplx* b0 = vec + 2 * (size_t)b.s_n;  // [2][n]
    for (int e = tid; e < 2 * n; e += nt) stg[e] = x[e];
    __syncthreads();
    blk_matvec2(n, n, W, n, stg, aN, 1, b.s_n, false);  // aN = W y
    blk_matvec2(n, n, Q, n, stg, y2, 2, 1, false);      // Q y
    __syncthreads();
    for (int e = tid; e < 2 * n; e += nt) {
        const cplx v = cscale(csub(stg[e], y2[e]), 0.5);
        y2[e] = v;
        zz[e] = S[(size_t)(e / 2) * ld + n + (e % 2)];  // u
    }
    __syncthreads();
    for (int e = tid; e < 2 * n; e += nt) stg[e] = y2[e];
    __syncthreads();
    blk_matvec2(n, n, S, ld, stg, zz, 2, 1, true);  // u + S12 y2
    __syncthreads();
    // b0 = T12 zz + T11 (D y2)
    const cplx* T11 = at(b.T11, b.s_nn, cell);
    const cplx* T12 = at(b.T12, b.s_nn, cell);
    for (int e = tid; e < 2 * n; e += nt) stg[e] = zz[e];
    __syncthreads();
    blk_matvec2(n, n, T12, n, stg, b0, 1, b.s_n, false);
    __syncthreads();
    for (int e = tid; e < 2 * n; e += nt) stg[e] = cmul(cexpi(cscale(q1[e / 2], c.h)), y2[e]);
    __syncthreads();
    blk_matvec2(n, n, T11, n, stg, b0, 1, b.s_n, true);
}

// ---- multi-layer stacks ----------------------------------------------------------------------
// A stack is its incident half-space, nl patterned layers and the substrate. The
// layers run through the single-layer stages up to the eigenvectors as separate
// cells; rcwa_layer_out keeps each layer's region data (phi = W, kp phi = A,
// q, thickness) in a layer store; rcwa_stack_smat then runs the reference's
// S-matrix recursion over the nl + 1 interfaces (rcwa2d.cpp:376-401) for the two
// excitation columns (bN = 0, so only S11 a0 and S21 a0 are needed, with S12 and
// S22 kept whole for the recursion).
struct StackDev {
    int nl;     // patterned layers
    int slot0;  // first layer's slot in the layer store (layers are consecutive)
};
struct StackBucket {
    int Mx, My, N, n, nstack;
    const CellDev* cells;  // shared parameters of each stack (its first layer's descriptor)
    const StackDev* stacks;
    cplx *LW, *LA, *Lq;    // layer store: W [n*n], A [n*n], q [n] per slot
    const double* Lh;      // thickness per slot
    cplx *S12, *S22, *Q, *P, *X, *Y, *Z1;  // per stack, n*n each
    cplx* vec;             // per stack 10n: aN_X, aN_Y, b0_X, b0_Y | u [n x 2] | w [n x 2] | unused [n x 2]
    int* piv;
    int* info;
    size_t s_nn, s_n;
};

// Region data of one layer for the recursion: A = kp W (the operator of
// rcwa2d.cpp:344-349 applied to the eigenvectors), copied with W, q and the
// thickness into the layer store. Z and X are free after the eigenvectors.
__global__ void __launch_bounds__(kRT) rcwa_layer_out(Bucket b, cplx* LW, cplx* LA, cplx* Lq, double* Lh,
                                                      const int* slot) {
    __shared__ GemmSmem gs;
    const int cell = blockIdx.x;
    const CellDev c = b.cells[cell];
    const int N = b.N, n = b.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    const double w2 = c.omega * c.omega;
    const cplx* W = at(b.W, b.s_nn, cell);
    const cplx* Einv = at(b.Einv, b.s_NN, cell);
    cplx* V = at(b.Z, b.s_nn, cell);
    cplx* U = at(b.X, b.s_nn, cell);
    const int sl = slot[cell];
    cplx* Wo = LW + b.s_nn * sl;
    cplx* Ao = LA + b.s_nn * sl;
    // V = Jk^T W = Kx W_bottom - Ky W_top; U = Einv V
    for (int e = tid; e < N * n; e += nt) {
        const int i = e / n, j = e % n;
        V[e] = cfma(kx_of(b, c, i), W[(size_t)(N + i) * n + j], cneg(cmul(ky_of(b, c, i), W[(size_t)i * n + j])));
    }
    blk_gemm(N, n, N, C(1.0, 0.0), Einv, N, V, n, C(0.0, 0.0), U, n, &gs);
    // kp W = w^2 W + [Ky U; -Kx U]
    for (int e = tid; e < N * n; e += nt) {
        const int i = e / n;
        Ao[e] = cfma(ky_of(b, c, i), U[e], cscale(W[e], w2));
        Ao[(size_t)N * n + e] = cfms(kx_of(b, c, i), U[e], cscale(W[(size_t)N * n + e], w2));
    }
    for (int e = tid; e < n * n; e += nt) Wo[e] = W[e];
    for (int i = tid; i < n; i += nt) Lq[b.s_n * sl + i] = at(b.q1, b.s_n, cell)[i];
    if (tid == 0) Lh[sl] = c.h;
}

// kp block (2 x 2 per order) and kz of a homogeneous half-space (rcwa2d.cpp:254-273)
__device__ __forceinline__ void half_space(const StackBucket& sb, const CellDev& c, cplx nreg, int i, cplx& ka,
                                           cplx& kb, cplx& kc, cplx& kd, cplx& kz) {
    const int p = i / (2 * sb.My + 1) - sb.Mx, q = i % (2 * sb.My + 1) - sb.My;
    const cplx kx = csub(c.kx0, C(2.0 * PI * (double)p / c.px, 0.0));
    const cplx ky = csub(c.ky0, C(2.0 * PI * (double)q / c.py, 0.0));
    const cplx er = cmul(nreg, nreg);
    kp_uniform(cinv(er), c.omega, kx, ky, ka, kb, kc, kd);
    kz = kz_uniform(er, c.omega, kx, ky);
}

// One CTA per stack, two per SM (measured faster than one at 255 registers despite
// the spills at 128). dynamic smem: lu_stage_bytes(n)
__global__ void __launch_bounds__(kRT, 2) rcwa_stack_smat(StackBucket sb) {
    extern __shared__ __align__(16) unsigned char smem[];
    cplx* stg = reinterpret_cast<cplx*>(smem);
    __shared__ GemmSmem gs;
    __shared__ RedScratch rs;
    const int st = blockIdx.x;
    const CellDev c = sb.cells[st];
    const StackDev sd = sb.stacks[st];
    const int N = sb.N, n = sb.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    const size_t nn = sb.s_nn;
    cplx* S12 = sb.S12 + nn * st;
    cplx* S22 = sb.S22 + nn * st;
    cplx* Q = sb.Q + nn * st;
    cplx* P = sb.P + nn * st;
    cplx* X = sb.X + nn * st;
    cplx* Y = sb.Y + nn * st;
    cplx* Z1 = sb.Z1 + nn * st;
    cplx* vec = sb.vec + 10 * sb.s_n * st;
    cplx* u = vec + 4 * sb.s_n;  // S11 a0, [n x 2]
    cplx* w = vec + 6 * sb.s_n;  // T12 u, [n x 2]
    int* piv = sb.piv + sb.s_n * st;
    const int i0 = sb.Mx * (2 * sb.My + 1) + sb.My;
    int status = 0;
    // S11 a0 = a0 (columns X: Ex0 = 1, Y: Ey0 = 1), S21 a0 = 0, S12 = 0, S22 = I
    for (int e = tid; e < 2 * n; e += nt) {
        const int i = e / 2, r = e % 2;
        u[e] = (r == 0) ? C(i == N + i0 ? 1.0 : 0.0, 0.0) : C(i == i0 ? -1.0 : 0.0, 0.0);
        vec[(size_t)r * sb.s_n + i] = C(0.0, 0.0);
        vec[(2 + (size_t)r) * sb.s_n + i] = C(0.0, 0.0);
    }
    for (int e = tid; e < n * n; e += nt) {
        S12[e] = C(0.0, 0.0);
        S22[e] = C(e / n == e % n ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    const int NL = sd.nl + 2;  // regions: incident, layers, substrate
    for (int ia = 0; ia + 1 < NL; ++ia) {
        const int ib = ia + 1;
        const bool a_inc = ia == 0, b_sub = ib == NL - 1;
        const int sa = sd.slot0 + ia - 1, sbb = sd.slot0 + ib - 1;
        const cplx* qa = a_inc ? nullptr : sb.Lq + sb.s_n * sa;
        const cplx* qb = b_sub ? nullptr : sb.Lq + sb.s_n * sbb;
        const double ha = a_inc ? 0.0 : sb.Lh[sa], hb = b_sub ? 0.0 : sb.Lh[sbb];
        // Q = phi_a^-1 phi_b ; P = A_a^-1 A_b  (A = kp phi; half-spaces: phi = I, A = kp)
        for (int e = tid; e < n * n; e += nt) {
            const int i = e / n, j = e % n;
            cplx qv, pv;
            if (b_sub) {
                qv = C(i == j ? 1.0 : 0.0, 0.0);
                const int m = i % N;
                cplx ka, kb, kc, kd, kz;
                half_space(sb, c, c.n_sub, m, ka, kb, kc, kd, kz);
                // kp of the substrate: [[ka, kb], [kc, kd]] on rows / columns (m, N + m)
                pv = C(0.0, 0.0);
                if (j == m) pv = i < N ? ka : kc;
                else if (j == N + m) pv = i < N ? kb : kd;
            } else {
                qv = sb.LW[nn * sbb + e];
                pv = sb.LA[nn * sbb + e];
            }
            Q[e] = qv;
            P[e] = pv;
        }
        __syncthreads();
        if (a_inc) {
            // phi_a = I: Q is phi_b already; P <- kp_inc^-1 P by 2 x 2 blocks per order
            for (int e = tid; e < N * n; e += nt) {
                const int m = e / n, j = e % n;
                cplx ka, kb, kc, kd, kz;
                half_space(sb, c, c.n_inc, m, ka, kb, kc, kd, kz);
                const cplx idet = cinv(csub(cmul(ka, kd), cmul(kb, kc)));
                const cplx x0 = P[(size_t)m * n + j], x1 = P[(size_t)(N + m) * n + j];
                P[(size_t)m * n + j] = cmul(idet, csub(cmul(kd, x0), cmul(kb, x1)));
                P[(size_t)(N + m) * n + j] = cmul(idet, csub(cmul(ka, x1), cmul(kc, x0)));
            }
        } else {
            // the layer store's W and A of region a are not needed after this interface
            cplx* Wa = sb.LW + nn * sa;
            cplx* Aa = sb.LA + nn * sa;
            int inf = blk_lu_blocked(n, Wa, n, piv, &rs, stg, &gs);
            blk_lu_solve_blocked(n, Wa, n, piv, n, Q, n, stg, &gs);
            if (inf) status = inf;
            inf = blk_lu_blocked(n, Aa, n, piv, &rs, stg, &gs);
            blk_lu_solve_blocked(n, Aa, n, piv, n, P, n, stg, &gs);
            if (inf) status = inf;
        }
        __syncthreads();
        // P <- diag(q_a) P diag(1/q_b); T11 = (Q + P)/2 -> Q, T12 = (Q - P)/2 -> P
        for (int e = tid; e < n * n; e += nt) {
            const int i = e / n, j = e % n;
            cplx qai, qbj;
            if (a_inc) {
                cplx ka, kb, kc, kd;
                half_space(sb, c, c.n_inc, i % N, ka, kb, kc, kd, qai);
            } else {
                qai = qa[i];
            }
            if (b_sub) {
                cplx ka, kb, kc, kd;
                half_space(sb, c, c.n_sub, j % N, ka, kb, kc, kd, qbj);
            } else {
                qbj = qb[j];
            }
            const cplx pv = cdiv(cmul(qai, P[e]), qbj), qv = Q[e];
            Q[e] = cscale(cadd(qv, pv), 0.5);
            P[e] = cscale(csub(qv, pv), 0.5);
        }
        // X = T11 - d1 S12 T12 ; Y = d1 S12 T11 - T12   (d1 = exp(i q_a h_a) on the rows)
        blk_gemm(n, n, n, C(1.0, 0.0), S12, n, P, n, C(0.0, 0.0), X, n, &gs);
        blk_gemm(n, n, n, C(1.0, 0.0), S12, n, Q, n, C(0.0, 0.0), Y, n, &gs);
        for (int e = tid; e < n * n; e += nt) {
            const int i = e / n;
            const cplx d1 = a_inc ? C(1.0, 0.0) : cexpi(cscale(qa[i], ha));
            X[e] = cfms(d1, X[e], Q[e]);
            Y[e] = csub(cmul(d1, Y[e]), P[e]);
        }
        for (int e = tid; e < 2 * n; e += nt) {
            const int i = e / 2;
            const cplx d1 = a_inc ? C(1.0, 0.0) : cexpi(cscale(qa[i], ha));
            u[e] = cmul(d1, u[e]);
        }
        const int inf = blk_lu_blocked(n, X, n, piv, &rs, stg, &gs);
        if (inf) status = inf;
        blk_lu_solve_blocked(n, X, n, piv, n, Y, n, stg, &gs);  // Y = X^-1 (d1 S12 T11 - T12)
        blk_lu_solve_blocked(n, X, n, piv, 2, u, 2, stg, &gs);  // u = S11' a0 = X^-1 d1 S11 a0
        // S12' = Y diag(d2)
        for (int e = tid; e < n * n; e += nt) {
            const int j = e % n;
            const cplx d2 = b_sub ? C(1.0, 0.0) : cexpi(cscale(qb[j], hb));
            S12[e] = cmul(Y[e], d2);
        }
        // S21' a0 = S21 a0 + S22 T12 u'
        for (int e = tid; e < 2 * n; e += nt) stg[e] = u[e];
        __syncthreads();
        blk_matvec2(n, n, P, n, stg, w, 2, 1, false);  // w = T12 u'
        __syncthreads();
        for (int e = tid; e < 2 * n; e += nt) stg[e] = w[e];
        __syncthreads();
        blk_matvec2(n, n, S22, n, stg, vec + 2 * sb.s_n, 1, sb.s_n, true);
        // S22' = S22 (T12 S12' + T11 diag(d2))
        blk_gemm(n, n, n, C(1.0, 0.0), P, n, S12, n, C(0.0, 0.0), Z1, n, &gs);
        for (int e = tid; e < n * n; e += nt) {
            const int j = e % n;
            const cplx d2 = b_sub ? C(1.0, 0.0) : cexpi(cscale(qb[j], hb));
            Z1[e] = cfma(Q[e], d2, Z1[e]);
        }
        blk_gemm(n, n, n, C(1.0, 0.0), S22, n, Z1, n, C(0.0, 0.0), X, n, &gs);  // X is free after the solves
        for (int e = tid; e < n * n; e += nt) S22[e] = X[e];
        __syncthreads();
    }
    // exterior amplitudes for the epilogue: aN = S11 a0 (2 columns)
    for (int e = tid; e < 2 * n; e += nt) {
        const int i = e / 2, r = e % 2;
        vec[(size_t)r * sb.s_n + i] = u[e];
    }
    if (tid == 0 && status != 0) sb.info[st] = -status;
}

// ---- standalone eigensolve (eig.hpp:25) ------------------------------------------------------
// The RCWA eigen-stages on caller matrices: eig_load transposes a column-major
// (Eigen / LAPACK) matrix into the row-major H of its cell; eig_store writes the
// eigenvalues (diagonal of the Schur form) and the eigenvectors W = Z X in
// column-major order, each scaled to unit 2-norm with its largest-magnitude
// component real and positive (zgeev's normalisation).
__global__ void __launch_bounds__(kRT) eig_load(const cplx* __restrict__ A, Bucket b) {
    const int cell = blockIdx.x, n = b.n;
    const cplx* src = A + b.s_nn * cell;
    cplx* H = at(b.H, b.s_nn, cell);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e / n, j = e % n;
        H[e] = src[(size_t)j * n + i];
    }
}

__global__ void __launch_bounds__(kRT) eig_store(Bucket b, cplx* __restrict__ evals, cplx* __restrict__ evecs) {
    __shared__ RedScratch rs;
    const int cell = blockIdx.x, n = b.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    const cplx* H = at(b.H, b.s_nn, cell);
    const cplx* W = at(b.W, b.s_nn, cell);
    cplx* out = evecs + b.s_nn * cell;
    for (int i = tid; i < n; i += nt) evals[(size_t)cell * n + i] = H[(size_t)i * n + i];
    for (int j = 0; j < n; ++j) {
        double s2 = 0.0, big = -1.0;
        int arg = 0;
        for (int i = tid; i < n; i += nt) {
            const double m2 = cnorm2(W[(size_t)i * n + j]);
            s2 += m2;
            if (m2 > big) {
                big = m2;
                arg = i;
            }
        }
        const double tot = blk_sum(s2, &rs);
        const int imax = blk_argmax(big, arg, &rs);
        const cplx wm = W[(size_t)imax * n + j];
        const double am = cabs(wm);
        // conj(phase of the largest component) / norm
        const cplx sc = am > 0.0 && tot > 0.0 ? cscale(cconj(wm), 1.0 / (am * sqrt(tot))) : C(1.0, 0.0);
        for (int i = tid; i < n; i += nt) out[(size_t)j * n + i] = cmul(W[(size_t)i * n + j], sc);
        __syncthreads();
    }
}

// ---- flux and order-0 field (rcwa2d.cpp:416-463) ---------------------------------------------
__global__ void __launch_bounds__(kRT) rcwa_epilogue(Bucket b) {
    __shared__ RedScratch rs;
    __shared__ double sums[4];
    const int cell = blockIdx.x;
    const CellDev c = b.cells[cell];
    const int N = b.N;
    const int tid = threadIdx.x, nt = blockDim.x;
    const cplx* vec = at(b.vec, 10 * b.s_n, cell);
    const int i0 = b.Mx * (2 * b.My + 1) + b.My;
    const cplx er_i = cmul(c.n_inc, c.n_inc), ier_i = cinv(er_i);
    const cplx er_s = cmul(c.n_sub, c.n_sub), ier_s = cinv(er_s);
    const double norm = c.n_inc.x / cos(c.theta);  // rcwa2d.cpp:437
    for (int ex = 0; ex < c.nexc; ++ex) {
        // excitation coefficients: slot 0 = (ex0, ey0), slot 1 = Y (0, 1)
        const cplx fx = ex == 0 ? c.ex0 : C(0.0, 0.0);
        const cplx fy = ex == 0 ? c.ey0 : C(1.0, 0.0);
        double sR = 0.0, sT = 0.0;
        for (int i = tid; i < N; i += nt) {
            const cplx kx = kx_of(b, c, i), ky = ky_of(b, c, i);
            // incident region: a0 = -Ey0 e_i0 + Ex0 e_{N+i0}; b0 = fx b0_X + fy b0_Y
            const cplx a0s = i == i0 ? cneg(fy) : C(0.0, 0.0);
            const cplx a0p = i == i0 ? fx : C(0.0, 0.0);
            const cplx b0s = cfma(fx, vec[2 * b.s_n + i], cmul(fy, vec[3 * b.s_n + i]));
            const cplx b0p = cfma(fx, vec[2 * b.s_n + N + i], cmul(fy, vec[3 * b.s_n + N + i]));
            const cplx aNs = cfma(fx, vec[i], cmul(fy, vec[b.s_n + i]));
            const cplx aNp = cfma(fx, vec[N + i], cmul(fy, vec[b.s_n + N + i]));
            cplx ka, kb, kc, kd;
            // incident: A = kp diag(1/(omega q)), phi = I
            kp_uniform(ier_i, c.omega, kx, ky, ka, kb, kc, kd);
            const cplx iwq_i = cinv(cscale(kz_uniform(er_i, c.omega, kx, ky), c.omega));
            const cplx Aa0 = cmul(cfma(ka, a0s, cmul(kb, a0p)), iwq_i), Aa1 = cmul(cfma(kc, a0s, cmul(kd, a0p)), iwq_i);
            const cplx Ab0 = cmul(cfma(ka, b0s, cmul(kb, b0p)), iwq_i), Ab1 = cmul(cfma(kc, b0s, cmul(kd, b0p)), iwq_i);
            // bwd flux of the incident region: bxy = -Re(conj(Ab) pb) + conj(diff)
            const cplx d0 = cscale(csub(cmulc(b0s, Aa0), cmulc(Ab0, a0s)), 0.5);
            const cplx d1 = cscale(csub(cmulc(b0p, Aa1), cmulc(Ab1, a0p)), 0.5);
            const double bw = -cmulc(Ab0, b0s).x + d0.x - cmulc(Ab1, b0p).x + d1.x;  // Re(bxy_i + bxy_{N+i})
            // substrate: forward flux fxy = Re(conj(Aa) pa) + diff, b = 0
            kp_uniform(ier_s, c.omega, kx, ky, ka, kb, kc, kd);
            const cplx iwq_s = cinv(cscale(kz_uniform(er_s, c.omega, kx, ky), c.omega));
            const cplx Sa0 = cmul(cfma(ka, aNs, cmul(kb, aNp)), iwq_s), Sa1 = cmul(cfma(kc, aNs, cmul(kd, aNp)), iwq_s);
            const double fw = cmulc(Sa0, aNs).x + cmulc(Sa1, aNp).x;
            sR += -bw * norm;
            sT += fw * norm;
            if (b.ord) {  // rcwa2d.cpp:479-480
                double* o = b.ord + 2 * ((size_t)(cell * c.nexc + ex) * N + i);
                o[0] = fw * norm;
                o[1] = -bw * norm;
            }
            if (i == i0) {
                sums[0] = -bw * norm;   // de_r0
                sums[1] = fw * norm;    // de_t0
                // order-0 fields: Esub = A_sub aN, Einc = A_inc a0
                const cplx ex_inc = Aa1;
                const cplx den = cabs(ex_inc) > 1e-30 ? ex_inc : C(1.0, 0.0);
                const cplx tx = cdiv(Sa1, den), ty = cneg(cdiv(Sa0, den));
                celeris_rcwa_result* r = &b.res[(size_t)cell * c.nexc + ex];
                r->tx0[0] = tx.x;
                r->tx0[1] = tx.y;
                r->ty0[0] = ty.x;
                r->ty0[1] = ty.y;
            }
        }
        const double R = blk_sum(sR, &rs);
        const double T = blk_sum(sT, &rs);
        if (tid == 0) {
            celeris_rcwa_result* r = &b.res[(size_t)cell * c.nexc + ex];
            r->R = R;
            r->T = T;
            r->sum_de = R + T;
            r->de_r0 = sums[0];
            r->de_t0 = sums[1];
            if (b.info[cell] != 0) {
                const double nan = __longlong_as_double(0x7ff8000000000000LL);
                r->R = r->T = r->sum_de = r->de_t0 = r->de_r0 = nan;
                r->tx0[0] = r->tx0[1] = r->ty0[0] = r->ty0[1] = nan;
            }
        }
        __syncthreads();
    }
}

// ---- mirror-symmetric cells: the eigenproblem in four parity classes -------------------------
// A cell whose pattern is symmetric under x -> -x and under y -> -y (every
// unrotated shape of rcwa2d.cpp:37-72) at normal incidence (kx0 = ky0 = 0) has
// Kx odd and Ky even under the order map p -> -p (Px), and Einv, Exx, Eyy
// invariant under it; so M = ep2 kp - kkT commutes with Sx = diag(Px, -Px)
// (the two field blocks of rcwa2d.cpp:346-364) and likewise with Sy = diag(Py,
// -Py). Their joint eigenspaces - parity classes (a, b), a, b = +-1 - split M
// into four blocks of about n/4: the block-1 part of class (a, b) has parity
// (a, b) under (Px, Py), the block-2 part parity (-a, -b). Each class has an
// orthonormal basis of orbit vectors (the orders (+-p, +-q) of one orbit
// combined with signs a, b and weight 1/sqrt(count)). With P_c that basis,
//   M = sum_c P_c M_c P_c^T,  M_c = P_c^T M P_c,
// so the eigenpairs of M are those of the M_c mapped by P_c: W = [P_c W_c]_c.
// The eigen-stages then run on matrices of order ~n/4 (16x fewer QR
// rotations per class, 64x fewer flops each); the S-matrix stages use the
// full W unchanged, so t, R and T are those of the full eigensolve up to
// rounding. M_c is built straight from the scalar parity blocks of Exx, Eyy
// and Einv (rcwa_sym_build; the Laurent Einv itself comes from four block
// inverses), never forming M. A cell whose eps operators are not mirror
// symmetric to rounding (a raster sample falling exactly on a shape boundary
// one way and not the other) is flagged kInfoAsym and solved again by the full
// eigensolve. When the cell is
// also symmetric under the 90 degree rotation R (square period, Mx = My,
// fill_x = fill_y), R commutes with every operator and maps the X excitation
// onto the Y excitation, so only the X class is solved and the Y solution is R
// applied to the X one (a cell that fails that check to rounding is flagged too).
__host__ __device__ __forceinline__ int sym_class_size(int Mx, int My, int c) {
    const int a = sym_class_a(c), b = sym_class_b(c);
    return sym_count(Mx, a) * sym_count(My, b) + sym_count(Mx, -a) * sym_count(My, -b);
}

// Basis vector i of class c: its entries (2N-space indices and coefficients),
// returns their count (1, 2 or 4).
__device__ int sym_vector(int Mx, int My, int c, int i, int* idx, double* coef) {
    const int N = (2 * Mx + 1) * (2 * My + 1);
    const int a = sym_class_a(c), b = sym_class_b(c);
    const int nu = sym_count(Mx, a) * sym_count(My, b);
    int blk, pa, pb;  // field block, parities under Px, Py
    if (i < nu) {
        blk = 0, pa = a, pb = b;
    } else {
        i -= nu;
        blk = 1, pa = -a, pb = -b;
    }
    const int nq = sym_count(My, pb);
    const int p = i / nq + (pa > 0 ? 0 : 1), q = i % nq + (pb > 0 ? 0 : 1);
    const int cnt = (p > 0 ? 2 : 1) * (q > 0 ? 2 : 1);
    const double w = cnt == 4 ? 0.5 : (cnt == 2 ? 0.70710678118654752440 : 1.0);
    int k = 0;
    for (int sp = 0; sp < (p > 0 ? 2 : 1); ++sp)
        for (int sq = 0; sq < (q > 0 ? 2 : 1); ++sq) {
            const int pp = sp ? -p : p, qq = sq ? -q : q;
            idx[k] = blk * N + (pp + Mx) * (2 * My + 1) + (qq + My);
            coef[k] = w * (sp ? pa : 1) * (sq ? pb : 1);
            ++k;
        }
    return k;
}

// Entry (k, l) of a per-order block operator of a homogeneous half-space
// (non-zero only within one order: the 2 x 2 block of indices i, N + i).
// which = 0: incident diag(kz) kp^-1 (rcwa2d.cpp:376-388, P1 of the first
// interface); which = 1: substrate kp diag(1/kz) (K of the last interface).
__device__ cplx halfspace_entry(const Bucket& b, const CellDev& c, int which, int k, int l) {
    const int N = b.N;
    const int ok = k % N, ol = l % N;
    if (ok != ol) return C(0.0, 0.0);
    const cplx nr = which == 0 ? c.n_inc : c.n_sub;
    const cplx er = cmul(nr, nr), ier = cinv(er);
    const cplx kx = kx_of(b, c, ok), ky = ky_of(b, c, ok);
    cplx ka, kb, kc, kd;
    kp_uniform(ier, c.omega, kx, ky, ka, kb, kc, kd);
    const cplx kz = kz_uniform(er, c.omega, kx, ky);
    const int r = k / N, s = l / N;
    if (which == 0) {  // kz [[kd, -kb], [-kc, ka]] / det
        const cplx idet = cmul(kz, cinv(csub(cmul(ka, kd), cmul(kb, kc))));
        const cplx v = r == 0 ? (s == 0 ? kd : cneg(kb)) : (s == 0 ? cneg(kc) : ka);
        return cmul(v, idet);
    }
    const cplx v = r == 0 ? (s == 0 ? ka : kb) : (s == 0 ? kc : kd);
    return cmul(v, cinv(kz));
}

// Orbit (p, q) >= 0 of index i in scalar parity class (a, bb).
__device__ __forceinline__ void scalar_orbit(int My, int a, int bb, int i, int& p, int& q) {
    const int nb = sym_count(My, bb);
    p = i / nb + (a > 0 ? 0 : 1);
    q = i % nb + (bb > 0 ? 0 : 1);
}
// Index of orbit (p, q) >= 0 in scalar parity class (a, bb), -1 if it has none there.
__device__ __forceinline__ int scalar_orbit_index(int My, int a, int bb, int p, int q) {
    if ((p == 0 && a < 0) || (q == 0 && bb < 0)) return -1;
    return (p - (a > 0 ? 0 : 1)) * sym_count(My, bb) + (q - (bb > 0 ? 0 : 1));
}
// Entry (i, j) of S^T E S for the unit orbit vectors S of scalar class (a, bb)
// and an N x N order-space operator E that commutes with both mirrors.
__device__ cplx scalar_block_entry(const cplx* E, int N, int Mx, int My, int a, int bb, int i, int j) {
    const int ny = 2 * My + 1;
    int pi, qi, pj, qj;
    scalar_orbit(My, a, bb, i, pi, qi);
    scalar_orbit(My, a, bb, j, pj, qj);
    cplx v = C(0.0, 0.0);
    for (int sp = 1; sp >= (pi > 0 ? -1 : 1); sp -= 2)
        for (int sq = 1; sq >= (qi > 0 ? -1 : 1); sq -= 2) {
            const cplx* row = E + (size_t)((sp * pi + Mx) * ny + (sq * qi + My)) * N;
            const int si = (sp < 0 ? a : 1) * (sq < 0 ? bb : 1);
            for (int tp = 1; tp >= (pj > 0 ? -1 : 1); tp -= 2)
                for (int tq = 1; tq >= (qj > 0 ? -1 : 1); tq -= 2) {
                    const int sg = si * (tp < 0 ? a : 1) * (tq < 0 ? bb : 1);
                    v = cadd(v, cscale(row[(tp * pj + Mx) * ny + (tq * qj + My)], (double)sg));
                }
        }
    return cscale(v, orbit_weight((pi > 0) + (qi > 0) + (pj > 0) + (qj > 0)));
}

// The class operators of a mirror-symmetric cell, built from the scalar parity
// blocks of its eps operators (on the class path this replaces the full
// M = [Eyy; Exx] J Einv J' + ... of rcwa_build_M and its projection).
// Vector class c = (a, b) has its u field block in scalar class (a, b) and its
// v block in (-a, -b). Every operator of M maps parity classes onto parity
// classes: with kx0 = ky0 = 0, Kx takes the unit orbit vector of (|p|, |q|) in
// class (a, b) to kx = -2 pi |p| / px times the orbit vector of the same orbit
// in (-a, b), and Ky likewise in q. So with Eu = Eyy^(a,b), Ev = Exx^(-a,-b)
// and G = Einv^(a,-b), the one block of Einv that the class meets, and s(j) the
// index in (a, -b) of the orbit of j (its k is 0 where it has none):
//   Yt = Lt G, Lt[i][t] = Eu[i][t] (-ky(t));   Yb = Lb G, Lb[l][t] = Ev[l][t] kx(t)
//   M(u,u) = Yt[i][s(j)] ky(j) + w^2 Eu[i][j] - [i = j] kx^2
//   M(u,v) = -Yt[i][s(j)] kx(j) - [same orbit] kx ky
//   M(v,u) = Yb[l][s(j)] ky(j) - [same orbit] ky kx
//   M(v,v) = w^2 Ev[l][m] - Yb[l][s(m)] kx(m) - [l = m] ky^2
// (the order-space M of rcwa_build_M), the layer kp = w^2 - J Einv J^T
// (rcwa2d.cpp:346-352) as kp(u,u) = w^2 [i = j] - ky G ky, kp(u,v) = ky G kx,
// kp(v,u) = kx G ky, kp(v,v) = w^2 [i = j] - kx G kx, and each half-space
// operator as the 2 x 2 block of an orbit's representative order (|p|, |q|) (its
// u-v entries are odd in p and in q, the u-u and v-v entries even).
// Flags kInfoAsym when Exx, Eyy or Einv is not mirror symmetric to the
// tolerance, or, for a C4 bucket (ncls = 1), when Eyy[k][l] != Exx[rho k][rho l]
// or Einv[rho k][rho l] != Einv[k][l] (rho: order (p, q) -> (-q, p)); these
// make M commute with the mirrors (and with R).
// Scratch: the cell's full-order Z and X (free on the class path).
__global__ void __launch_bounds__(kRT) rcwa_sym_build(Bucket b) {
    __shared__ GemmSmem gs;
    __shared__ double red[6][32];
    const int cell = blockIdx.x;
    const CellDev cd = b.cells[cell];
    const int N = b.N, Mx = b.Mx, My = b.My, ny = 2 * My + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    const cplx* Exx = at(b.Exx, b.s_NN, cell);
    const cplx* Eyy = b.ng > 0 ? Exx : at(b.Eyy, b.s_NN, cell);
    const cplx* Einv = at(b.Einv, b.s_NN, cell);
    // symmetry of the ingredients: deviation and magnitude of Exx, Eyy, Einv
    double dv[3] = {0.0, 0.0, 0.0}, mg[3] = {0.0, 0.0, 0.0};
    for (int e = tid; e < N * N; e += nt) {
        const int k = e / N, l = e % N;
        const int pk = k / ny - Mx, qk = k % ny - My, pl = l / ny - Mx, ql = l % ny - My;
        const size_t ex = (size_t)((-pk + Mx) * ny + qk + My) * N + (-pl + Mx) * ny + ql + My;
        const size_t ey = (size_t)((pk + Mx) * ny - qk + My) * N + (pl + Mx) * ny - ql + My;
        const cplx* X[3] = {Exx, Eyy, Einv};
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            const cplx v = X[t][e];
            dv[t] = fmax(dv[t], fmax(cabs(csub(v, X[t][ex])), cabs(csub(v, X[t][ey]))));
            mg[t] = fmax(mg[t], cabs(v));
        }
        if (b.ncls == 1) {  // rho k = (-qk, pk): Mx = My, so ny indexes both axes
            const size_t er = (size_t)((-qk + Mx) * ny + pk + My) * N + (-ql + Mx) * ny + pl + My;
            dv[1] = fmax(dv[1], cabs(csub(Eyy[e], Exx[er])));
            dv[2] = fmax(dv[2], cabs(csub(Einv[e], Einv[er])));
        }
    }
#pragma unroll
    for (int t = 0; t < 3; ++t)
        for (int o = 16; o > 0; o >>= 1) {
            dv[t] = fmax(dv[t], __shfl_down_sync(0xffffffffu, dv[t], o));
            mg[t] = fmax(mg[t], __shfl_down_sync(0xffffffffu, mg[t], o));
        }
    if ((tid & 31) == 0)
        for (int t = 0; t < 3; ++t) {
            red[t][tid >> 5] = dv[t];
            red[3 + t][tid >> 5] = mg[t];
        }
    __syncthreads();
    if (tid == 0) {
        bool asym = false;
        for (int t = 0; t < 3; ++t) {
            double d = 0.0, m = 0.0;
            for (int w = 0; w < nt / 32; ++w) {
                d = fmax(d, red[t][w]);
                m = fmax(m, red[3 + t][w]);
            }
            asym = asym || !(d < b.sym_tol * m);  // strict: tolerance 0 flags every cell
        }
        if (asym && b.info[cell] == 0) b.info[cell] = kInfoAsym;
    }
    const double w2 = cd.omega * cd.omega;
    const int m = b.m[0];
    cplx* Zs = at(b.Z, b.s_nn, cell);
    cplx* Xs = at(b.X, b.s_nn, cell);
    for (int cc = 0; cc < b.ncls; ++cc) {
        const int c = b.cls0 + cc;
        const int a = sym_class_a(c), bb = sym_class_b(c);
        const int su = sym_count(Mx, a) * sym_count(My, bb);    // u block: (a, b)
        const int sv = sym_count(Mx, -a) * sym_count(My, -bb);  // v block: (-a, -b)
        const int st = sym_count(Mx, a) * sym_count(My, -bb);   // Einv block: (a, -b)
        cplx* Eu = Zs;
        cplx* Ev = Eu + (size_t)su * su;
        cplx* G = Ev + (size_t)sv * sv;
        cplx* Lt = G + (size_t)st * st;
        cplx* Lb = Xs;
        cplx* Yt = Lb + (size_t)sv * st;
        cplx* Yb = Yt + (size_t)su * st;
        __syncthreads();  // the previous class's readers of the scratch are done
        for (int e = tid; e < su * su; e += nt) Eu[e] = scalar_block_entry(Eyy, N, Mx, My, a, bb, e / su, e % su);
        for (int e = tid; e < sv * sv; e += nt) Ev[e] = scalar_block_entry(Exx, N, Mx, My, -a, -bb, e / sv, e % sv);
        for (int e = tid; e < st * st; e += nt) G[e] = scalar_block_entry(Einv, N, Mx, My, a, -bb, e / st, e % st);
        __syncthreads();
        // Lt[i][t] = Eu[i][orbit t in (a, b)] (-ky(t)), Lb[l][t] = Ev[l][orbit t in (-a, -b)] kx(t)
        for (int e = tid; e < (su + sv) * st; e += nt) {
            const int r = e / st, t = e % st;
            int pt, qt;
            scalar_orbit(My, a, -bb, t, pt, qt);
            if (r < su) {
                const int j = scalar_orbit_index(My, a, bb, pt, qt);
                const double ky = -(2.0 * PI * (double)qt / cd.py);
                Lt[(size_t)r * st + t] = j < 0 ? C(0.0, 0.0) : cscale(Eu[(size_t)r * su + j], -ky);
            } else {
                const int l = r - su;
                const int j = scalar_orbit_index(My, -a, -bb, pt, qt);
                const double kx = -(2.0 * PI * (double)pt / cd.px);
                Lb[(size_t)l * st + t] = j < 0 ? C(0.0, 0.0) : cscale(Ev[(size_t)l * sv + j], kx);
            }
        }
        blk_gemm(su, st, st, C(1.0, 0.0), Lt, st, G, st, C(0.0, 0.0), Yt, st, &gs);
        blk_gemm(sv, st, st, C(1.0, 0.0), Lb, st, G, st, C(0.0, 0.0), Yb, st, &gs);
        __syncthreads();
        const size_t mi = (size_t)(b.ncls * cell + cc) * m * m;
        cplx* Mc = b.sH[0] + mi;
        cplx* Kp = b.cKp + mi;
        cplx* C0 = b.cC0 + mi;
        cplx* Ks = b.cKs + mi;
        for (int e = tid; e < m * m; e += nt) {
            const int i = e / m, j = e % m;
            const bool ui = i < su, uj = j < su;
            const int li = ui ? i : i - su, lj = uj ? j : j - su;
            int pi, qi, pj, qj;
            scalar_orbit(My, ui ? a : -a, ui ? bb : -bb, li, pi, qi);
            scalar_orbit(My, uj ? a : -a, uj ? bb : -bb, lj, pj, qj);
            const int si = scalar_orbit_index(My, a, -bb, pi, qi), sj = scalar_orbit_index(My, a, -bb, pj, qj);
            const double kxi = -(2.0 * PI * (double)pi / cd.px), kyi = -(2.0 * PI * (double)qi / cd.py);
            const double kxj = -(2.0 * PI * (double)pj / cd.px), kyj = -(2.0 * PI * (double)qj / cd.py);
            const bool same = pi == pj && qi == qj;
            const cplx g = (si >= 0 && sj >= 0) ? G[(size_t)si * st + sj] : C(0.0, 0.0);
            cplx mv, kv;
            if (ui && uj) {
                mv = cscale(Eu[(size_t)li * su + lj], w2);
                if (sj >= 0) mv = cadd(mv, cscale(Yt[(size_t)li * st + sj], kyj));
                if (i == j) mv.x -= kxi * kxi;
                kv = cscale(g, -kyi * kyj);
                if (i == j) kv.x += w2;
            } else if (ui) {
                mv = sj >= 0 ? cscale(Yt[(size_t)li * st + sj], -kxj) : C(0.0, 0.0);
                if (same) mv.x -= kxi * kyi;
                kv = cscale(g, kyi * kxj);
            } else if (uj) {
                mv = sj >= 0 ? cscale(Yb[(size_t)li * st + sj], kyj) : C(0.0, 0.0);
                if (same) mv.x -= kyi * kxi;
                kv = cscale(g, kxi * kyj);
            } else {
                mv = cscale(Ev[(size_t)li * sv + lj], w2);
                if (sj >= 0) mv = csub(mv, cscale(Yb[(size_t)li * st + sj], kxj));
                if (i == j) mv.x -= kyi * kyi;
                kv = cscale(g, -kxi * kxj);
                if (i == j) kv.x += w2;
            }
            Mc[e] = mv;
            Kp[e] = kv;
            cplx h0 = C(0.0, 0.0), hs = C(0.0, 0.0);
            if (same) {  // the representative order (|p|, |q|) of the orbit, in each field block
                const int o = (pi + Mx) * ny + (qi + My);
                const int k = (ui ? 0 : N) + o, l = (uj ? 0 : N) + o;
                h0 = halfspace_entry(b, cd, 0, k, l);
                hs = halfspace_entry(b, cd, 1, k, l);
            }
            C0[e] = h0;
            Ks[e] = hs;
        }
    }
}

// Class S-matrix solves by Gauss-Jordan in shared memory when the widest
// augmented system [T11 | -T12 D | a0] (m x (2m + 1)) fits in 128 KB (classes
// up to m = 61, M <= 5 on square cells); larger classes use the blocked LU.
__host__ __device__ constexpr size_t sym_gj_bytes(int m) {
    return ((size_t)m * (2 * m + 2) + 2 * (2 * m + 1) + 1) * 16 + 16;
}
__host__ __device__ constexpr bool sym_gj_fits(int m) { return sym_gj_bytes(m) <= 128 * 1024; }

// The S-matrix of one excited class: rcwa_smat1 and rcwa_smat2 restricted to
// the class, with the class's one excitation (class 0: Y, a0 = -e_i0; class 1:
// X, a0 = e_{N+i0}, rcwa2d.cpp:403-411). In the class basis the half-spaces'
// phi stays I and their kz stays diagonal (kz is even in p and q), so the
// reference's recursion carries over with every matrix of order m:
//   A = kp W,  P = C0 A diag(1/q),  T11 = (W + P)/2,  T12 = (W - P)/2,
//   [S12 | u] = T11^-1 [-T12 D | a0],
//   Q = diag(q) A^-1 Ks W,  (I + Q - D S12 + D S12 Q) y = 2 D u,
//   aN = W y,  y2 = (y - Q y)/2,  b0 = T12 (u + S12 y2) + T11 D y2.
// Writes aN and b0 (class basis) to the class vector area.
// dynamic smem: sym_smat_smem(m) (LU staging, or the Gauss-Jordan systems)
__global__ void __launch_bounds__(kRT) rcwa_sym_smat(Bucket b) {
    extern __shared__ __align__(16) unsigned char smem[];
    cplx* stg = reinterpret_cast<cplx*>(smem);
    __shared__ GemmSmem gs;
    __shared__ RedScratch rs;
    const int mi = blockIdx.x, cell = mi / b.ncls, c = b.cls0 + mi % b.ncls;
    const CellDev cd = b.cells[cell];
    const int m = b.m[0], N = b.N, Mx = b.Mx, My = b.My;
    const int tid = threadIdx.x, nt = blockDim.x;
    const size_t o2 = (size_t)mi * m * m;
    const cplx* W = b.sW[0] + o2;
    const cplx* q = b.sq[0] + (size_t)mi * m;
    const cplx *Kp = b.cKp + o2, *C0 = b.cC0 + o2, *Ks = b.cKs + o2;
    cplx *A = b.cA + o2, *T11 = b.cT11 + o2, *T11lu = b.cT11lu + o2, *T12 = b.cT12 + o2;
    cplx *Q = b.cQ + o2, *SQ = b.cSQ + o2, *Cm = b.cCm + o2;
    cplx* S = b.cS12 + (size_t)mi * m * (m + 1);
    cplx* vec = b.cvec + (size_t)mi * 8 * m;  // aN | b0 | y | Q y | y2 | u + S12 y2 | D y2
    int* piv = b.cpiv + (size_t)mi * m;
    const int ld = m + 1;
    const cplx one = C(1.0, 0.0), zero = C(0.0, 0.0);
    // stage clocks: per-phase clock64 sums in slots 16.. of the cell's counters
    long long* pf = (b.dbg && tid == 0) ? b.dbg + kDbgSlots * (size_t)mi + 16 : nullptr;
    long long tp = clock64();
    auto phase = [&](int k) {
        if (pf) {
            const long long t = clock64();
            pf[k] += t - tp;
            tp = t;
        }
    };
    // A = kp W, then P = C0 A (into T12), T11 = (W + P diag(1/q))/2, T12 = (W - P diag(1/q))/2
    blk_gemm(m, m, m, one, Kp, m, W, m, zero, A, m, &gs);
    blk_gemm(m, m, m, one, C0, m, A, m, zero, T12, m, &gs);
    for (int e = tid; e < m * m; e += nt) {
        const cplx p = cmul(T12[e], cinv(q[e % m]));
        const cplx w = W[e];
        const cplx t = cscale(cadd(w, p), 0.5);
        T11[e] = t;
        T11lu[e] = t;
        T12[e] = cscale(csub(w, p), 0.5);
    }
    __syncthreads();
    // [-T12 D | a0]: a0 of the class's excitation in the class basis
    const int i0 = Mx * (2 * My + 1) + My;
    const int k0 = c == 1 ? N + i0 : i0;
    const double s0 = c == 1 ? 1.0 : -1.0;
    for (int e = tid; e < m * ld; e += nt) {
        const int i = e / ld, j = e % ld;
        cplx v;
        if (j < m) {
            v = cneg(cmul(T12[(size_t)i * m + j], cexpi(cscale(q[j], cd.h))));
        } else {
            int ii[4];
            double ci[4];
            const int ni = sym_vector(Mx, My, c, i, ii, ci);
            double a = 0.0;
            for (int u = 0; u < ni; ++u)
                if (ii[u] == k0) a += s0 * ci[u];
            v = C(a, 0.0);
        }
        S[e] = v;
    }
    __syncthreads();
    phase(0);
    const bool gj = sym_gj_fits(m);
    const int lg = 2 * m + 1;  // the augmented systems' row stride in shared memory (odd)
    cplx* gscr = stg + (size_t)m * lg;
    int* gsp = reinterpret_cast<int*>(gscr + 2 * (2 * m + 1) + 1);
    // [A | X] (X: nx columns of a global row-major array, ldx) -> X <- A^-1 X in shared memory
    auto gj_solve = [&](const cplx* Am, int lda, cplx* X, int ldx, int nx) {
        const int w = m + nx;
        for (int e = tid; e < m * w; e += nt) {
            const int i = e / w, j = e % w;
            stg[i * lg + j] = j < m ? Am[(size_t)i * lda + j] : X[(size_t)i * ldx + j - m];
        }
        const int inf = blk_gj_solve_smem(m, nx, stg, lg, gscr, gsp);
        if (tid == 0 && inf) atomicCAS(&b.info[cell], 0, -inf);
        for (int e = tid; e < m * nx; e += nt) X[(size_t)(e / nx) * ldx + e % nx] = stg[(e / nx) * lg + m + e % nx];
        __syncthreads();
    };
    int info = 0;
    if (gj) {
        gj_solve(T11, m, S, ld, m + 1);  // [S12 | u]
        phase(1);
    } else {
        info = blk_lu_blocked(m, T11lu, m, piv, &rs, stg, &gs);
        if (tid == 0 && info) atomicCAS(&b.info[cell], 0, -info);
        __syncthreads();
        phase(1);
        blk_lu_solve_blocked(m, T11lu, m, piv, ld, S, ld, stg, &gs);  // [S12 | u]
    }
    __syncthreads();
    phase(2);
    // interface to the substrate: Q = diag(q) A^-1 Ks W
    blk_gemm(m, m, m, one, Ks, m, W, m, zero, Q, m, &gs);
    __syncthreads();
    phase(3);
    if (gj) {
        gj_solve(A, m, Q, m, m);
        phase(4);
    } else {
        info = blk_lu_blocked(m, A, m, piv, &rs, stg, &gs);
        if (tid == 0 && info) atomicCAS(&b.info[cell], 0, -info);
        __syncthreads();
        phase(4);
        blk_lu_solve_blocked(m, A, m, piv, m, Q, m, stg, &gs);
    }
    __syncthreads();
    phase(5);
    for (int e = tid; e < m * m; e += nt) Q[e] = cmul(q[e / m], Q[e]);
    blk_gemm(m, m, m, one, S, ld, Q, m, zero, SQ, m, &gs);  // S12 Q
    __syncthreads();
    phase(6);
    cplx *aN = vec, *b0 = vec + m, *y = vec + 2 * m, *Qy = vec + 3 * m, *y2 = vec + 4 * m, *zz = vec + 5 * m,
         *dy2 = vec + 6 * m;
    for (int e = tid; e < m * m; e += nt) {
        const int i = e / m, j = e % m;
        const cplx d = cexpi(cscale(q[i], cd.h));
        cplx v = cadd(Q[e], cmul(d, csub(SQ[e], S[(size_t)i * ld + j])));
        if (i == j) v.x += 1.0;
        Cm[e] = v;
    }
    for (int i = tid; i < m; i += nt) y[i] = cscale(cmul(cexpi(cscale(q[i], cd.h)), S[(size_t)i * ld + m]), 2.0);
    __syncthreads();
    if (gj) {
        gj_solve(Cm, m, y, 1, 1);  // y
    } else {
        info = blk_lu_blocked(m, Cm, m, piv, &rs, stg, &gs);
        if (tid == 0 && info) atomicCAS(&b.info[cell], 0, -info);
        blk_lu_solve_blocked(m, Cm, m, piv, 1, y, 1, stg, &gs);  // y
    }
    blk_gemm(m, 1, m, one, W, m, y, 1, zero, aN, 1, &gs);    // aN = W y
    blk_gemm(m, 1, m, one, Q, m, y, 1, zero, Qy, 1, &gs);    // Q y
    for (int i = tid; i < m; i += nt) {
        const cplx v = cscale(csub(y[i], Qy[i]), 0.5);
        y2[i] = v;
        zz[i] = S[(size_t)i * ld + m];                              // u
        dy2[i] = cmul(cexpi(cscale(q[i], cd.h)), v);                // D y2
    }
    blk_gemm(m, 1, m, one, S, ld, y2, 1, one, zz, 1, &gs);    // u + S12 y2
    blk_gemm(m, 1, m, one, T12, m, zz, 1, zero, b0, 1, &gs);  // T12 (u + S12 y2)
    blk_gemm(m, 1, m, one, T11, m, dy2, 1, one, b0, 1, &gs);  // + T11 D y2
    __syncthreads();
    phase(7);
}

// aN and b0 of both excitations into the full basis (the vector area the
// epilogue reads: aN_X, aN_Y, b0_X, b0_Y); a class eigensolve failure becomes
// the cell's info (it is the cause of any later singular pivot).
__global__ void __launch_bounds__(kRT) rcwa_sym_expand(Bucket b) {
    const int cell = blockIdx.x;
    const int N = b.N, n = b.n, Mx = b.Mx, My = b.My, m = b.m[0], ny = 2 * My + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    cplx* vec = at(b.vec, 10 * b.s_n, cell);
    for (int e = tid; e < 4 * (int)b.s_n; e += nt) vec[e] = C(0.0, 0.0);
    __syncthreads();
    for (int cc = 0; cc < b.ncls; ++cc) {
        const int c = b.cls0 + cc, mi = b.ncls * cell + cc;
        const cplx* cv = b.cvec + (size_t)mi * 8 * m;
        cplx* dst_a = vec + (c == 1 ? 0 : b.s_n);       // aN_X : aN_Y
        cplx* dst_b = vec + (c == 1 ? 2 : 3) * b.s_n;   // b0_X : b0_Y
        for (int i = tid; i < m; i += nt) {
            int ii[4];
            double ci[4];
            const int ni = sym_vector(Mx, My, c, i, ii, ci);
            for (int u = 0; u < ni; ++u) {
                dst_a[ii[u]] = cscale(cv[i], ci[u]);
                dst_b[ii[u]] = cscale(cv[m + i], ci[u]);
            }
        }
    }
    if (b.ncls == 1) {
        // C4-symmetric cell: the Y solution is the X solution rotated by 90
        // degrees, R e_k = sigma(k) e_{rho k}: rho(u at (p, q)) = v at (-q, p)
        // with sigma = +1, rho(v at (p, q)) = u at (-q, p) with sigma = -1
        __syncthreads();
        for (int k = tid; k < n; k += nt) {
            const int bk = k / N, ok = k % N;
            const int pk = ok / ny - Mx, qk = ok % ny - My;
            const int rk = (1 - bk) * N + (-qk + Mx) * ny + (pk + My);
            const double sg = bk == 1 ? -1.0 : 1.0;
            vec[b.s_n + rk] = cscale(vec[k], sg);
            vec[3 * b.s_n + rk] = cscale(vec[2 * b.s_n + k], sg);
        }
    }
    if (tid == 0 && b.info[cell] != kInfoAsym) {
        for (int cc = 0; cc < b.ncls; ++cc) {
            const int e = b.sinfo[0][b.ncls * cell + cc];
            if (e != 0) {
                b.info[cell] = e;
                break;
            }
        }
    }
}

// The eigen-stage bucket of size class k of a mirror-symmetric bucket.
Bucket sym_eig_bucket(const Bucket& b, int k) {
    Bucket e;
    std::memset(&e, 0, sizeof(e));
    e.Mx = b.Mx;
    e.My = b.My;
    e.n = b.m[k];
    e.N = e.n / 2;
    e.ncell = b.ncls * b.ncell;
    e.cells = b.cells;
    e.H = b.sH[k];
    e.Z = b.sZ[k];
    e.X = b.sX[k];
    e.W = b.sW[k];
    e.A = b.sA[k];
    e.q1 = b.sq[k];
    e.info = b.sinfo[k];
    e.dbg = b.dbg;  // the stage-clock counters hold 2 slots per cell
    e.s_nn = (size_t)e.n * e.n;
    e.s_n = (size_t)e.n;
    return e;
}

// ---- host side ------------------------------------------------------------------------------------
struct HostCell {
    CellDev d;
    int Mx, My, ng;  // ng = 0: analytic rect path
    int index;       // position in the caller's array
    int sym;         // 1: mirror-symmetric cell at normal incidence (eigenproblem in parity classes)
};

// The parity-class eigensolve applies to unrotated shapes (all mirror
// symmetric, rcwa2d.cpp:37-72) at normal incidence with at least one order on
// each side of 0 in x and y; CELERIS_RCWA_SYMMETRY=0 turns it off.
bool symmetry_enabled() {
    const char* e = std::getenv("CELERIS_RCWA_SYMMETRY");
    return !(e && e[0] == '0');
}
// Mirror-asymmetry tolerance of the class split, relative to the largest entry
// of each eps operator (Exx, Eyy, Einv and the Laurent coefficients): rounding
// leaves ~1e-15; one raster sample on the other side of a shape boundary
// ~1e-6. CELERIS_RCWA_SYM_TOL overrides it (the test is strict, so 0 sends
// every cell to the full eigensolve through the fallback, for tests of that path).
double symmetry_tolerance() {
    const char* e = std::getenv("CELERIS_RCWA_SYM_TOL");
    return e ? std::atof(e) : 1e-9;
}
bool sym_eligible(const celeris_rcwa_cell& c) {
    return c.theta_rad == 0.0 && c.rotation_rad == 0.0 && c.Mx >= 1 && c.My >= 1 && symmetry_enabled();
}

int validate(const celeris_rcwa_cell& c) {
    // every real input must be finite: a NaN or Inf would run through the
    // eigensolve and come out as a silent non-finite t, R, T
    const double v[] = {c.period_x_um, c.period_y_um, c.wavelength_um, c.theta_rad, c.phi_rad,
                        c.n_inc[0], c.n_inc[1], c.n_sub[0], c.n_sub[1], c.eps_pillar[0], c.eps_pillar[1],
                        c.eps_bg[0], c.eps_bg[1], c.fill_x, c.fill_y, c.thickness_um, c.shape_param,
                        c.rotation_rad};
    for (double x : v)
        if (!std::isfinite(x)) return set_error(CELERIS_ERR_INVALID_ARG, "cell parameter is NaN or Inf");
    if (c.Mx < 0 || c.My < 0) return set_error(CELERIS_ERR_INVALID_ARG, "M must be >= 0");
    if (c.Mx > 15 || c.My > 15) return set_error(CELERIS_ERR_TOO_LARGE, "Mx, My <= 15 supported");
    if (!(c.wavelength_um > 0) || !(c.period_x_um > 0) || !(c.period_y_um > 0))
        return set_error(CELERIS_ERR_INVALID_ARG, "wavelength and periods must be > 0");
    if (c.shape < 0 || c.shape > 3) return set_error(CELERIS_ERR_INVALID_ARG, "unknown shape %d", c.shape);
    const int n = 2 * (2 * c.Mx + 1) * (2 * c.My + 1);
    if (n > kMaxN) return set_error(CELERIS_ERR_TOO_LARGE, "2N = %d > %d", n, kMaxN);
    if (c.grid > 1024) return set_error(CELERIS_ERR_TOO_LARGE, "grid %d > 1024", c.grid);
    return CELERIS_OK;
}

HostCell make_cell(const celeris_rcwa_cell& c, int index, double ex_re, double ex_im, double ey_re, double ey_im,
                   int nexc) {
    HostCell h;
    std::memset(&h, 0, sizeof(h));
    CellDev& d = h.d;
    d.omega = 2.0 * PI / c.wavelength_um;
    d.px = c.period_x_um;
    d.py = c.period_y_um;
    d.h = c.thickness_um;
    d.theta = c.theta_rad;
    d.fill_x = c.fill_x;
    d.fill_y = c.fill_y;
    d.shape_param = c.shape_param;
    d.rot = c.rotation_rad;
    const double ni_r = c.n_inc[0], ni_i = c.n_inc[1];
    const double st = std::sin(c.theta_rad);
    // kx0 = n_inc sin(theta) cos(phi) omega (rcwa2d.cpp:234-235)
    const double fx = st * std::cos(c.phi_rad) * d.omega, fy = st * std::sin(c.phi_rad) * d.omega;
    d.kx0 = make_double2(ni_r * fx, ni_i * fx);
    d.ky0 = make_double2(ni_r * fy, ni_i * fy);
    d.eps_p = make_double2(c.eps_pillar[0], c.eps_pillar[1]);
    d.eps_b = make_double2(c.eps_bg[0], c.eps_bg[1]);
    d.n_inc = make_double2(c.n_inc[0], c.n_inc[1]);
    d.n_sub = make_double2(c.n_sub[0], c.n_sub[1]);
    d.ex0 = make_double2(ex_re, ex_im);
    d.ey0 = make_double2(ey_re, ey_im);
    d.shape = c.shape;
    d.nexc = nexc;
    h.Mx = c.Mx;
    h.My = c.My;
    const bool plain_rect = c.shape == CELERIS_SHAPE_RECT && c.rotation_rad == 0.0 && !c.force_laurent;
    // reference raster size max(128, 8(2 max(Mx, My) + 1)) (rcwa2d.cpp:337)
    h.ng = plain_rect ? 0 : (c.grid > 0 ? c.grid : std::max(128, 8 * (2 * std::max(c.Mx, c.My) + 1)));
    h.index = index;
    // 2: also symmetric under the 90 degree rotation (square period, Mx = My,
    // fill_x = fill_y; every shape of rcwa2d.cpp:37-72 is then C4 symmetric):
    // the Y solution is the rotated X solution and one class is solved
    h.sym = !sym_eligible(c) ? 0
            : (c.period_x_um == c.period_y_um && c.Mx == c.My && c.fill_x == c.fill_y) ? 2 : 1;
    return h;
}

// Shared memory of the Schur kernel: two CTAs fit per SM with sizeof(AedShared);
// a launch with no more cells than SMs asks for more than half an SM's shared
// memory so that the cells spread one per SM instead of pairing up.
constexpr size_t kSchurSmemOneCta = 120 * 1024;
static_assert(sizeof(AedShared) <= kSchurSmemOneCta, "Schur shared block");
size_t schur_smem(int ncell) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
    }
    return ncell <= sms ? kSchurSmemOneCta : sizeof(AedShared);
}

// staging of blk_hessenberg_blocked
// Threads of the shared-memory Hessenberg kernel: 512 once H no longer lets
// two CTAs share an SM (order > 80), else the tuned size.
int hess_smem_threads(int n, int tuned) {
    return (size_t)n * n * sizeof(cplx) > 100 * 1024 ? kHessBigThreads : tuned;
}
size_t hess_stage_bytes(int n) { return (size_t)(n + LNB * LNB + 2 * LNB) * sizeof(cplx); }

// staging of blk_lu_blocked and the matvecs of the S-matrix kernels
size_t lu_stage_bytes(int n) { return (size_t)(2 * n + LNB * LNB) * sizeof(cplx); }

// dynamic shared memory of rcwa_sym_smat for class order m
size_t sym_smat_smem(int m) {
    return std::max(lu_stage_bytes(m), sym_gj_fits(m) ? sym_gj_bytes(m) : (size_t)0);
}

size_t laurent_smem(int Mx, int My, int ng) {
    const size_t mx4 = 4 * Mx + 1, my4 = 4 * My + 1;
    const int N = (2 * Mx + 1) * (2 * My + 1);
    const size_t raster = ((size_t)laurent_g1_rows(Mx) * ng + mx4 * my4) * sizeof(cplx) + (size_t)ng * ng;
    // the class path inverts its largest scalar parity block in place: s x (s + 1)
    // + 2 s + 1 complex, s + 1 ints
    const size_t sb = (size_t)(Mx + 1) * (My + 1);
    const size_t gj = (sb * (sb + 1) + 2 * sb + 1) * sizeof(cplx) + (sb + 1) * sizeof(int);
    return std::max(std::max(raster, gj), lu_stage_bytes(N) + sizeof(GemmSmem));
}

// ---- stage configuration and autotuning -------------------------------------------------
// Every stage kernel runs with blockDim in {128, 256} (they are written for any
// multiple of 32 >= 128). For each bucket shape (Mx, My, raster) the first batch
// that meets it times every stage at both sizes on the bucket's own cells and
// keeps the faster size per stage; the table lives for the process and can be
// read with celeris_rcwa_tuning_report. CELERIS_RCWA_AUTOTUNE=0 disables it
// (all stages at 256 threads).
enum Stage { ST_FOURIER, ST_BUILD, ST_HESS, ST_SCHUR, ST_VEC, ST_SMAT1, ST_SMAT2, ST_EPI, ST_COUNT };
const char* const kStageNames[ST_COUNT] = {"fourier", "build_M", "hessenberg", "schur", "eigvec",
                                           "smat1", "smat2", "epilogue"};
constexpr int kCand[2] = {128, 256};
struct StageCfg {
    int threads[ST_COUNT];
};
StageCfg uniform_cfg(int t) {
    StageCfg c;
    for (int i = 0; i < ST_COUNT; ++i) c.threads[i] = t;
    return c;
}

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, StageCfg>& tune_table() {
    static auto* m = new std::map<std::tuple<int, int, int>, StageCfg>();
    return *m;
}
bool tuning_enabled() {
    const char* e = std::getenv("CELERIS_RCWA_AUTOTUNE");
    return !(e && e[0] == '0');
}

struct BucketPlan {
    int Mx, My, ng, N, n, sym;
    std::vector<int> ids;  // indices into the cell list
    size_t per_cell = 0, bytes = 0;
    Bucket b;
};

size_t per_cell_bytes(int n, int nexc) {
    const int N = n / 2;
    const size_t s_nn = (size_t)n * n, s_ns = (size_t)n * (n + 2), s_NN = (size_t)N * N, s_n = (size_t)n;
    return celeris_rt::align256((8 * s_nn + s_ns + 3 * s_NN + 11 * s_n) * sizeof(cplx)) +
           celeris_rt::align256(s_n * sizeof(int)) + 256 + celeris_rt::align256(sizeof(celeris_rcwa_result) * nexc) +
           celeris_rt::align256(sizeof(CellDev)) + 14 * 256;
}

// Device memory of one mirror-symmetric cell: of the full-order buffers only
// H (M, and the Laurent LU scratch), Z, X (build_M's products), the Fourier
// operators, the vector area and pivots; per excited class (two per cell) the
// eigen-stage matrices H, Z, X, W, scratch, q and info, and the class S-matrix's
// ten m x m matrices, S12 (m x (m + 1)), 8 m vector entries and m pivots.
size_t sym_per_cell_bytes(int Mx, int My, int nexc, int ncls) {
    const int N = (2 * Mx + 1) * (2 * My + 1), n = 2 * N;
    const size_t m = (size_t)sym_class_size(Mx, My, 0);
    const size_t full = (3 * (size_t)n * n + 3 * (size_t)N * N + 10 * (size_t)n) * sizeof(cplx) +
                        (size_t)n * sizeof(int) + sizeof(int) + sizeof(celeris_rcwa_result) * nexc + sizeof(CellDev);
    const size_t cls = ncls * (((5 * m * m + m) * sizeof(cplx) + sizeof(int)) +
                               ((10 * m * m + m * (m + 1) + 8 * m) * sizeof(cplx) + m * sizeof(int)));
    return full + cls + 32 * 256;
}

// The largest dynamic shared memory each stage kernel needs over a wave's
// buckets; raised once per wave, outside any capture.
struct SmemNeeds {
    size_t laurent = 0, rect = 0, hess_s = 0, hess_g = 0, smat = 0, smat_sym = 0;
    bool aed = false;
    void add_eig(int n) {
        if (n <= kSmemEigMaxN) hess_s = std::max(hess_s, ((size_t)n * n + 2 * n) * sizeof(cplx));
        else hess_g = std::max(hess_g, hess_stage_bytes(n));
        aed = true;
    }
    void add(int Mx, int My, int ng, int n, int sym = 0) {
        if (ng > 0) {
            laurent = std::max(laurent, laurent_smem(Mx, My, ng));
        } else {
            const int nx = 2 * Mx + 1, ny = 2 * My + 1;
            rect = std::max(rect, ((size_t)2 * (nx * nx + ny * ny) + 2 * std::max(nx, ny)) * sizeof(cplx));
        }
        if (sym) {
            add_eig(sym_class_size(Mx, My, 0));
            smat_sym = std::max(smat_sym, sym_smat_smem(sym_class_size(Mx, My, 0)));
        } else {
            add_eig(n);
            smat = std::max(smat, lu_stage_bytes(n));
        }
    }
};

// Dynamic shared-memory limits are per kernel function and process-wide, so
// they only ever grow: a call that needs less never lowers the limit another
// thread's launch relies on (a larger limit does not change a launch that asks
// for less).
int raise_dyn_smem(const void* fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> cur;
    int dev = 0;
    CEL_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t& c = cur[{dev, fn}];
    if (bytes <= c) return CELERIS_OK;
    CEL_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    c = bytes;
    return CELERIS_OK;
}

int set_smem_limits(const SmemNeeds& s) {
    if (s.laurent)
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_fourier_laurent), s.laurent));
    if (s.rect)
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_fourier_rect), s.rect));
    if (s.aed)
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_schur), kSchurSmemOneCta));
    if (s.hess_g)
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_hess<false>), s.hess_g));
    if (s.hess_s) {
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_hess<true>), s.hess_s));
    }
    if (s.smat) {
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_smat1), s.smat));
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_smat2), s.smat));
    }
    if (s.smat_sym) CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_sym_smat), s.smat_sym));
    return CELERIS_OK;
}

// Launch the stage sequence of one bucket on `st`. ev (ST_COUNT + 1 events) is
// optional: stage boundaries are recorded into it.
// eig_only: stop after the eigenvectors (the layers of a multi-layer stack).
void launch_bucket(const Bucket& b, const StageCfg& cfg, cudaStream_t st, cudaEvent_t* ev, bool eig_only = false) {
    const int nc = b.ncell, n = b.n;
    const int* T = cfg.threads;
    if (ev) cudaEventRecord(ev[0], st);
    cudaMemsetAsync(b.info, 0, sizeof(int) * nc, st);
    if (b.ng > 0) {
        const int Mx = b.Mx, My = b.My, ng = b.ng;
        rcwa_phase_table<<<((4 * Mx + 1) * ng + 255) / 256, 256, 0, st>>>(ng, 2 * Mx, const_cast<cplx*>(b.phx));
        rcwa_phase_table<<<((4 * My + 1) * ng + 255) / 256, 256, 0, st>>>(ng, 2 * My, const_cast<cplx*>(b.phy));
        rcwa_fourier_laurent<<<nc, T[ST_FOURIER], laurent_smem(Mx, My, ng), st>>>(b);
        count_launch(3);
    } else {
        const int nx = 2 * b.Mx + 1, ny = 2 * b.My + 1;
        const size_t sm = ((size_t)2 * (nx * nx + ny * ny) + 2 * std::max(nx, ny)) * sizeof(cplx);
        rcwa_fourier_rect<<<nc, T[ST_FOURIER], sm, st>>>(b);
        count_launch(1);
    }
    if (ev) cudaEventRecord(ev[1], st);
    if (b.sym) {
        // the excited parity classes: their operators (in place of build_M),
        // eigen-stages (ncls matrices of order m[0] per cell), the class
        // S-matrix, expand into the epilogue's vectors
        rcwa_sym_build<<<nc, T[ST_BUILD], 0, st>>>(b);
        if (ev) cudaEventRecord(ev[2], st);
        const Bucket e = sym_eig_bucket(b, 0);
        cudaMemsetAsync(e.info, 0, sizeof(int) * e.ncell, st);
        const int m = e.n;
        if (m <= kSmemEigMaxN)
            rcwa_hess<true><<<e.ncell, hess_smem_threads(m, T[ST_HESS]), ((size_t)m * m + 2 * m) * sizeof(cplx),
                              st>>>(e);
        else
            rcwa_hess<false><<<e.ncell, T[ST_HESS], hess_stage_bytes(m), st>>>(e);
        if (ev) cudaEventRecord(ev[3], st);
        rcwa_schur<<<e.ncell, kSchurThreads, schur_smem(e.ncell), st>>>(e);
        if (ev) cudaEventRecord(ev[4], st);
        rcwa_vec<<<e.ncell, T[ST_VEC], 0, st>>>(e);
        if (ev) cudaEventRecord(ev[5], st);
        rcwa_sym_smat<<<e.ncell, T[ST_SMAT1], sym_smat_smem(m), st>>>(b);
        if (ev) cudaEventRecord(ev[6], st);
        rcwa_sym_expand<<<nc, T[ST_SMAT2], 0, st>>>(b);
        if (ev) cudaEventRecord(ev[7], st);
        rcwa_epilogue<<<nc, T[ST_EPI], 0, st>>>(b);
        if (ev) cudaEventRecord(ev[8], st);
        count_launch(7);
        return;
    }
    rcwa_build_M<<<nc, T[ST_BUILD], 0, st>>>(b, b.ng > 0 ? 1 : 0);
    if (ev) cudaEventRecord(ev[2], st);
    if (n <= kSmemEigMaxN) {
        const size_t sm = ((size_t)n * n + 2 * n) * sizeof(cplx);
        rcwa_hess<true><<<nc, hess_smem_threads(n, T[ST_HESS]), sm, st>>>(b);
        if (ev) cudaEventRecord(ev[3], st);
        rcwa_schur<<<nc, kSchurThreads, schur_smem(nc), st>>>(b);
    } else {
        rcwa_hess<false><<<nc, T[ST_HESS], hess_stage_bytes(n), st>>>(b);
        if (ev) cudaEventRecord(ev[3], st);
        rcwa_schur<<<nc, kSchurThreads, schur_smem(nc), st>>>(b);
    }
    if (ev) cudaEventRecord(ev[4], st);
    rcwa_vec<<<nc, T[ST_VEC], 0, st>>>(b);
    if (ev) cudaEventRecord(ev[5], st);
    if (eig_only) {
        count_launch(4);
        return;
    }
    const size_t sm_stage = lu_stage_bytes(n);
    rcwa_smat1<<<nc, T[ST_SMAT1], sm_stage, st>>>(b);
    if (ev) cudaEventRecord(ev[6], st);
    rcwa_smat2<<<nc, T[ST_SMAT2], sm_stage, st>>>(b);
    if (ev) cudaEventRecord(ev[7], st);
    rcwa_epilogue<<<nc, T[ST_EPI], 0, st>>>(b);
    if (ev) cudaEventRecord(ev[8], st);
    count_launch(7);
}

// Time each stage at every candidate size on (up to) the first 2 x SMs cells
// of the bucket; keep the faster size per stage.
int autotune(const BucketPlan& p, cudaStream_t st, StageCfg* out) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    Bucket t = p.b;
    t.ncell = std::min(t.ncell, 2 * sms);
    cudaEvent_t ev[ST_COUNT + 1];
    for (auto& e : ev) CEL_CUDA(cudaEventCreate(&e));
    float best[ST_COUNT];
    StageCfg cfg = uniform_cfg(256);
    for (int c = 0; c < 2; ++c) {
        launch_bucket(t, uniform_cfg(kCand[c]), st, ev);
        CEL_CUDA(cudaStreamSynchronize(st));
        for (int s = 0; s < ST_COUNT; ++s) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[s], ev[s + 1]);
            if (c == 0 || ms < best[s]) {
                best[s] = ms;
                cfg.threads[s] = kCand[c];
            }
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    CEL_CUDA(cudaGetLastError());
    *out = cfg;
    return CELERIS_OK;
}

// Per-thread execution context: streams, pinned staging and the cached graph.
// The device objects follow the thread's current device (rebuilt when it
// changes) and are released, with the main stream's workspace arena, when the
// thread exits.
struct BatchCtx {
    int dev = -1;
    cudaStream_t main = nullptr;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> fork, join;
    void* pinned = nullptr;
    size_t pinned_cap = 0;
    cudaGraphExec_t exec = nullptr;
    std::string sig;
    uint64_t nkern = 0;  // kernels per graph launch

    void drop_device_objects() {
        if (!main) return;
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(dev);
        cudaStreamSynchronize(main);
        for (cudaStream_t s : side) cudaStreamSynchronize(s);
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        sig.clear();
        Workspace::release_stream(main);
        for (cudaStream_t s : side) {
            Workspace::release_stream(s);
            cudaStreamDestroy(s);
        }
        for (cudaEvent_t e : fork) cudaEventDestroy(e);
        for (cudaEvent_t e : join) cudaEventDestroy(e);
        cudaStreamDestroy(main);
        side.clear();
        fork.clear();
        join.clear();
        main = nullptr;
        dev = -1;
        cudaSetDevice(cur);
        cudaGetLastError();  // a failure here (e.g. the runtime shutting down) is nobody's call's error
    }
    ~BatchCtx() {
        drop_device_objects();
        if (pinned) cudaFreeHost(pinned);
        cudaGetLastError();
    }
};
thread_local BatchCtx t_ctx;

int ensure_streams(int nb) {
    BatchCtx& c = t_ctx;
    int cur = 0;
    CEL_CUDA(cudaGetDevice(&cur));
    if (c.main && c.dev != cur) c.drop_device_objects();
    if (!c.main) {
        CEL_CUDA(cudaStreamCreateWithFlags(&c.main, cudaStreamNonBlocking));
        c.dev = cur;
    }
    while ((int)c.side.size() < nb) {
        cudaStream_t s;
        cudaEvent_t f, j;
        CEL_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        CEL_CUDA(cudaEventCreateWithFlags(&f, cudaEventDisableTiming));
        CEL_CUDA(cudaEventCreateWithFlags(&j, cudaEventDisableTiming));
        c.side.push_back(s);
        c.fork.push_back(f);
        c.join.push_back(j);
    }
    return CELERIS_OK;
}

// Free device memory, cached per device for the batch planner.
struct FreeMemCache {
    std::mutex mu;
    std::map<int, std::pair<size_t, std::chrono::steady_clock::time_point>> by_dev;
};
FreeMemCache& free_mem_cache() {
    static FreeMemCache c;
    return c;
}
int query_free_memory(int dev, size_t* free_b) {
    size_t total_b = 0;
    CEL_CUDA(cudaMemGetInfo(free_b, &total_b));
    FreeMemCache& c = free_mem_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    c.by_dev[dev] = {*free_b, std::chrono::steady_clock::now()};
    return CELERIS_OK;
}
// The cached figure if it is under 2 s old, else 0.
size_t cached_free_memory(int dev) {
    FreeMemCache& c = free_mem_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    const auto it = c.by_dev.find(dev);
    if (it == c.by_dev.end()) return 0;
    const double age = std::chrono::duration<double>(std::chrono::steady_clock::now() - it->second.second).count();
    return age < 2.0 ? it->second.first : 0;
}

int run_cells(std::vector<HostCell>& cells, celeris_rcwa_result* out, int* info_out, int nexc) {
    CEL_TRY(celeris_rt::require_device());
    // ---- plan: buckets by (Mx, My, raster), largest first so they start first
    std::map<std::tuple<int, int, int, int>, std::vector<int>> by;
    for (int i = 0; i < (int)cells.size(); ++i)
        by[std::make_tuple(cells[i].Mx, cells[i].My, cells[i].ng, cells[i].sym)].push_back(i);
    std::vector<BucketPlan> plans;
    std::vector<std::vector<int>> waves;
    CEL_TRY(ensure_streams(1));
    int dev = 0, smem_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    Workspace& ws0 = Workspace::for_stream(t_ctx.main);
    // the memory budget: a free-memory figure up to 2 s old is used only when
    // the resulting plan needs no larger arena (no allocation can then fail);
    // the query itself is a driver call that costs ~0.1-1 ms, a sizeable part
    // of a small batch
    bool fresh = false;
    size_t free_b = cached_free_memory(dev);
    if (free_b == 0) {
        CEL_TRY(query_free_memory(dev, &free_b));
        fresh = true;
    }
    auto make_plan = [&](size_t free_now) -> int {
        plans.clear();
        waves.clear();
        const size_t budget = (size_t)(0.6 * (double)(free_now + ws0.capacity()));
        for (auto& kv : by) {
            BucketPlan p;
            p.Mx = std::get<0>(kv.first);
            p.My = std::get<1>(kv.first);
            p.ng = std::get<2>(kv.first);
            p.sym = std::get<3>(kv.first);
            p.N = (2 * p.Mx + 1) * (2 * p.My + 1);
            p.n = 2 * p.N;
            if (p.ng > 0 && laurent_smem(p.Mx, p.My, p.ng) + 1024 > (size_t)smem_optin)
                return set_error(CELERIS_ERR_TOO_LARGE, "raster %d with M=(%d,%d) exceeds shared memory", p.ng, p.Mx, p.My);
            p.per_cell = p.sym ? sym_per_cell_bytes(p.Mx, p.My, nexc, p.sym == 2 ? 1 : 2) : per_cell_bytes(p.n, nexc);
            // split buckets that alone exceed the budget
            const size_t max_cells = std::max<size_t>(1, budget / std::max<size_t>(1, p.per_cell));
            for (size_t c0 = 0; c0 < kv.second.size(); c0 += max_cells) {
                BucketPlan q = p;
                const size_t c1 = std::min(kv.second.size(), c0 + max_cells);
                q.ids.assign(kv.second.begin() + c0, kv.second.begin() + c1);
                q.bytes = q.per_cell * q.ids.size() +
                          (q.ng > 0 ? celeris_rt::align256(((size_t)(4 * q.Mx + 1) + (4 * q.My + 1)) * q.ng *
                                                           sizeof(cplx)) + 512
                                    : 0);
                plans.push_back(q);
            }
        }
        std::sort(plans.begin(), plans.end(), [](const BucketPlan& a, const BucketPlan& b) { return a.n > b.n; });
        // ---- waves of buckets that fit the memory budget together
        size_t acc = 0;
        for (int i = 0; i < (int)plans.size(); ++i) {
            if (waves.empty() || acc + plans[i].bytes > budget) {
                waves.emplace_back();
                acc = 0;
            }
            waves.back().push_back(i);
            acc += plans[i].bytes;
        }
        return CELERIS_OK;
    };
    CEL_TRY(make_plan(free_b));
    if (!fresh) {
        size_t max_need = 0;
        for (const auto& wave : waves) {
            size_t need = 0;
            for (int i : wave) need += plans[i].bytes + 4096;
            max_need = std::max(max_need, need);
        }
        if (max_need > ws0.capacity()) {  // the arena must grow: plan on a fresh figure
            CEL_TRY(query_free_memory(dev, &free_b));
            CEL_TRY(make_plan(free_b));
        }
    }
    std::vector<celeris_rcwa_result> hres(cells.size() * nexc);
    std::vector<int> hinfo(cells.size(), 0);
    const bool prof = std::getenv("CELERIS_RCWA_STAGE_CLOCKS") != nullptr;
    for (const auto& wave : waves) {
        CEL_TRY(ensure_streams((int)wave.size()));
        BatchCtx& ctx = t_ctx;
        cudaStream_t st = ctx.main;
        Workspace& ws = Workspace::for_stream(st);
        size_t need = 0, pin_need = 0;
        for (int i : wave) {
            need += plans[i].bytes + 4096;
            pin_need += celeris_rt::align256(sizeof(CellDev) * plans[i].ids.size()) +
                        celeris_rt::align256(sizeof(celeris_rcwa_result) * nexc * plans[i].ids.size()) +
                        celeris_rt::align256(sizeof(int) * plans[i].ids.size());
        }
        void* old_base = ws.base();
        CEL_TRY(ws.reserve(st, need));
        if (ws.base() != old_base && ctx.exec) {  // the cached graph points at the old arena
            cudaGraphExecDestroy(ctx.exec);
            ctx.exec = nullptr;
            ctx.sig.clear();
        }
        if (ctx.pinned_cap < pin_need) {
            if (ctx.exec) {
                cudaGraphExecDestroy(ctx.exec);
                ctx.exec = nullptr;
                ctx.sig.clear();
            }
            if (ctx.pinned) cudaFreeHost(ctx.pinned);
            ctx.pinned = nullptr;
            ctx.pinned_cap = 0;
            CEL_CUDA(cudaHostAlloc(&ctx.pinned, pin_need, cudaHostAllocDefault));
            ctx.pinned_cap = pin_need;
        }
        // ---- carve the arena and the pinned staging, fill the descriptors
        char* pin = static_cast<char*>(ctx.pinned);
        std::string sig = "n" + std::to_string(nexc);
        std::vector<CellDev*> hdesc(wave.size());
        std::vector<celeris_rcwa_result*> hres_pin(wave.size());
        std::vector<int*> hinfo_pin(wave.size());
        SmemNeeds needs;
        for (size_t w = 0; w < wave.size(); ++w) {
            BucketPlan& p = plans[wave[w]];
            const int nc = (int)p.ids.size();
            Bucket& b = p.b;
            std::memset(&b, 0, sizeof(b));
            b.Mx = p.Mx;
            b.My = p.My;
            b.N = p.N;
            b.n = p.n;
            b.ng = p.ng;
            b.ncell = nc;
            b.s_nn = (size_t)p.n * p.n;
            b.s_ns = (size_t)p.n * (p.n + 2);
            b.s_NN = (size_t)p.N * p.N;
            b.s_n = (size_t)p.n;
            CellDev* dcells = static_cast<CellDev*>(ws.take(sizeof(CellDev) * nc));
            b.cells = dcells;
            // full-order buffers: the class path needs only H, Z, X (M and
            // build_M's products) besides the Fourier operators and vectors
            cplx** mats[] = {&b.H, &b.Z, &b.X, &b.W, &b.A, &b.T11, &b.T11lu, &b.T12};
            for (int k = 0; k < (p.sym ? 3 : 8); ++k) *mats[k] = static_cast<cplx*>(ws.take(sizeof(cplx) * b.s_nn * nc));
            if (!p.sym) b.S12 = static_cast<cplx*>(ws.take(sizeof(cplx) * b.s_ns * nc));
            b.Einv = static_cast<cplx*>(ws.take(sizeof(cplx) * b.s_NN * nc));
            b.Exx = static_cast<cplx*>(ws.take(sizeof(cplx) * b.s_NN * nc));
            b.Eyy = static_cast<cplx*>(ws.take(sizeof(cplx) * b.s_NN * nc));
            if (!p.sym) b.q1 = static_cast<cplx*>(ws.take(sizeof(cplx) * b.s_n * nc));
            b.vec = static_cast<cplx*>(ws.take(sizeof(cplx) * 10 * b.s_n * nc));
            b.piv = static_cast<int*>(ws.take(sizeof(int) * b.s_n * nc));
            b.info = static_cast<int*>(ws.take(sizeof(int) * nc));
            b.res = static_cast<celeris_rcwa_result*>(ws.take(sizeof(celeris_rcwa_result) * nexc * nc));
            if (p.ng > 0) {
                b.phx = static_cast<cplx*>(ws.take(sizeof(cplx) * (4 * p.Mx + 1) * p.ng));
                b.phy = static_cast<cplx*>(ws.take(sizeof(cplx) * (4 * p.My + 1) * p.ng));
            }
            b.sym = p.sym;
            b.sym_tol = symmetry_tolerance();
            if (p.sym) {
                // the two excited classes (order m[0]), two matrices per cell
                b.ncls = p.sym == 2 ? 1 : 2;
                b.cls0 = p.sym == 2 ? 1 : 0;
                const size_t nm = (size_t)b.ncls * nc;  // class matrices in the bucket
                const size_t m = (size_t)sym_class_size(p.Mx, p.My, 0), mm = m * m * nm;
                b.m[0] = (int)m;
                b.m[1] = sym_class_size(p.Mx, p.My, 2);
                cplx** sm[] = {&b.sH[0], &b.sZ[0], &b.sX[0], &b.sW[0], &b.sA[0]};
                for (cplx** x : sm) *x = static_cast<cplx*>(ws.take(sizeof(cplx) * mm));
                b.sq[0] = static_cast<cplx*>(ws.take(sizeof(cplx) * m * nm));
                b.sinfo[0] = static_cast<int*>(ws.take(sizeof(int) * nm));
                cplx** cm[] = {&b.cKp, &b.cC0, &b.cKs, &b.cA, &b.cT11, &b.cT11lu, &b.cT12, &b.cQ, &b.cSQ, &b.cCm};
                for (cplx** x : cm) *x = static_cast<cplx*>(ws.take(sizeof(cplx) * mm));
                b.cS12 = static_cast<cplx*>(ws.take(sizeof(cplx) * m * (m + 1) * nm));
                b.cvec = static_cast<cplx*>(ws.take(sizeof(cplx) * 8 * m * nm));
                b.cpiv = static_cast<int*>(ws.take(sizeof(int) * m * nm));
            }
            hdesc[w] = reinterpret_cast<CellDev*>(pin);
            pin += celeris_rt::align256(sizeof(CellDev) * nc);
            hres_pin[w] = reinterpret_cast<celeris_rcwa_result*>(pin);
            pin += celeris_rt::align256(sizeof(celeris_rcwa_result) * nexc * nc);
            hinfo_pin[w] = reinterpret_cast<int*>(pin);
            pin += celeris_rt::align256(sizeof(int) * nc);
            for (int i = 0; i < nc; ++i) hdesc[w][i] = cells[p.ids[i]].d;
            needs.add(p.Mx, p.My, p.ng, p.n, p.sym);
            sig += "|" + std::to_string(p.Mx) + "," + std::to_string(p.My) + "," + std::to_string(p.ng) + "," +
                   std::to_string(p.sym) + "," + std::to_string(nc) + "," + std::to_string(b.sym_tol);
        }
        CEL_TRY(set_smem_limits(needs));
        // ---- tune unseen bucket shapes (descriptors must be on the device)
        std::vector<StageCfg> cfgs(wave.size(), uniform_cfg(256));
        for (size_t w = 0; w < wave.size(); ++w) {
            const BucketPlan& p = plans[wave[w]];
            // key: shape and batch class (fewer than, or at least, one cell per SM)
            int sms = 148;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            const auto key = std::make_tuple(p.Mx, p.My, 4 * p.ng + 2 * p.sym + ((int)p.ids.size() >= sms ? 1 : 0));
            bool have = false;
            {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                auto it = tune_table().find(key);
                if (it != tune_table().end()) {
                    cfgs[w] = it->second;
                    have = true;
                }
            }
            if (!have && tuning_enabled() && !prof) {
                CEL_CUDA(cudaMemcpyAsync(const_cast<CellDev*>(p.b.cells), hdesc[w], sizeof(CellDev) * p.ids.size(),
                                         cudaMemcpyHostToDevice, st));
                CEL_TRY(autotune(p, st, &cfgs[w]));
                std::lock_guard<std::mutex> lk(g_tune_mu);
                tune_table()[key] = cfgs[w];
            }
            for (int s = 0; s < ST_COUNT; ++s) sig += (cfgs[w].threads[s] == 128 ? "a" : "b");
        }
        if (prof) {
            // diagnostics: one bucket after the other, events per stage
            for (size_t w = 0; w < wave.size(); ++w) {
                BucketPlan& p = plans[wave[w]];
                const int nc = (int)p.ids.size();
                CEL_CUDA(cudaMemcpyAsync(const_cast<CellDev*>(p.b.cells), hdesc[w], sizeof(CellDev) * nc,
                                         cudaMemcpyHostToDevice, st));
                long long* dbg = nullptr;  // 2 nc slots: a class bucket has up to two matrices per cell
                CEL_CUDA(cudaMalloc(&dbg, sizeof(long long) * kDbgSlots * 2 * nc));
                CEL_CUDA(cudaMemsetAsync(dbg, 0, sizeof(long long) * kDbgSlots * 2 * nc, st));
                p.b.dbg = dbg;
                cudaEvent_t ev[ST_COUNT + 1];
                for (auto& e : ev) cudaEventCreate(&e);
                launch_bucket(p.b, cfgs[w], st, ev);
                CEL_CUDA(cudaMemcpyAsync(hres_pin[w], p.b.res, sizeof(celeris_rcwa_result) * nexc * nc,
                                         cudaMemcpyDeviceToHost, st));
                CEL_CUDA(cudaMemcpyAsync(hinfo_pin[w], p.b.info, sizeof(int) * nc, cudaMemcpyDeviceToHost, st));
                CEL_CUDA(cudaStreamSynchronize(st));
                std::vector<long long> h(kDbgSlots * 2 * nc);
                cudaMemcpy(h.data(), dbg, sizeof(long long) * kDbgSlots * 2 * nc, cudaMemcpyDeviceToHost);
                double sw = 0, ph[kDbgSlots] = {};
                for (int i = 0; i < 2 * nc; ++i) {
                    sw += (double)h[kDbgSlots * i + 6];
                    for (int q = 0; q < kDbgSlots; ++q) ph[q] += (double)h[kDbgSlots * i + q];
                }
                std::string line = "[rcwa stages] n=" + std::to_string(p.n) + " cells=" + std::to_string(nc) + " ms:";
                for (int s = 0; s < ST_COUNT; ++s) {
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, ev[s], ev[s + 1]);
                    char buf[64];
                    std::snprintf(buf, sizeof(buf), " %s %.2f", kStageNames[s], ms);
                    line += buf;
                }
                char buf[64];
                std::snprintf(buf, sizeof(buf), " | sweeps/cell %.1f", sw / nc);
                char buf2[640];
                std::snprintf(buf2, sizeof(buf2), " | schur Mcycles/cell: aed %.2f (qr %.2f, %.0f rot) aed_far %.2f sweep %.2f (%.0f steps) sweep_far %.2f small %.2f"
                              " | hess Mcycles/cell: columns %.2f (matvec %.2f) updates %.2f"
                              " | small QR Mcycles/cell: aed chase %.2f deferred %.2f, block chase %.2f deferred %.2f"
                              " | class smat Mcycles/cell: kpW+C0A %.2f LU(T11) %.2f solve %.2f KsW %.2f LU(A) %.2f solve %.2f S12Q %.2f rest %.2f\n",
                              ph[0] / nc * 1e-6, ph[5] / nc * 1e-6, ph[8] / nc, ph[1] / nc * 1e-6, ph[2] / nc * 1e-6,
                              ph[7] / nc, ph[3] / nc * 1e-6, ph[4] / nc * 1e-6, ph[9] / nc * 1e-6, ph[10] / nc * 1e-6,
                              ph[11] / nc * 1e-6, ph[12] / nc * 1e-6, ph[13] / nc * 1e-6, ph[14] / nc * 1e-6,
                              ph[15] / nc * 1e-6, ph[16] / nc * 1e-6, ph[17] / nc * 1e-6, ph[18] / nc * 1e-6,
                              ph[19] / nc * 1e-6, ph[20] / nc * 1e-6, ph[21] / nc * 1e-6, ph[22] / nc * 1e-6,
                              ph[23] / nc * 1e-6);
                std::fprintf(stderr, "%s%s%s", line.c_str(), buf, buf2);
                for (auto& e : ev) cudaEventDestroy(e);
                cudaFree(dbg);
                p.b.dbg = nullptr;
            }
        } else {
            // ---- the whole wave as one CUDA graph: descriptors in, every bucket
            // on its own stream (fork/join), results out; cached per shape.
            if (!ctx.exec || ctx.sig != sig) {
                if (ctx.exec) {
                    cudaGraphExecDestroy(ctx.exec);
                    ctx.exec = nullptr;
                }
                cudaGraph_t graph = nullptr;
                CEL_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                celeris_rt::set_launch_counting(false);
                uint64_t nk = 0;
                for (size_t w = 0; w < wave.size(); ++w) {
                    const BucketPlan& p = plans[wave[w]];
                    const int nc = (int)p.ids.size();
                    cudaStream_t bs = ctx.side[w];
                    cudaEventRecord(ctx.fork[w], st);
                    cudaStreamWaitEvent(bs, ctx.fork[w], 0);
                    cudaMemcpyAsync(const_cast<CellDev*>(p.b.cells), hdesc[w], sizeof(CellDev) * nc,
                                    cudaMemcpyHostToDevice, bs);
                    launch_bucket(p.b, cfgs[w], bs, nullptr);
                    nk += (p.ng > 0 ? 3 : 1) + 7;
                    cudaMemcpyAsync(hres_pin[w], p.b.res, sizeof(celeris_rcwa_result) * nexc * nc,
                                    cudaMemcpyDeviceToHost, bs);
                    cudaMemcpyAsync(hinfo_pin[w], p.b.info, sizeof(int) * nc, cudaMemcpyDeviceToHost, bs);
                    cudaEventRecord(ctx.join[w], bs);
                    cudaStreamWaitEvent(st, ctx.join[w], 0);
                }
                const cudaError_t ce = cudaStreamEndCapture(st, &graph);
                celeris_rt::set_launch_counting(true);
                if (ce != cudaSuccess) return celeris_rt::cuda_error(ce, "capture of the RCWA batch");
                const cudaError_t ie = cudaGraphInstantiate(&ctx.exec, graph, 0);
                cudaGraphDestroy(graph);
                if (ie != cudaSuccess) {
                    ctx.exec = nullptr;
                    return celeris_rt::cuda_error(ie, "instantiate the RCWA batch graph");
                }
                ctx.sig = sig;
                ctx.nkern = nk;
            }
            CEL_CUDA(cudaGraphLaunch(ctx.exec, st));
            count_launch(ctx.nkern);
            CEL_CUDA(cudaStreamSynchronize(st));
        }
        CEL_CUDA(cudaGetLastError());
        for (size_t w = 0; w < wave.size(); ++w) {
            const BucketPlan& p = plans[wave[w]];
            for (int i = 0; i < (int)p.ids.size(); ++i) {
                const int idx = cells[p.ids[i]].index;
                for (int e = 0; e < nexc; ++e) hres[(size_t)idx * nexc + e] = hres_pin[w][(size_t)i * nexc + e];
                hinfo[idx] = hinfo_pin[w][i];
            }
        }
    }
    // cells flagged as not mirror symmetric to rounding: solve again with the
    // full eigensolve
    std::vector<int> redo;
    for (size_t i = 0; i < hinfo.size(); ++i)
        if (hinfo[i] == kInfoAsym) redo.push_back((int)i);
    if (!redo.empty()) {
        std::vector<int> pos(cells.size(), -1);
        for (int i = 0; i < (int)cells.size(); ++i) pos[cells[i].index] = i;
        std::vector<HostCell> sub;
        for (size_t j = 0; j < redo.size(); ++j) {
            HostCell h = cells[pos[redo[j]]];
            h.sym = 0;
            h.index = (int)j;
            sub.push_back(h);
        }
        std::vector<celeris_rcwa_result> sub_out(sub.size() * nexc);
        std::vector<int> sub_info(sub.size(), 0);
        CEL_TRY(run_cells(sub, sub_out.data(), sub_info.data(), nexc));
        for (size_t j = 0; j < redo.size(); ++j) {
            for (int e = 0; e < nexc; ++e) hres[(size_t)redo[j] * nexc + e] = sub_out[j * nexc + e];
            hinfo[redo[j]] = sub_info[j];
        }
    }
    std::memcpy(out, hres.data(), sizeof(celeris_rcwa_result) * hres.size());
    int first_bad = -1;
    for (size_t i = 0; i < hinfo.size(); ++i) {
        if (info_out) info_out[i] = hinfo[i];
        if (hinfo[i] != 0 && first_bad < 0) first_bad = (int)i;
    }
    // with an info array the per-cell codes are the report (LAPACK style)
    if (first_bad >= 0 && !info_out) {
        const int v = hinfo[first_bad];
        return set_error(v > 0 ? CELERIS_ERR_EIG_NOCONV : CELERIS_ERR_SINGULAR,
                         "cell %d: %s (info %d)", first_bad,
                         v > 0 ? "QR eigensolve did not converge" : "singular pivot in an LU factorization", v);
    }
    return CELERIS_OK;
}

// ---- multi-layer stacks ----------------------------------------------------------------------
// Sub-allocation from one reserved region (the stack path's per-stream
// workspace arena): no cudaMalloc / cudaFree per call.
struct Bump {
    char* p = nullptr;
    size_t left = 0;
    template <typename T>
    int get(T** out, size_t count) {
        const size_t b = celeris_rt::align256(std::max<size_t>(count, 1) * sizeof(T));
        if (b > left) return set_error(CELERIS_ERR_OOM, "stack workspace: carve of %zu bytes over its plan", b);
        *out = reinterpret_cast<T*>(p);
        p += b;
        left -= b;
        return CELERIS_OK;
    }
};
size_t a256(size_t b) { return celeris_rt::align256(std::max<size_t>(b, 1)); }

// stacks[s] = (first layer index, layer count) into `layers`; exc holds 4 doubles
// (Ex0 re, im, Ey0 re, im) per stack; results nexc per stack.
// ord_out (may be NULL): per stack and excitation N x (de_t, de_r).
int run_stacks(const celeris_rcwa_cell* layers, const std::vector<std::pair<int, int>>& stacks,
               const double* exc, celeris_rcwa_result* out, int* info_out, int nexc, double* ord_out = nullptr) {
    CEL_TRY(celeris_rt::require_device());
    int dev = 0, smem_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // one stream (and so one workspace arena) per calling thread for the stack path
    static thread_local celeris_rt::ThreadStream t_stack_st;
    cudaStream_t st = nullptr;
    CEL_TRY(t_stack_st.get(&st));
    Workspace& ws = Workspace::for_stream(st);
    // stacks grouped by (Mx, My): one layer store and one recursion launch per group
    std::map<std::pair<int, int>, std::vector<int>> groups;
    for (int s = 0; s < (int)stacks.size(); ++s) {
        const celeris_rcwa_cell& f = layers[stacks[s].first];
        groups[{f.Mx, f.My}].push_back(s);
    }
    size_t free_b = 0, total_b = 0;
    CEL_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = free_b / 2;
    for (auto& g : groups) {
        const int Mx = g.first.first, My = g.first.second;
        const int N = (2 * Mx + 1) * (2 * My + 1), n = 2 * N;
        const size_t s_nn = (size_t)n * n, s_n = (size_t)n, s_NN = (size_t)N * N;
        // stacks in chunks whose layer store, eigen buffers and recursion buffers fit the budget
        const size_t per_layer = (7 * s_nn + 3 * s_NN + 4 * s_n) * sizeof(cplx) + 4096;
        const size_t per_stack = (7 * s_nn + 11 * s_n) * sizeof(cplx) + 4096;
        size_t c0 = 0;
        while (c0 < g.second.size()) {
            std::vector<int> ids;
            size_t bytes = 0;
            while (c0 < g.second.size()) {
                const size_t need = per_stack + per_layer * stacks[g.second[c0]].second;
                if (!ids.empty() && bytes + need > budget) break;
                ids.push_back(g.second[c0++]);
                bytes += need;
            }
            const int ns = (int)ids.size();
            // layer store slots, in stack order
            std::vector<HostCell> sub;
            std::vector<int> first_slot(ns);
            for (int k = 0; k < ns; ++k) {
                first_slot[k] = (int)sub.size();
                const auto& sp = stacks[ids[k]];
                for (int l = 0; l < sp.second; ++l)
                    sub.push_back(make_cell(layers[sp.first + l], (int)sub.size(), 1.0, 0.0, 0.0, 0.0, 2));
            }
            const int nslot = (int)sub.size();
            std::map<int, std::vector<int>> by_ng;
            for (int i = 0; i < nslot; ++i) by_ng[sub[i].ng].push_back(i);
            // region plan: layer store + recursion, then one raster class's bucket at a time
            const size_t c16 = sizeof(cplx);
            size_t fixed = 2 * a256(s_nn * nslot * c16) + a256(s_n * nslot * c16) + a256(nslot * sizeof(double)) +
                           7 * a256(s_nn * ns * c16) + a256(10 * s_n * ns * c16) + a256(s_n * ns * sizeof(int)) +
                           a256(ns * sizeof(int)) + a256(ns * sizeof(CellDev)) + a256(ns * sizeof(StackDev)) +
                           a256(ns * nexc * sizeof(celeris_rcwa_result));
            if (ord_out) fixed += a256((size_t)ns * nexc * N * 2 * sizeof(double));
            size_t class_max = 0;
            for (auto& kv : by_ng) {
                const size_t nc = kv.second.size(), ng = (size_t)std::max(kv.first, 0);
                size_t b = a256(nc * sizeof(CellDev)) + 5 * a256(s_nn * nc * c16) + 3 * a256(s_NN * nc * c16) +
                           a256(s_n * nc * c16) + a256(s_n * nc * sizeof(int)) + 2 * a256(nc * sizeof(int));
                if (ng > 0) b += a256((4 * Mx + 1) * ng * c16) + a256((4 * My + 1) * ng * c16);
                class_max = std::max(class_max, b);
            }
            CEL_TRY(ws.reserve(st, fixed + class_max));
            char* region = static_cast<char*>(ws.take(fixed + class_max));
            Bump mem{region, fixed};
            cplx *LW, *LA, *Lq;
            double* Lh;
            CEL_TRY(mem.get(&LW, s_nn * nslot));
            CEL_TRY(mem.get(&LA, s_nn * nslot));
            CEL_TRY(mem.get(&Lq, s_n * nslot));
            CEL_TRY(mem.get(&Lh, (size_t)nslot));
            std::vector<int> sub_info(nslot, 0);
            // eigen-solutions of every layer, one bucket per raster class
            for (auto& kv : by_ng) {
                const int ng = kv.first;
                const std::vector<int>& si = kv.second;
                const int nc = (int)si.size();
                if (ng > 0 && laurent_smem(Mx, My, ng) + 1024 > (size_t)smem_optin)
                    return set_error(CELERIS_ERR_TOO_LARGE, "raster %d with M=(%d,%d) exceeds shared memory", ng,
                                     Mx, My);
                Bump bm{region + fixed, class_max};  // reused by each class in turn (the stream is synchronised)
                Bucket b;
                std::memset(&b, 0, sizeof(b));
                b.Mx = Mx;
                b.My = My;
                b.N = N;
                b.n = n;
                b.ng = ng;
                b.ncell = nc;
                b.s_nn = s_nn;
                b.s_ns = (size_t)n * (n + 2);
                b.s_NN = s_NN;
                b.s_n = s_n;
                CellDev* dcells;
                CEL_TRY(bm.get(&dcells, (size_t)nc));
                b.cells = dcells;
                cplx** mats[] = {&b.H, &b.Z, &b.X, &b.W, &b.A};
                for (cplx** m : mats) CEL_TRY(bm.get(m, s_nn * nc));
                CEL_TRY(bm.get(&b.Einv, s_NN * nc));
                CEL_TRY(bm.get(&b.Exx, s_NN * nc));
                CEL_TRY(bm.get(&b.Eyy, s_NN * nc));
                CEL_TRY(bm.get(&b.q1, s_n * nc));
                CEL_TRY(bm.get(&b.piv, s_n * nc));
                CEL_TRY(bm.get(&b.info, (size_t)nc));
                if (ng > 0) {
                    cplx *phx, *phy;
                    CEL_TRY(bm.get(&phx, (size_t)(4 * Mx + 1) * ng));
                    CEL_TRY(bm.get(&phy, (size_t)(4 * My + 1) * ng));
                    b.phx = phx;
                    b.phy = phy;
                }
                std::vector<CellDev> hd(nc);
                std::vector<int> hslot(nc);
                for (int i = 0; i < nc; ++i) {
                    hd[i] = sub[si[i]].d;
                    hslot[i] = si[i];
                }
                int* dslot;
                CEL_TRY(bm.get(&dslot, (size_t)nc));
                CEL_CUDA(cudaMemcpyAsync(dcells, hd.data(), sizeof(CellDev) * nc, cudaMemcpyHostToDevice, st));
                CEL_CUDA(cudaMemcpyAsync(dslot, hslot.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
                SmemNeeds needs;
                needs.add(Mx, My, ng, n);
                CEL_TRY(set_smem_limits(needs));
                launch_bucket(b, uniform_cfg(256), st, nullptr, true);
                rcwa_layer_out<<<nc, kRT, 0, st>>>(b, LW, LA, Lq, Lh, dslot);
                count_launch(1);
                CEL_CUDA(cudaGetLastError());
                std::vector<int> hinfo(nc);
                CEL_CUDA(cudaMemcpyAsync(hinfo.data(), b.info, sizeof(int) * nc, cudaMemcpyDeviceToHost, st));
                CEL_CUDA(cudaStreamSynchronize(st));
                for (int i = 0; i < nc; ++i) sub_info[si[i]] = hinfo[i];
            }
            // S-matrix recursion and outputs, one CTA per stack
            StackBucket sb;
            std::memset(&sb, 0, sizeof(sb));
            sb.Mx = Mx;
            sb.My = My;
            sb.N = N;
            sb.n = n;
            sb.nstack = ns;
            sb.LW = LW;
            sb.LA = LA;
            sb.Lq = Lq;
            sb.Lh = Lh;
            sb.s_nn = s_nn;
            sb.s_n = s_n;
            cplx** smats[] = {&sb.S12, &sb.S22, &sb.Q, &sb.P, &sb.X, &sb.Y, &sb.Z1};
            for (cplx** m : smats) CEL_TRY(mem.get(m, s_nn * ns));
            CEL_TRY(mem.get(&sb.vec, 10 * s_n * ns));
            CEL_TRY(mem.get(&sb.piv, s_n * ns));
            CEL_TRY(mem.get(&sb.info, (size_t)ns));
            CellDev* scells;
            StackDev* sdev;
            celeris_rcwa_result* dres;
            CEL_TRY(mem.get(&scells, (size_t)ns));
            CEL_TRY(mem.get(&sdev, (size_t)ns));
            CEL_TRY(mem.get(&dres, (size_t)ns * nexc));
            std::vector<CellDev> hc(ns);
            std::vector<StackDev> hs(ns);
            std::vector<int> hinfo(ns, 0);
            for (int k = 0; k < ns; ++k) {
                const auto& sp = stacks[ids[k]];
                const double* e = exc + 4 * (size_t)ids[k];
                hc[k] = make_cell(layers[sp.first], ids[k], e[0], e[1], e[2], e[3], nexc).d;
                hs[k].nl = sp.second;
                hs[k].slot0 = first_slot[k];
                for (int l = 0; l < sp.second; ++l)
                    if (sub_info[first_slot[k] + l] != 0 && hinfo[k] == 0) hinfo[k] = sub_info[first_slot[k] + l];
            }
            CEL_CUDA(cudaMemcpyAsync(scells, hc.data(), sizeof(CellDev) * ns, cudaMemcpyHostToDevice, st));
            CEL_CUDA(cudaMemcpyAsync(sdev, hs.data(), sizeof(StackDev) * ns, cudaMemcpyHostToDevice, st));
            CEL_CUDA(cudaMemcpyAsync(sb.info, hinfo.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
            sb.cells = scells;
            sb.stacks = sdev;
            const size_t sm_stage = lu_stage_bytes(n);
            CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_stack_smat), sm_stage));
            rcwa_stack_smat<<<ns, kRT, sm_stage, st>>>(sb);
            Bucket eb;
            std::memset(&eb, 0, sizeof(eb));
            eb.Mx = Mx;
            eb.My = My;
            eb.N = N;
            eb.n = n;
            eb.ncell = ns;
            eb.cells = scells;
            eb.vec = sb.vec;
            eb.info = sb.info;
            eb.res = dres;
            eb.s_n = s_n;
            eb.s_nn = s_nn;
            if (ord_out) CEL_TRY(mem.get(&eb.ord, (size_t)ns * nexc * N * 2));
            rcwa_epilogue<<<ns, kRT, 0, st>>>(eb);
            count_launch(2);
            CEL_CUDA(cudaGetLastError());
            std::vector<celeris_rcwa_result> hres((size_t)ns * nexc);
            CEL_CUDA(cudaMemcpyAsync(hres.data(), dres, sizeof(celeris_rcwa_result) * ns * nexc,
                                     cudaMemcpyDeviceToHost, st));
            CEL_CUDA(cudaMemcpyAsync(hinfo.data(), sb.info, sizeof(int) * ns, cudaMemcpyDeviceToHost, st));
            std::vector<double> hord;
            if (ord_out) {
                hord.resize((size_t)ns * nexc * N * 2);
                CEL_CUDA(cudaMemcpyAsync(hord.data(), eb.ord, sizeof(double) * hord.size(), cudaMemcpyDeviceToHost,
                                         st));
            }
            CEL_CUDA(cudaStreamSynchronize(st));
            if (ord_out)
                for (int k = 0; k < ns; ++k)
                    std::memcpy(ord_out + (size_t)ids[k] * nexc * N * 2, hord.data() + (size_t)k * nexc * N * 2,
                                sizeof(double) * nexc * N * 2);
            for (int k = 0; k < ns; ++k) {
                for (int e = 0; e < nexc; ++e) out[(size_t)ids[k] * nexc + e] = hres[(size_t)k * nexc + e];
                if (info_out) info_out[ids[k]] = hinfo[k];
            }
            if (!info_out)
                for (int k = 0; k < ns; ++k) {
                    if (hinfo[k] > 0)
                        return set_error(CELERIS_ERR_EIG_NOCONV, "eigensolve did not converge (a layer of stack %d)",
                                         ids[k]);
                    if (hinfo[k] < 0)
                        return set_error(CELERIS_ERR_SINGULAR, "singular interface system (stack %d)", ids[k]);
                }
        }
    }
    return CELERIS_OK;
}

// Layers of one stack must share everything but the pattern, materials and thickness.
int validate_stack(const celeris_rcwa_cell* l, int nl) {
    if (nl < 1) return set_error(CELERIS_ERR_INVALID_ARG, "a stack needs at least one layer");
    for (int i = 0; i < nl; ++i) CEL_TRY(validate(l[i]));
    const celeris_rcwa_cell& f = l[0];
    for (int i = 1; i < nl; ++i) {
        const celeris_rcwa_cell& c = l[i];
        if (c.Mx != f.Mx || c.My != f.My || c.period_x_um != f.period_x_um || c.period_y_um != f.period_y_um ||
            c.wavelength_um != f.wavelength_um || c.theta_rad != f.theta_rad || c.phi_rad != f.phi_rad ||
            c.n_inc[0] != f.n_inc[0] || c.n_inc[1] != f.n_inc[1] || c.n_sub[0] != f.n_sub[0] ||
            c.n_sub[1] != f.n_sub[1])
            return set_error(CELERIS_ERR_INVALID_ARG,
                             "layer %d of a stack differs from layer 0 in orders, periods, wavelength, angles or "
                             "half-spaces",
                             i);
    }
    return CELERIS_OK;
}

// ---- standalone eigensolve: batches of n x n matrices through the eigen-stages ------------
int run_eig(const double* A, int n, int count, double* evals, double* evecs, int* info_out) {
    CEL_TRY(celeris_rt::require_device());
    const size_t s_nn = (size_t)n * n, s_n = (size_t)n;
    int dev = 0;
    CEL_CUDA(cudaGetDevice(&dev));
    static thread_local celeris_rt::ThreadStream t_eig_st;  // one stream and arena per calling thread
    cudaStream_t st = nullptr;
    CEL_TRY(t_eig_st.get(&st));
    Workspace& ws = Workspace::for_stream(st);
    if (n <= kSmemEigMaxN)
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_hess<true>), (s_nn + 2 * s_n) * sizeof(cplx)));
    else
        CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_hess<false>), hess_stage_bytes(n)));
    CEL_TRY(raise_dyn_smem(reinterpret_cast<const void*>(rcwa_schur), kSchurSmemOneCta));
    size_t free_b = 0, total_b = 0;
    CEL_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t per = (7 * s_nn + 2 * s_n) * sizeof(cplx) + 4096;
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)count, (free_b / 2) / per));
    for (int c0 = 0; c0 < count; c0 += chunk) {
        const int nc = std::min(chunk, count - c0);
        const size_t c16 = sizeof(cplx);
        const size_t plan = 6 * a256(s_nn * nc * c16) + 2 * a256(s_n * nc * c16) + a256(nc * sizeof(int));
        CEL_TRY(ws.reserve(st, plan));
        Bump mem{static_cast<char*>(ws.take(plan)), plan};
        Bucket b;
        std::memset(&b, 0, sizeof(b));
        b.n = n;
        b.N = n / 2;
        b.ncell = nc;
        b.s_nn = s_nn;
        b.s_n = s_n;
        cplx *dA, *dval, *dvec;
        CEL_TRY(mem.get(&dA, s_nn * nc));
        cplx** mats[] = {&b.H, &b.Z, &b.X, &b.W, &b.A};
        for (cplx** m : mats) CEL_TRY(mem.get(m, s_nn * nc));
        CEL_TRY(mem.get(&b.q1, s_n * nc));
        CEL_TRY(mem.get(&b.info, (size_t)nc));
        CEL_TRY(mem.get(&dval, s_n * nc));
        dvec = b.A;  // free after the eigenvectors
        CEL_CUDA(cudaMemcpyAsync(dA, A + 2 * s_nn * c0, sizeof(cplx) * s_nn * nc, cudaMemcpyHostToDevice, st));
        CEL_CUDA(cudaMemsetAsync(b.info, 0, sizeof(int) * nc, st));
        eig_load<<<nc, kRT, 0, st>>>(dA, b);
        if (n <= kSmemEigMaxN)
            rcwa_hess<true><<<nc, kRT, (s_nn + 2 * s_n) * sizeof(cplx), st>>>(b);
        else
            rcwa_hess<false><<<nc, kRT, hess_stage_bytes(n), st>>>(b);
        rcwa_schur<<<nc, kSchurThreads, schur_smem(nc), st>>>(b);
        rcwa_vec<<<nc, kRT, 0, st>>>(b);
        eig_store<<<nc, kRT, 0, st>>>(b, dval, dvec);
        count_launch(6);
        CEL_CUDA(cudaGetLastError());
        std::vector<int> hinfo(nc);
        CEL_CUDA(cudaMemcpyAsync(evals + 2 * s_n * c0, dval, sizeof(cplx) * s_n * nc, cudaMemcpyDeviceToHost, st));
        CEL_CUDA(cudaMemcpyAsync(evecs + 2 * s_nn * c0, dvec, sizeof(cplx) * s_nn * nc, cudaMemcpyDeviceToHost, st));
        CEL_CUDA(cudaMemcpyAsync(hinfo.data(), b.info, sizeof(int) * nc, cudaMemcpyDeviceToHost, st));
        CEL_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < nc; ++i) {
            if (info_out) info_out[c0 + i] = hinfo[i];
            else if (hinfo[i] != 0)
                return set_error(CELERIS_ERR_EIG_NOCONV, "QR did not converge (info %d)", hinfo[i]);
        }
    }
    return CELERIS_OK;
}

}  // namespace

extern "C" {

int celeris_solve_rcwa_2d(const celeris_rcwa_cell* cell, const double* Ex0, const double* Ey0,
                          celeris_rcwa_result* out) {
    if (!cell || !Ex0 || !Ey0 || !out) return set_error(CELERIS_ERR_INVALID_ARG, "NULL argument");
    CEL_TRY(validate(*cell));
    std::vector<HostCell> cells{make_cell(*cell, 0, Ex0[0], Ex0[1], Ey0[0], Ey0[1], 1)};
    return run_cells(cells, out, nullptr, 1);
}

int celeris_rcwa_tuning_report(char* buf, int len) {
    if (!buf || len <= 0) return set_error(CELERIS_ERR_INVALID_ARG, "bad buffer");
    std::string s;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto& kv : tune_table()) {
        s += "Mx=" + std::to_string(std::get<0>(kv.first)) + " My=" + std::to_string(std::get<1>(kv.first)) +
             " grid=" + std::to_string(std::get<2>(kv.first) / 4) +
             ((std::get<2>(kv.first) & 2) ? " parity-classes" : "") +
             ((std::get<2>(kv.first) & 1) ? " batch>=SMs:" : " batch<SMs:");
        for (int st = 0; st < ST_COUNT; ++st)
            s += std::string(" ") + kStageNames[st] + "=" + std::to_string(kv.second.threads[st]);
        s += "\n";
    }
    std::snprintf(buf, (size_t)len, "%s", s.c_str());
    return CELERIS_OK;
}

int celeris_solve_rcwa_2d_stack(const celeris_rcwa_cell* layers, int nlayers, const double* Ex0, const double* Ey0,
                                celeris_rcwa_result* out) {
    if (!layers || !Ex0 || !Ey0 || !out) return set_error(CELERIS_ERR_INVALID_ARG, "NULL argument");
    CEL_TRY(validate_stack(layers, nlayers));
    const double exc[4] = {Ex0[0], Ex0[1], Ey0[0], Ey0[1]};
    return run_stacks(layers, {{0, nlayers}}, exc, out, nullptr, 1);
}

int celeris_eig_general_batch(const double* A, int n, int count, double* evals, double* evecs, int* info) {
    if (n < 1 || count < 0) return set_error(CELERIS_ERR_INVALID_ARG, "n must be >= 1 and count >= 0");
    if (n > kMaxN) return set_error(CELERIS_ERR_TOO_LARGE, "n = %d > %d", n, kMaxN);
    if (count == 0) return CELERIS_OK;
    if (!A || !evals || !evecs) return set_error(CELERIS_ERR_INVALID_ARG, "NULL argument");
    {   // x * 0 is NaN exactly when x is NaN or Inf: one branch-free pass
        const size_t per = 2 * (size_t)n * n;
        for (int c = 0; c < count; ++c) {
            double z = 0.0;
            for (size_t i = 0; i < per; ++i) z += A[c * per + i] * 0.0;
            if (z != 0.0) return set_error(CELERIS_ERR_INVALID_ARG, "matrix %d holds NaN or Inf", c);
        }
    }
    if (n == 1) {  // nothing to reduce
        for (int c = 0; c < count; ++c) {
            evals[2 * c] = A[2 * c];
            evals[2 * c + 1] = A[2 * c + 1];
            evecs[2 * c] = 1.0;
            evecs[2 * c + 1] = 0.0;
            if (info) info[c] = 0;
        }
        return CELERIS_OK;
    }
    return run_eig(A, n, count, evals, evecs, info);
}

int celeris_eig_general(const double* A, int n, double* evals, double* evecs) {
    return celeris_eig_general_batch(A, n, 1, evals, evecs, nullptr);
}

int celeris_solve_rcwa_2d_orders(const celeris_rcwa_cell* layers, int nlayers, const double* Ex0, const double* Ey0,
                                 celeris_rcwa_result* out, celeris_rcwa_order* orders, int max_orders) {
    if (!layers || !Ex0 || !Ey0 || !out || !orders) return set_error(CELERIS_ERR_INVALID_ARG, "NULL argument");
    CEL_TRY(validate_stack(layers, nlayers));
    const celeris_rcwa_cell& f = layers[0];
    const int N = (2 * f.Mx + 1) * (2 * f.My + 1);
    if (max_orders < N) return set_error(CELERIS_ERR_INVALID_ARG, "orders holds %d records, %d needed", max_orders, N);
    const double exc[4] = {Ex0[0], Ex0[1], Ey0[0], Ey0[1]};
    std::vector<double> ord((size_t)N * 2);
    CEL_TRY(run_stacks(layers, {{0, nlayers}}, exc, out, nullptr, 1, ord.data()));
    // order labels and the propagation test of rcwa2d.cpp:469-484 (same arithmetic)
    typedef std::complex<double> cd;
    const double k0 = 2.0 * PI / f.wavelength_um;
    const cd n_inc(f.n_inc[0], f.n_inc[1]);
    const cd kx0 = n_inc * std::sin(f.theta_rad) * std::cos(f.phi_rad) * k0;
    const cd ky0 = n_inc * std::sin(f.theta_rad) * std::sin(f.phi_rad) * k0;
    const double k0sub = (f.n_sub[0] * k0) * (f.n_sub[0] * k0);
    const double k0inc = (f.n_inc[0] * k0) * (f.n_inc[0] * k0);
    for (int p = -f.Mx; p <= f.Mx; ++p)
        for (int q = -f.My; q <= f.My; ++q) {
            const int i = (p + f.Mx) * (2 * f.My + 1) + (q + f.My);
            const cd kx = kx0 - 2.0 * PI * (double)p / f.period_x_um;
            const cd ky = ky0 - 2.0 * PI * (double)q / f.period_y_um;
            const double kt2 = (kx * kx + ky * ky).real();
            celeris_rcwa_order& o = orders[i];
            o.p = p;
            o.q = q;
            o.de_t = ord[2 * (size_t)i];
            o.de_r = ord[2 * (size_t)i + 1];
            o.prop_t = k0sub - kt2 > 0.0;
            o.prop_r = k0inc - kt2 > 0.0;
        }
    return CELERIS_OK;
}

int celeris_rcwa_stack_batch(const celeris_rcwa_cell* layers, const int* layer_start, int nstack,
                             celeris_rcwa_result* out, int* info) {
    if (nstack < 0) return set_error(CELERIS_ERR_INVALID_ARG, "nstack < 0");
    if (nstack == 0) return CELERIS_OK;
    if (!layers || !layer_start || !out) return set_error(CELERIS_ERR_INVALID_ARG, "NULL argument");
    std::vector<std::pair<int, int>> stacks;
    std::vector<double> exc(4 * (size_t)nstack, 0.0);
    for (int s = 0; s < nstack; ++s) {
        const int a = layer_start[s], nl = layer_start[s + 1] - layer_start[s];
        if (a < 0 || nl < 1) return set_error(CELERIS_ERR_INVALID_ARG, "stack %d: bad layer range", s);
        CEL_TRY(validate_stack(layers + a, nl));
        stacks.push_back({a, nl});
        exc[4 * (size_t)s] = 1.0;  // slot 0 = X polarization (Ex0 = 1), slot 1 = Y
    }
    return run_stacks(layers, stacks, exc.data(), out, info, 2);
}

int celeris_rcwa_batch(const celeris_rcwa_cell* cells, int ncell, celeris_rcwa_result* out, int* info) {
    if (ncell < 0) return set_error(CELERIS_ERR_INVALID_ARG, "ncell < 0");
    if (ncell == 0) return CELERIS_OK;
    if (!cells || !out) return set_error(CELERIS_ERR_INVALID_ARG, "NULL argument");
    std::vector<HostCell> hc;
    hc.reserve(ncell);
    for (int i = 0; i < ncell; ++i) {
        const int v = validate(cells[i]);
        if (v != CELERIS_OK) {
            const std::string msg = celeris_last_error();
            return set_error(v, "cell %d: %s", i, msg.c_str());
        }
        hc.push_back(make_cell(cells[i], i, 1.0, 0.0, 0.0, 0.0, 2));
    }
    return run_cells(hc, out, info, 2);
}

int celeris_debug_qr_iteration_cap(int cap) {
    if (cap < 0) return set_error(CELERIS_ERR_INVALID_ARG, "cap < 0");
    CEL_TRY(celeris_rt::require_device());
    CEL_CUDA(cudaMemcpyToSymbol(g_qr_iter_cap, &cap, sizeof(int)));
    return CELERIS_OK;
}

}  // extern "C"
