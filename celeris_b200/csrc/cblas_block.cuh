// Block-level complex FP64 dense linear algebra for the batched RCWA solve.
//
// Every routine here is executed cooperatively by ALL threads of one CTA on
// one unit cell's matrices (one CTA per cell; the batch is the grid). Matrices
// are row-major complex (double2) with an explicit leading dimension and may
// live in global memory (L2-resident working set) or in shared memory: the
// routines take generic pointers. Each routine begins and ends at a block-wide
// barrier, so consecutive calls compose without extra synchronization.
//
// Routines (all O(n^3) work is spread over the block; loops are bounded):
//   blk_gemm        C = alpha A B + beta C (smem-staged 32x32 tiles)
//   blk_lu          partial-pivot LU in place (LAPACK zgetrf semantics: pivot =
//                   first max |re|+|im| in the column)
//   blk_lu_solve    X = A^{-1} B from the LU factors, any number of RHS
//   blk_hessenberg  Householder reduction to upper Hessenberg, Z accumulated
//   blk_schur       complex single-shift QR (Wilkinson shift, deflation on
//                   negligible subdiagonals, exceptional shifts) to upper
//                   triangular T, Z updated; sweep cap -> info > 0
//   blk_trevc       right eigenvectors of triangular T by back substitution
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace cb {

typedef double2 cplx;

__device__ __forceinline__ cplx C(double r, double i) { return make_double2(r, i); }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return C(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return C(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cplx cneg(cplx a) { return C(-a.x, -a.y); }
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return C(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__device__ __forceinline__ cplx cmulc(cplx a, cplx b) {
    return C(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// c + a * b
__device__ __forceinline__ cplx cfma(cplx a, cplx b, cplx c) {
    return C(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// c - a * b
__device__ __forceinline__ cplx cfms(cplx a, cplx b, cplx c) {
    return C(fma(-a.x, b.x, fma(a.y, b.y, c.x)), fma(-a.x, b.y, fma(-a.y, b.x, c.y)));
}
__device__ __forceinline__ cplx cconj(cplx a) { return C(a.x, -a.y); }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return C(a.x * s, a.y * s); }
__device__ __forceinline__ double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ double cabs(cplx a) { return hypot(a.x, a.y); }
__device__ __forceinline__ double cnorm2(cplx a) { return a.x * a.x + a.y * a.y; }
// a / b (Smith's algorithm)
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + b.y * r;
        return C((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    const double r = b.x / b.y, d = b.x * r + b.y;
    return C((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ cplx cinv(cplx b) { return cdiv(C(1.0, 0.0), b); }
// principal square root (branch cut on the negative real axis, sign of the
// imaginary part carried through, as C99 csqrt / std::sqrt)
__device__ __forceinline__ cplx csqrt_p(cplx z) {
    const double x = z.x, y = z.y;
    if (x == 0.0 && y == 0.0) return C(0.0, y);
    const double m = hypot(x, y);
    if (x >= 0.0) {
        const double t = sqrt(0.5 * (m + x));
        return C(t, y / (2.0 * t));
    }
    const double t = sqrt(0.5 * (m - x));
    return C(fabs(y) / (2.0 * t), copysign(t, y));
}
// exp(i w)
__device__ __forceinline__ cplx cexpi(cplx w) {
    double s, c;
    sincos(w.x, &s, &c);
    const double e = exp(-w.y);
    return C(e * c, e * s);
}

// ---- block reductions ------------------------------------------------------------
// Shared scratch for reductions: at least 32 doubles + 32 ints.
struct RedScratch {
    double d[64];
    int i[32];
};

__device__ __forceinline__ double blk_sum(double v, RedScratch* rs) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (l == 0) rs->d[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int q = 0; q < nw; ++q) s += rs->d[q];  // same order in every thread
    return s;
}

// Complex sum: returns the same value in every thread.
__device__ __forceinline__ cplx blk_csum(cplx v, RedScratch* rs) {
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (l == 0) {
        rs->d[2 * w] = v.x;
        rs->d[2 * w + 1] = v.y;
    }
    __syncthreads();
    cplx s = C(0.0, 0.0);
    for (int q = 0; q < nw; ++q) {
        s.x += rs->d[2 * q];
        s.y += rs->d[2 * q + 1];
    }
    return s;
}

// argmax of val over the block; ties -> smallest index. Same result everywhere.
__device__ __forceinline__ int blk_argmax(double val, int idx, RedScratch* rs) {
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, val, o);
        const int oi = __shfl_down_sync(0xffffffffu, idx, o);
        if (ov > val || (ov == val && oi < idx)) {
            val = ov;
            idx = oi;
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (l == 0) {
        rs->d[w] = val;
        rs->i[w] = idx;
    }
    __syncthreads();
    double bv = rs->d[0];
    int bi = rs->i[0];
    for (int q = 1; q < nw; ++q) {
        if (rs->d[q] > bv || (rs->d[q] == bv && rs->i[q] < bi)) {
            bv = rs->d[q];
            bi = rs->i[q];
        }
    }
    return bi;
}

// ---- GEMM -------------------------------------------------------------------------
constexpr int GT = 32;  // output tile
constexpr int GK = 16;  // k chunk
struct GemmSmem {
    cplx a[GT][GK + 1];
    cplx b[GK][GT + 1];
};

// C[m x n] = alpha * A[m x k] * B[k x n] + beta * C  (row-major). C may not alias A or B.
__device__ void blk_gemm(int m, int n, int k, cplx alpha, const cplx* A, int lda, const cplx* B, int ldb,
                         cplx beta, cplx* Cm, int ldc, GemmSmem* sm) {
    const int tid = threadIdx.x, nt = blockDim.x;
    // each thread owns outputs (r, c) of the tile with index tid + s*nt
    const int per = (GT * GT + nt - 1) / nt;
    __syncthreads();
    for (int i0 = 0; i0 < m; i0 += GT) {
        for (int j0 = 0; j0 < n; j0 += GT) {
            cplx acc[8];
#pragma unroll
            for (int s = 0; s < 8; ++s) acc[s] = C(0.0, 0.0);
            for (int k0 = 0; k0 < k; k0 += GK) {
                for (int e = tid; e < GT * GK; e += nt) {
                    const int r = e / GK, c = e % GK;
                    sm->a[r][c] = (i0 + r < m && k0 + c < k) ? A[(size_t)(i0 + r) * lda + k0 + c] : C(0.0, 0.0);
                }
                for (int e = tid; e < GK * GT; e += nt) {
                    const int r = e / GT, c = e % GT;
                    sm->b[r][c] = (k0 + r < k && j0 + c < n) ? B[(size_t)(k0 + r) * ldb + j0 + c] : C(0.0, 0.0);
                }
                __syncthreads();
#pragma unroll
                for (int s = 0; s < 8; ++s) {
                    if (s >= per) break;
                    const int e = tid + s * nt;
                    if (e >= GT * GT) break;
                    const int r = e / GT, c = e % GT;
                    cplx a = acc[s];
#pragma unroll 4
                    for (int kk = 0; kk < GK; ++kk) a = cfma(sm->a[r][kk], sm->b[kk][c], a);
                    acc[s] = a;
                }
                __syncthreads();
            }
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                if (s >= per) break;
                const int e = tid + s * nt;
                if (e >= GT * GT) break;
                const int r = e / GT, c = e % GT;
                if (i0 + r < m && j0 + c < n) {
                    cplx* dst = &Cm[(size_t)(i0 + r) * ldc + j0 + c];
                    cplx v = cmul(alpha, acc[s]);
                    if (beta.x != 0.0 || beta.y != 0.0) v = cfma(beta, *dst, v);
                    *dst = v;
                }
            }
        }
    }
    __syncthreads();
}

// ---- LU ------------------------------------------------------------------------------
// In-place LU with partial pivoting of the n x n matrix A. piv[k] = row swapped
// with k at step k. Returns 0, or k+1 for the first exactly-zero pivot (the
// factorization continues, like zgetrf).
__device__ int blk_lu(int n, cplx* A, int lda, int* piv, RedScratch* rs) {
    const int tid = threadIdx.x, nt = blockDim.x;
    int info = 0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        double best = -1.0;
        int bi = k;
        for (int i = k + tid; i < n; i += nt) {
            const double v = cabs1(A[(size_t)i * lda + k]);
            if (v > best) {
                best = v;
                bi = i;
            }
        }
        const int p = blk_argmax(best, bi, rs);
        if (tid == 0) piv[k] = p;
        if (p != k) {
            for (int j = tid; j < n; j += nt) {
                const cplx t = A[(size_t)k * lda + j];
                A[(size_t)k * lda + j] = A[(size_t)p * lda + j];
                A[(size_t)p * lda + j] = t;
            }
        }
        __syncthreads();
        const cplx akk = A[(size_t)k * lda + k];
        if (akk.x == 0.0 && akk.y == 0.0) {
            if (info == 0) info = k + 1;
            __syncthreads();
            continue;
        }
        const cplx inv = cinv(akk);
        for (int i = k + 1 + tid; i < n; i += nt) A[(size_t)i * lda + k] = cmul(A[(size_t)i * lda + k], inv);
        __syncthreads();
        const int w = n - k - 1;
        for (int e = tid; e < w * w; e += nt) {
            const int i = k + 1 + e / w, j = k + 1 + e % w;
            A[(size_t)i * lda + j] = cfms(A[(size_t)i * lda + k], A[(size_t)k * lda + j], A[(size_t)i * lda + j]);
        }
        __syncthreads();
    }
    return info;
}

// B (n x nrhs, row-major, ldb) <- A^{-1} B using the factors of blk_lu.
__device__ void blk_lu_solve(int n, const cplx* LU, int lda, const int* piv, int nrhs, cplx* B, int ldb) {
    const int tid = threadIdx.x, nt = blockDim.x;
    __syncthreads();
    // row interchanges in factorization order
    for (int k = 0; k < n; ++k) {
        const int p = piv[k];
        if (p != k)
            for (int r = tid; r < nrhs; r += nt) {
                const cplx t = B[(size_t)k * ldb + r];
                B[(size_t)k * ldb + r] = B[(size_t)p * ldb + r];
                B[(size_t)p * ldb + r] = t;
            }
        __syncthreads();
    }
    // forward: unit lower L
    for (int j = 0; j < n - 1; ++j) {
        const int w = n - j - 1;
        for (int e = tid; e < w * nrhs; e += nt) {
            const int i = j + 1 + e / nrhs, r = e % nrhs;
            B[(size_t)i * ldb + r] = cfms(LU[(size_t)i * lda + j], B[(size_t)j * ldb + r], B[(size_t)i * ldb + r]);
        }
        __syncthreads();
    }
    // backward: U
    for (int j = n - 1; j >= 0; --j) {
        const cplx inv = cinv(LU[(size_t)j * lda + j]);
        for (int r = tid; r < nrhs; r += nt) B[(size_t)j * ldb + r] = cmul(B[(size_t)j * ldb + r], inv);
        __syncthreads();
        for (int e = tid; e < j * nrhs; e += nt) {
            const int i = e / nrhs, r = e % nrhs;
            B[(size_t)i * ldb + r] = cfms(LU[(size_t)i * lda + j], B[(size_t)j * ldb + r], B[(size_t)i * ldb + r]);
        }
        __syncthreads();
    }
}

// ---- Hessenberg reduction ------------------------------------------------------------
// H (n x n) <- Q^H H Q upper Hessenberg; Z <- Q (Z is initialised here).
// v, w: scratch vectors of length n (shared or global).
__device__ void blk_hessenberg(int n, cplx* H, int ldh, cplx* Z, int ldz, cplx* v, cplx* w, RedScratch* rs) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nwarp = nt >> 5;
    for (int e = tid; e < n * n; e += nt) {
        const int i = e / n, j = e % n;
        Z[(size_t)i * ldz + j] = C(i == j ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;  // length of x = H[k+1:, k]
        double s = 0.0;
        for (int i = tid; i < m; i += nt) s += cnorm2(H[(size_t)(k + 1 + i) * ldh + k]);
        const double xnorm2 = blk_sum(s, rs);
        const cplx x0 = H[(size_t)(k + 1) * ldh + k];
        const double tail = xnorm2 - cnorm2(x0);
        if (tail <= 0.0) {  // already zero below the subdiagonal
            __syncthreads();
            continue;
        }
        const double xn = sqrt(xnorm2);
        const double ax0 = cabs(x0);
        const cplx ph = ax0 > 0.0 ? cscale(x0, 1.0 / ax0) : C(1.0, 0.0);
        const cplx alpha = cscale(ph, -xn);          // -e^{i arg x0} ||x||
        const cplx v0 = csub(x0, alpha);
        const double vnorm2 = tail + cnorm2(v0);
        const double beta = 2.0 / vnorm2;            // H <- (I - beta v v^H) H (...)
        for (int i = tid; i < m; i += nt) v[i] = (i == 0) ? v0 : H[(size_t)(k + 1 + i) * ldh + k];
        __syncthreads();
        // left: rows k+1.., columns k+1..n-1 (column k becomes alpha e1)
        for (int j = k + 1 + tid; j < n; j += nt) {
            cplx acc = C(0.0, 0.0);
            for (int i = 0; i < m; ++i) acc = cfma(cconj(v[i]), H[(size_t)(k + 1 + i) * ldh + j], acc);
            w[j] = cscale(acc, beta);
        }
        __syncthreads();
        for (int e = tid; e < m * (n - k - 1); e += nt) {
            const int i = e / (n - k - 1), j = k + 1 + e % (n - k - 1);
            H[(size_t)(k + 1 + i) * ldh + j] = cfms(v[i], w[j], H[(size_t)(k + 1 + i) * ldh + j]);
        }
        for (int i = tid; i < m; i += nt) H[(size_t)(k + 1 + i) * ldh + k] = (i == 0) ? alpha : C(0.0, 0.0);
        __syncthreads();
        // right: all rows, columns k+1..n-1: H <- H (I - beta v v^H)
        for (int i = warp; i < n; i += nwarp) {
            cplx acc = C(0.0, 0.0);
            for (int j = lane; j < m; j += 32) acc = cfma(H[(size_t)i * ldh + k + 1 + j], v[j], acc);
            for (int o = 16; o > 0; o >>= 1) {
                acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
                acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
            }
            if (lane == 0) w[i] = cscale(acc, beta);
        }
        __syncthreads();
        for (int e = tid; e < n * m; e += nt) {
            const int i = e / m, j = e % m;
            H[(size_t)i * ldh + k + 1 + j] = cfms(w[i], cconj(v[j]), H[(size_t)i * ldh + k + 1 + j]);
        }
        __syncthreads();
        // Z <- Z (I - beta v v^H)
        for (int i = warp; i < n; i += nwarp) {
            cplx acc = C(0.0, 0.0);
            for (int j = lane; j < m; j += 32) acc = cfma(Z[(size_t)i * ldz + k + 1 + j], v[j], acc);
            for (int o = 16; o > 0; o >>= 1) {
                acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
                acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
            }
            if (lane == 0) w[i] = cscale(acc, beta);
        }
        __syncthreads();
        for (int e = tid; e < n * m; e += nt) {
            const int i = e / m, j = e % m;
            Z[(size_t)i * ldz + k + 1 + j] = cfms(w[i], cconj(v[j]), Z[(size_t)i * ldz + k + 1 + j]);
        }
        __syncthreads();
    }
}

// ---- complex Schur by shifted QR ------------------------------------------------------
// Givens G = [[c, s], [-conj(s), c]] with G [a; b] = [r; 0], c real.
__device__ __forceinline__ void givens(cplx a, cplx b, double& c, cplx& s) {
    const double aa = cabs(a), ab = cabs(b);
    if (ab == 0.0) {
        c = 1.0;
        s = C(0.0, 0.0);
        return;
    }
    if (aa == 0.0) {
        c = 0.0;
        s = cscale(cconj(b), 1.0 / ab);
        return;
    }
    const double r = hypot(aa, ab);
    c = aa / r;
    s = cscale(cmul(cscale(a, 1.0 / aa), cconj(b)), 1.0 / r);
}

// eigenvalue of [[a, b], [c, d]] closest to d
__device__ __forceinline__ cplx wilkinson(cplx a, cplx b, cplx c, cplx d) {
    const cplx half = cscale(csub(a, d), 0.5);
    const cplx disc = csqrt_p(cfma(half, half, cmul(b, c)));
    const cplx mid = cscale(cadd(a, d), 0.5);
    const cplx e1 = cadd(mid, disc), e2 = csub(mid, disc);
    return cabs1(csub(e1, d)) <= cabs1(csub(e2, d)) ? e1 : e2;
}

struct SchurShared {
    int lo, hi, done, info;
    double c[2];
    cplx s[2];
};

// T <- Q^H H Q upper triangular, Z <- Z Q. Returns info (0, or hi+1 when the
// sweep cap ran out with rows 0..hi unconverged).
//
// Each sweep chases one bulge down [lo, hi]. Thread 0 owns the near-diagonal
// "corner" of every step k (column k-1 of rows k, k+1; the 2x2 block at
// (k, k); row k+2 at columns k, k+1) and computes rotation k+1 from it, while
// the other threads apply rotation k to the far parts (rows k, k+1 right of
// column k+1; columns k, k+1 above row k; Z). The write sets are disjoint and
// rotation k+1 depends only on the corner, so each step needs one barrier.
__device__ int blk_schur(int n, cplx* H, int ldh, cplx* Z, int ldz, SchurShared* sh, int max_sweeps_per_row) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const double eps = 2.220446049250313e-16;
    const double smallnum = 2.2250738585072014e-308 * (n / eps);
    if (tid == 0) {
        sh->hi = n - 1;
        sh->lo = 0;
        sh->done = 0;
        sh->info = 0;
    }
    __syncthreads();
    int iter_row = 0;
    const long max_total = (long)max_sweeps_per_row * n;
    long total = 0;
    while (true) {
        if (tid == 0) {
            int hi = sh->hi;
            while (hi > 0) {
                const cplx sub = H[(size_t)hi * ldh + hi - 1];
                const double tst = cabs1(H[(size_t)(hi - 1) * ldh + hi - 1]) + cabs1(H[(size_t)hi * ldh + hi]);
                if (cabs1(sub) <= fmax(eps * tst, smallnum)) {
                    H[(size_t)hi * ldh + hi - 1] = C(0.0, 0.0);
                    --hi;
                    iter_row = 0;
                } else {
                    break;
                }
            }
            int lo = hi;
            while (lo > 0) {
                const cplx sub = H[(size_t)lo * ldh + lo - 1];
                const double tst = cabs1(H[(size_t)(lo - 1) * ldh + lo - 1]) + cabs1(H[(size_t)lo * ldh + lo]);
                if (cabs1(sub) <= fmax(eps * tst, smallnum)) {
                    H[(size_t)lo * ldh + lo - 1] = C(0.0, 0.0);
                    break;
                }
                --lo;
            }
            sh->hi = hi;
            sh->lo = lo;
            if (hi <= 0) {
                sh->done = 1;
            } else if (total >= max_total) {
                sh->done = 1;
                sh->info = hi + 1;
            } else {
                ++iter_row;
                ++total;
                cplx shift;
                if (iter_row == 10 || iter_row == 30) {  // exceptional shift
                    const double e = fabs(H[(size_t)hi * ldh + hi - 1].x) +
                                     (hi >= 2 ? fabs(H[(size_t)(hi - 1) * ldh + hi - 2].x) : 0.0);
                    shift = cadd(H[(size_t)hi * ldh + hi], C(e, 0.0));
                } else {
                    shift = wilkinson(H[(size_t)(hi - 1) * ldh + hi - 1], H[(size_t)(hi - 1) * ldh + hi],
                                      H[(size_t)hi * ldh + hi - 1], H[(size_t)hi * ldh + hi]);
                }
                double c;
                cplx s;
                givens(csub(H[(size_t)lo * ldh + lo], shift), H[(size_t)(lo + 1) * ldh + lo], c, s);
                sh->c[lo & 1] = c;
                sh->s[lo & 1] = s;
            }
        }
        __syncthreads();
        if (sh->done) break;
        const int lo = sh->lo, hi = sh->hi;
        for (int k = lo; k < hi; ++k) {
            const double c = sh->c[k & 1];
            const cplx s = sh->s[k & 1];
            const cplx ms = cneg(cconj(s));  // row rotation, second row: -conj(s) x + c y
            const cplx cs = cconj(s), ns = cneg(s);  // column rotation
            if (tid == 0) {
                // corner: bulge column k-1, 2x2 block, row k+2
                if (k > lo) {
                    const cplx a = H[(size_t)k * ldh + k - 1], b = H[(size_t)(k + 1) * ldh + k - 1];
                    H[(size_t)k * ldh + k - 1] = cfma(s, b, cscale(a, c));
                    H[(size_t)(k + 1) * ldh + k - 1] = C(0.0, 0.0);
                }
                cplx h00 = H[(size_t)k * ldh + k], h01 = H[(size_t)k * ldh + k + 1];
                cplx h10 = H[(size_t)(k + 1) * ldh + k], h11 = H[(size_t)(k + 1) * ldh + k + 1];
                const cplx r00 = cfma(s, h10, cscale(h00, c)), r01 = cfma(s, h11, cscale(h01, c));
                const cplx r10 = cfma(ms, h00, cscale(h10, c)), r11 = cfma(ms, h01, cscale(h11, c));
                H[(size_t)k * ldh + k] = cfma(cs, r01, cscale(r00, c));
                H[(size_t)k * ldh + k + 1] = cfma(ns, r00, cscale(r01, c));
                H[(size_t)(k + 1) * ldh + k] = cfma(cs, r11, cscale(r10, c));
                H[(size_t)(k + 1) * ldh + k + 1] = cfma(ns, r10, cscale(r11, c));
                if (k + 2 <= hi) {
                    const cplx x = H[(size_t)(k + 2) * ldh + k], y = H[(size_t)(k + 2) * ldh + k + 1];
                    H[(size_t)(k + 2) * ldh + k] = cfma(cs, y, cscale(x, c));
                    H[(size_t)(k + 2) * ldh + k + 1] = cfma(ns, x, cscale(y, c));
                }
                if (k + 1 < hi) {  // next rotation annihilates the new bulge H[k+2][k]
                    double c2;
                    cplx s2;
                    givens(H[(size_t)(k + 1) * ldh + k], H[(size_t)(k + 2) * ldh + k], c2, s2);
                    sh->c[(k + 1) & 1] = c2;
                    sh->s[(k + 1) & 1] = s2;
                }
            }
            // far part of the row rotation: rows k, k+1, columns k+2..n-1
            for (int j = k + 2 + tid; j < n; j += nt) {
                const cplx x = H[(size_t)k * ldh + j], y = H[(size_t)(k + 1) * ldh + j];
                H[(size_t)k * ldh + j] = cfma(s, y, cscale(x, c));
                H[(size_t)(k + 1) * ldh + j] = cfma(ms, x, cscale(y, c));
            }
            // far part of the column rotation: rows 0..k-1, columns k, k+1
            for (int i = tid; i < k; i += nt) {
                const cplx x = H[(size_t)i * ldh + k], y = H[(size_t)i * ldh + k + 1];
                H[(size_t)i * ldh + k] = cfma(cs, y, cscale(x, c));
                H[(size_t)i * ldh + k + 1] = cfma(ns, x, cscale(y, c));
            }
            for (int i = tid; i < n; i += nt) {
                const cplx x = Z[(size_t)i * ldz + k], y = Z[(size_t)i * ldz + k + 1];
                Z[(size_t)i * ldz + k] = cfma(cs, y, cscale(x, c));
                Z[(size_t)i * ldz + k + 1] = cfma(ns, x, cscale(y, c));
            }
            __syncthreads();
        }
    }
    const int info = sh->info;
    __syncthreads();
    return info;
}

// ---- eigenvectors of the triangular Schur factor ----------------------------------------
// X (n x n, row-major) <- right eigenvectors of upper-triangular T: column k
// solves (T - t_kk I) x = 0 with x_k = 1, x_i = 0 for i > k (ztrevc's back
// substitution, with tiny denominators replaced by smin). Columns are then
// scaled to unit max |re|+|im|.
__device__ void blk_trevc(int n, const cplx* T, int ldt, cplx* X, int ldx) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const double eps = 2.220446049250313e-16;
    const double tiny = 2.2250738585072014e-308 / eps;
    for (int e = tid; e < n * n; e += nt) {
        const int i = e / n, k = e % n;
        X[(size_t)i * ldx + k] = C(i == k ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int k = tid; k < n; k += nt) {
        const cplx lam = T[(size_t)k * ldt + k];
        const double smin = fmax(eps * cabs1(lam), tiny);
        double xmax = 1.0;
        for (int i = k - 1; i >= 0; --i) {
            cplx acc = C(0.0, 0.0);
            for (int j = i + 1; j <= k; ++j) acc = cfma(T[(size_t)i * ldt + j], X[(size_t)j * ldx + k], acc);
            cplx den = csub(T[(size_t)i * ldt + i], lam);
            if (cabs1(den) < smin) den = C(smin, 0.0);
            const cplx xi = cneg(cdiv(acc, den));
            X[(size_t)i * ldx + k] = xi;
            xmax = fmax(xmax, cabs1(xi));
            if (xmax > 1e100) {  // rescale the partial vector to avoid overflow
                const double sc = 1.0 / xmax;
                for (int j = i; j <= k; ++j) X[(size_t)j * ldx + k] = cscale(X[(size_t)j * ldx + k], sc);
                xmax = 1.0;
            }
        }
        const double sc = 1.0 / xmax;
        for (int j = 0; j <= k; ++j) X[(size_t)j * ldx + k] = cscale(X[(size_t)j * ldx + k], sc);
    }
    __syncthreads();
}

}  // namespace cb
