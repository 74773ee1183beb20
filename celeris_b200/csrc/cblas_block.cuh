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
//   blk_gemm        C = alpha A B + beta C (FP64 tensor-core DMMA, smem-staged k chunks)
//   blk_lu          partial-pivot LU in place (LAPACK zgetrf semantics: pivot =
//                   first max |re|+|im| in the column); blk_lu_blocked: panels
//                   of LNB columns with GEMM trailing updates, same pivots
//   blk_lu_solve    X = A^{-1} B from the LU factors, any number of RHS
//                   (blk_lu_solve_blocked: block rows with GEMM updates)
//   blk_hessenberg_refl  Householder reduction to upper Hessenberg (shared H),
//                   reflectors recorded; blk_form_q forms Q from them
//                   (blk_hessenberg_blocked: compact-WY panels, GEMM updates, Z
//                   accumulated)
//   givens, wilkinson  rotation and shift helpers of the Schur form (schur_aed.cuh)
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
// FP64 tensor cores: mma.sync.m8n8k4 (DMMA). The CTA computes a 64 x (NT/4)
// output tile from k-chunks of GKC; each warp owns a 32 x 16 block = 4 x 2 tiles
// of 8 x 8. A complex product over a k-step of 4 is four real DMMAs per tile:
// Re += Ar Br + (-Ai) Bi, Im += Ar Bi + Ai Br. Fragment layout of m8n8k4
// (g = lane / 4, t = lane % 4): A[g][t] (row-major 8 x 4), B[t][g] (column-major
// 4 x 8), C[g][2t], C[g][2t + 1].
// Chunks stream into two shared buffers with cp.async (16-byte copies,
// zero-filled past the edges): chunk g+1 is in flight while chunk g is
// multiplied, in one pipeline over all (tile, chunk) steps. The accumulators
// start from (beta / alpha) C and the tile is stored as alpha * acc.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    const int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

constexpr int GM = 64;   // tile rows
constexpr int GKC = 8;   // k chunk
struct GemmSmem {
    cplx a[2][GM][GKC + 1];  // A chunks, row-major; +1 spreads a fragment's rows over the banks
    cplx b[2][GKC][64];      // B chunks
};

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <int NT>
__device__ __forceinline__ void gemm_tiles(int m, int n, int k, cplx alpha, const cplx* A, int lda, const cplx* B,
                                           int ldb, cplx beta, cplx* Cm, int ldc, GemmSmem* sm) {
    constexpr int GN = NT / 4;
    constexpr int WC = GN / 16;  // warps across the columns (4 or 2); 2 across the rows
    const int tid = threadIdx.x;
    const bool act = tid < NT;
    const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
    const int wr = (warp / WC) * 32, wc = (warp % WC) * 16;  // warp block origin in the tile
    const int mt = (m + GM - 1) / GM, ntl = (n + GN - 1) / GN;
    const int nk = (k + GKC - 1) / GKC;
    const int total = mt * ntl * nk;  // (tile, k-chunk) steps
    if (total == 0) return;
    const bool use_beta = beta.x != 0.0 || beta.y != 0.0;
    const cplx ab = use_beta ? cdiv(beta, alpha) : C(0.0, 0.0);
    double cr[4][2][2], ci[4][2][2];  // [row tile][col tile][2 per thread]
    auto issue = [&](int gi) {
        const int t = gi / nk, k0 = (gi - t * nk) * GKC;
        const int i0 = (t / ntl) * GM, j0 = (t % ntl) * GN, buf = gi & 1;
        if (act) {
            for (int e = tid; e < GM * GKC; e += NT) {
                const int r = e / GKC, c = e % GKC;
                const bool v = i0 + r < m && k0 + c < k;
                cp_async16(&sm->a[buf][r][c], v ? A + (size_t)(i0 + r) * lda + k0 + c : A, v);
            }
            for (int e = tid; e < GKC * GN; e += NT) {
                const int r = e / GN, c = e % GN;
                const bool v = k0 + r < k && j0 + c < n;
                cp_async16(&sm->b[buf][r][c], v ? B + (size_t)(k0 + r) * ldb + j0 + c : B, v);
            }
        }
        cp_async_commit();
    };
    auto init_acc = [&](int t) {
        const int i0 = (t / ntl) * GM, j0 = (t % ntl) * GN;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = i0 + wr + 8 * i + g;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = j0 + wc + 8 * j + 2 * t4 + h;
                    cplx v = C(0.0, 0.0);
                    if (use_beta && act && r < m && c < n) v = cmul(ab, Cm[(size_t)r * ldc + c]);
                    cr[i][j][h] = v.x;
                    ci[i][j][h] = v.y;
                }
            }
        }
    };
    init_acc(0);
    issue(0);
    for (int gi = 0; gi < total; ++gi) {
        if (gi + 1 < total) {
            issue(gi + 1);
            cp_async_wait1();
        } else {
            cp_async_wait0();
        }
        __syncthreads();
        if (act) {
            const int buf = gi & 1;
#pragma unroll
            for (int ks = 0; ks < GKC; ks += 4) {
                double ar[4], ai[4], nai[4], br[2], bi[2];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const cplx v = sm->a[buf][wr + 8 * i + g][ks + t4];
                    ar[i] = v.x;
                    ai[i] = v.y;
                    nai[i] = -v.y;
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const cplx v = sm->b[buf][ks + t4][wc + 8 * j + g];
                    br[j] = v.x;
                    bi[j] = v.y;
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        dmma(cr[i][j][0], cr[i][j][1], ar[i], br[j]);
                        dmma(cr[i][j][0], cr[i][j][1], nai[i], bi[j]);
                        dmma(ci[i][j][0], ci[i][j][1], ar[i], bi[j]);
                        dmma(ci[i][j][0], ci[i][j][1], ai[i], br[j]);
                    }
            }
        }
        __syncthreads();  // buffer gi & 1 is refilled by the issue of step gi + 2
        const int t = gi / nk;
        if (gi - t * nk == nk - 1) {  // last chunk of tile t: store it, start the next
            if (act) {
                const int i0 = (t / ntl) * GM, j0 = (t % ntl) * GN;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = i0 + wr + 8 * i + g;
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int c = j0 + wc + 8 * j + 2 * t4 + h;
                            if (r < m && c < n) Cm[(size_t)r * ldc + c] = cmul(alpha, C(cr[i][j][h], ci[i][j][h]));
                        }
                    }
                }
            }
            if (gi + 1 < total) init_acc(t + 1);
        }
    }
}

// Warp-tiled product for small inner dimension or a thin output (k <= 32, m <= 16
// or n <= 16: the rank-16 updates of the blocked LU, solves and Hessenberg, and
// the 16-wide products of the compact WY form). Each warp owns 16 x (8 TN)
// output blocks, round-robin, and streams its A rows and B columns straight from
// memory into DMMA fragments, so the eight warps keep eight tiles' loads in
// flight instead of one CTA-wide tile's.
template <int TN>
__device__ __forceinline__ void gemm_warps(int m, int n, int k, cplx alpha, const cplx* A, int lda, const cplx* B,
                                           int ldb, cplx beta, cplx* Cm, int ldc) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int mt = (m + 15) / 16, ntl = (n + 8 * TN - 1) / (8 * TN);
    const bool use_beta = beta.x != 0.0 || beta.y != 0.0;
    const cplx ab = use_beta ? cdiv(beta, alpha) : C(0.0, 0.0);
    for (int t = warp; t < mt * ntl; t += nwarp) {
        const int r0 = (t / ntl) * 16, c0 = (t % ntl) * (8 * TN);
        double cr[2][TN][2], ci[2][TN][2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = r0 + 8 * i + g;
#pragma unroll
            for (int j = 0; j < TN; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = c0 + 8 * j + 2 * t4 + h;
                    cplx v = C(0.0, 0.0);
                    if (use_beta && r < m && c < n) v = cmul(ab, Cm[(size_t)r * ldc + c]);
                    cr[i][j][h] = v.x;
                    ci[i][j][h] = v.y;
                }
        }
#pragma unroll 4
        for (int k0 = 0; k0 < k; k0 += 4) {
            const int kk = k0 + t4;
            cplx a[2], b[TN];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = r0 + 8 * i + g;
                a[i] = (r < m && kk < k) ? A[(size_t)r * lda + kk] : C(0.0, 0.0);
            }
#pragma unroll
            for (int j = 0; j < TN; ++j) {
                const int c = c0 + 8 * j + g;
                b[j] = (kk < k && c < n) ? B[(size_t)kk * ldb + c] : C(0.0, 0.0);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) {
                    dmma(cr[i][j][0], cr[i][j][1], a[i].x, b[j].x);
                    dmma(cr[i][j][0], cr[i][j][1], -a[i].y, b[j].y);
                    dmma(ci[i][j][0], ci[i][j][1], a[i].x, b[j].y);
                    dmma(ci[i][j][0], ci[i][j][1], a[i].y, b[j].x);
                }
        }
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = r0 + 8 * i + g;
            if (r >= m) continue;
#pragma unroll
            for (int j = 0; j < TN; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = c0 + 8 * j + 2 * t4 + h;
                    if (c < n) Cm[(size_t)r * ldc + c] = cmul(alpha, C(cr[i][j][h], ci[i][j][h]));
                }
        }
    }
}

// C[m x n] = alpha * A[m x k] * B[k x n] + beta * C  (row-major). C may not alias A
// or B. blockDim.x >= 128 (every kernel here runs 128 or 256 threads).
__device__ void blk_gemm(int m, int n, int k, cplx alpha, const cplx* A, int lda, const cplx* B, int ldb,
                         cplx beta, cplx* Cm, int ldc, GemmSmem* sm) {
    __syncthreads();
    if (n <= 16)
        gemm_warps<2>(m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc);
    else if (k <= 32 || m <= 16)
        gemm_warps<4>(m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc);
    else if (blockDim.x >= 256)
        gemm_tiles<256>(m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, sm);
    else
        gemm_tiles<128>(m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, sm);
    __syncthreads();
}

// ---- rank-1 update ----------------------------------------------------------------------
// A[i][j] -= x[i] * y[j] (or * conj(y[j])) for i < rows, j < cols. Warps take
// rows, lanes take columns (32 apart, up to 128 columns per pass, y held in
// registers for the pass); each warp loads two rows' elements before it stores
// any (a load-use-store loop would wait on every load, the compiler being
// unable to move loads past stores to the same array), so up to 8 loads per
// thread are in flight, and no index is divided.
// x and y are shared-memory vectors that do not overlap A.
template <bool CONJ_Y>
__device__ __forceinline__ void blk_rank1(int rows, int cols, cplx* A, int lda, const cplx* x, const cplx* y) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int j0 = 0; j0 < cols; j0 += 128) {
        cplx yy[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = j0 + 32 * u + lane;
            ok[u] = j < cols;
            yy[u] = ok[u] ? (CONJ_Y ? cconj(y[j]) : y[j]) : C(0.0, 0.0);
        }
        for (int i = warp; i < rows; i += 2 * nwarp) {
            const int i2 = i + nwarp;
            const bool two = i2 < rows;
            cplx* r1 = A + (size_t)i * lda + j0 + lane;
            cplx* r2 = A + (size_t)(two ? i2 : i) * lda + j0 + lane;
            cplx a[4], c[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (ok[u]) a[u] = r1[32 * u];
                if (ok[u] && two) c[u] = r2[32 * u];
            }
            const cplx x1 = x[i], x2 = two ? x[i2] : C(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (ok[u]) r1[32 * u] = cfms(x1, yy[u], a[u]);
                if (ok[u] && two) r2[32 * u] = cfms(x2, yy[u], c[u]);
            }
        }
    }
}

// ---- LU ------------------------------------------------------------------------------
// In-place LU with partial pivoting of the n x n matrix A. piv[k] = row swapped
// with k at step k. Returns 0, or k+1 for the first exactly-zero pivot (the
// factorization continues, like zgetrf). stage: shared scratch of 2n complex
// (the pivot column and row of each step, so the trailing update reads only
// its own element from A).
__device__ int blk_lu(int n, cplx* A, int lda, int* piv, RedScratch* rs, cplx* stage) {
    const int tid = threadIdx.x, nt = blockDim.x;
    int info = 0;
    cplx* colk = stage;
    cplx* rowk = stage + n;
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
        const int w = n - k - 1;
        for (int i = tid; i < w; i += nt) {
            const cplx l = cmul(A[(size_t)(k + 1 + i) * lda + k], inv);
            A[(size_t)(k + 1 + i) * lda + k] = l;
            colk[i] = l;
            rowk[i] = A[(size_t)k * lda + k + 1 + i];
        }
        __syncthreads();
        blk_rank1<false>(w, w, A + (size_t)(k + 1) * lda + k + 1, lda, colk, rowk);
        __syncthreads();
    }
    return info;
}

// B (n x nrhs, row-major, ldb) <- A^{-1} B using the factors of blk_lu.
// stage: shared scratch of n + nrhs complex.
__device__ void blk_lu_solve(int n, const cplx* LU, int lda, const int* piv, int nrhs, cplx* B, int ldb,
                             cplx* stage) {
    const int tid = threadIdx.x, nt = blockDim.x;
    cplx* lcol = stage;
    cplx* brow = stage + n;
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
        for (int i = tid; i < w; i += nt) lcol[i] = LU[(size_t)(j + 1 + i) * lda + j];
        for (int r = tid; r < nrhs; r += nt) brow[r] = B[(size_t)j * ldb + r];
        __syncthreads();
        blk_rank1<false>(w, nrhs, B + (size_t)(j + 1) * ldb, ldb, lcol, brow);
        __syncthreads();
    }
    // backward: U
    for (int j = n - 1; j >= 0; --j) {
        const cplx inv = cinv(LU[(size_t)j * lda + j]);
        for (int r = tid; r < nrhs; r += nt) {
            const cplx x = cmul(B[(size_t)j * ldb + r], inv);
            B[(size_t)j * ldb + r] = x;
            brow[r] = x;
        }
        for (int i = tid; i < j; i += nt) lcol[i] = LU[(size_t)i * lda + j];
        __syncthreads();
        blk_rank1<false>(j, nrhs, B, ldb, lcol, brow);
        __syncthreads();
    }
}

// w[i] = beta * sum_j A[i][j] v[j] for i < rows, j < cols: one warp per group
// of 4 rows, lanes over j, so every lane has 4 row loads in flight.
__device__ __forceinline__ void blk_matvec_rows(int rows, int cols, const cplx* A, int lda, const cplx* v, cplx* w,
                                                double beta, int warp, int lane, int nwarp) {
    for (int i0 = 4 * warp; i0 < rows; i0 += 4 * nwarp) {
        cplx acc[4] = {C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0)};
#pragma unroll 4
        for (int j = lane; j < cols; j += 32) {
            const cplx vj = v[j];
            cplx h[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) h[r] = (i0 + r < rows) ? A[(size_t)(i0 + r) * lda + j] : C(0.0, 0.0);
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[r] = cfma(h[r], vj, acc[r]);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            for (int o = 16; o > 0; o >>= 1) {
                acc[r].x += __shfl_down_sync(0xffffffffu, acc[r].x, o);
                acc[r].y += __shfl_down_sync(0xffffffffu, acc[r].y, o);
            }
            if (lane == 0 && i0 + r < rows) w[i0 + r] = cscale(acc[r], beta);
        }
    }
}

// Two right-hand sides at once: w(i, r) (+)= sum_j A[i][j] v[j][r], r = 0, 1,
// v row-major [cols][2] (shared memory), w(i, r) stored at w[i * wi + r * wr].
// One warp per pair of rows, lanes over j (coalesced row reads).
__device__ __forceinline__ void blk_matvec2(int rows, int cols, const cplx* A, int lda, const cplx* v, cplx* w,
                                            size_t wi, size_t wr, bool accumulate) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int i0 = 2 * warp; i0 < rows; i0 += 2 * nwarp) {
        cplx acc[2][2] = {{C(0.0, 0.0), C(0.0, 0.0)}, {C(0.0, 0.0), C(0.0, 0.0)}};
        const bool two = i0 + 1 < rows;
#pragma unroll 2
        for (int j = lane; j < cols; j += 32) {
            const cplx v0 = v[2 * j], v1 = v[2 * j + 1];
            const cplx a0 = A[(size_t)i0 * lda + j];
            const cplx a1 = two ? A[(size_t)(i0 + 1) * lda + j] : C(0.0, 0.0);
            acc[0][0] = cfma(a0, v0, acc[0][0]);
            acc[0][1] = cfma(a0, v1, acc[0][1]);
            acc[1][0] = cfma(a1, v0, acc[1][0]);
            acc[1][1] = cfma(a1, v1, acc[1][1]);
        }
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int r = 0; r < 2; ++r)
                for (int o = 16; o > 0; o >>= 1) {
                    acc[q][r].x += __shfl_down_sync(0xffffffffu, acc[q][r].x, o);
                    acc[q][r].y += __shfl_down_sync(0xffffffffu, acc[q][r].y, o);
                }
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (q == 1 && !two) break;
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                    cplx* dst = w + (size_t)(i0 + q) * wi + (size_t)r * wr;
                    *dst = accumulate ? cadd(*dst, acc[q][r]) : acc[q][r];
                }
            }
        }
    }
}

// ---- blocked LU and solves ----------------------------------------------------------------
// Column-wise triangular solves of a kb x kb diagonal block T (shared memory,
// row-major kb x kb) against columns j0 .. j0+ncols-1 of the kb-row panel B: one
// thread per column, in place (each thread rereads only what it wrote).
__device__ __forceinline__ void trsm_unit_lower_cols(int kb, const cplx* T, cplx* B, int ldb, int j0, int ncols) {
    for (int j = j0 + threadIdx.x; j < j0 + ncols; j += blockDim.x) {
        cplx* col = B + j;
        for (int r = 1; r < kb; ++r) {
            cplx s = col[(size_t)r * ldb];
            for (int c = 0; c < r; ++c) s = cfms(T[r * kb + c], col[(size_t)c * ldb], s);
            col[(size_t)r * ldb] = s;
        }
    }
}
__device__ __forceinline__ void trsm_upper_cols(int kb, const cplx* T, cplx* B, int ldb, int j0, int ncols) {
    for (int j = j0 + threadIdx.x; j < j0 + ncols; j += blockDim.x) {
        cplx* col = B + j;
        for (int r = kb - 1; r >= 0; --r) {
            cplx s = col[(size_t)r * ldb];
            for (int c = r + 1; c < kb; ++c) s = cfms(T[r * kb + c], col[(size_t)c * ldb], s);
            col[(size_t)r * ldb] = cdiv(s, T[r * kb + r]);
        }
    }
}

// Right-looking LU with partial pivoting in panels of LNB columns: the panel is
// factored with rank-1 steps (full rows swapped at once), the block row of U is
// a small triangular solve, and the trailing matrix is updated by blk_gemm, so
// the O(n^3) part is tiled through shared memory. Same pivot rule and same info
// as blk_lu. stage: >= 2n + LNB*LNB complex of shared memory.
constexpr int LNB = 16;

__device__ int blk_lu_blocked(int n, cplx* A, int lda, int* piv, RedScratch* rs, cplx* stage, GemmSmem* gs) {
    const int tid = threadIdx.x, nt = blockDim.x;
    int info = 0;
    cplx* colk = stage;
    cplx* rowk = stage + n;
    cplx* L11 = stage + 2 * n;
    __syncthreads();
    for (int k0 = 0; k0 < n; k0 += LNB) {
        const int kb = min(LNB, n - k0);
        for (int k = k0; k < k0 + kb; ++k) {
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
            const int m = n - k - 1, w = k0 + kb - 1 - k;  // rows below, panel columns right
            if (akk.x == 0.0 && akk.y == 0.0) {
                if (info == 0) info = k + 1;
                __syncthreads();
                continue;
            }
            const cplx inv = cinv(akk);
            for (int i = tid; i < m; i += nt) {
                const cplx l = cmul(A[(size_t)(k + 1 + i) * lda + k], inv);
                A[(size_t)(k + 1 + i) * lda + k] = l;
                colk[i] = l;
            }
            for (int j = tid; j < w; j += nt) rowk[j] = A[(size_t)k * lda + k + 1 + j];
            __syncthreads();
            if (w > 0) blk_rank1<false>(m, w, A + (size_t)(k + 1) * lda + k + 1, lda, colk, rowk);
            __syncthreads();
        }
        const int r0 = k0 + kb, nr = n - r0;
        if (nr <= 0) continue;
        // U12 = L11^{-1} A12 (unit lower L11), one thread per column
        for (int e = tid; e < kb * kb; e += nt) L11[e] = A[(size_t)(k0 + e / kb) * lda + k0 + e % kb];
        __syncthreads();
        trsm_unit_lower_cols(kb, L11, A + (size_t)k0 * lda, lda, r0, n - r0);
        __syncthreads();
        // A22 -= L21 U12
        blk_gemm(nr, nr, kb, C(-1.0, 0.0), A + (size_t)r0 * lda + k0, lda, A + (size_t)k0 * lda + r0, lda,
                 C(1.0, 0.0), A + (size_t)r0 * lda + r0, lda, gs);
    }
    return info;
}

// ---- Gauss-Jordan in shared memory ----------------------------------------------------
// For matrices small enough to sit in shared memory whole. Each column step
// takes three barriers: warp 0 finds the pivot (first max |re|+|im|, as
// blk_lu) with shuffles; every thread then swaps rows k and p and stages the
// pivot row (scaled by 1/a_kk) and the pivot column; every thread then
// applies the rank-1 elimination to its entries. No triangular solve follows,
// so there are no serial chains besides the pivot search.
// Step k of either routine; ncol columns of M (ld) take part, column k itself
// is handled by the caller's rule (solve: it becomes e_k; inverse: it turns
// into the k-th column of the inverse, Gauss-Jordan in place).
template <bool INVERSE>
__device__ __forceinline__ bool gj_step(int n, int ncol, cplx* M, int ld, int k, cplx* rowv, cplx* colv,
                                        int* sp, cplx* sd) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    if (tid < 32) {  // warp 0: the pivot
        double best = -1.0;
        int bi = k;
        for (int i = k + lane; i < n; i += 32) {
            const double v = cabs1(M[i * ld + k]);
            if (v > best) {
                best = v;
                bi = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            *sp = bi;
            const cplx akk = M[bi * ld + k];
            *sd = (akk.x == 0.0 && akk.y == 0.0) ? C(0.0, 0.0) : cinv(akk);
        }
    }
    __syncthreads();
    const int p = *sp;
    const cplx d = *sd;
    if (d.x == 0.0 && d.y == 0.0) return false;  // singular: the same decision in every thread
    // swap rows k and p; stage the scaled pivot row and the pivot column
    for (int j = tid; j < ncol; j += nt) {
        const cplx vk = M[k * ld + j], vp = M[p * ld + j];
        if (p != k) M[p * ld + j] = vk;
        rowv[j] = cmul(vp, d);
    }
    for (int i = tid; i < n; i += nt) colv[i] = i == p ? M[k * ld + k] : (i == k ? C(0.0, 0.0) : M[i * ld + k]);
    __syncthreads();
    // eliminate: M[i][j] -= colv[i] rowv[j] (i != k); row k <- rowv. A warp
    // per row, lanes over its columns (no index division)
    const int j0 = INVERSE ? 0 : k + 1;  // solve: the columns left of k (and k) are done
    const int warp = tid >> 5, nwarp = nt >> 5;
    for (int i = warp; i < n; i += nwarp) {
        cplx* row = M + i * ld;
        if (i == k) {
            for (int j = j0 + lane; j < ncol; j += 32) row[j] = (INVERSE && j == k) ? d : rowv[j];
        } else {
            const cplx ci = colv[i];
            for (int j = j0 + lane; j < ncol; j += 32)
                row[j] = (INVERSE && j == k) ? cneg(cmul(ci, d)) : cfms(ci, rowv[j], row[j]);
        }
    }
    __syncthreads();
    return true;
}

// [A | B] (n x (n + nrhs), shared; an odd ld keeps column walks free of bank
// conflicts) -> B <- A^-1 B by Gauss-Jordan with partial pivoting (A is
// destroyed). scratch: 2 (n + nrhs) + 1 complex and one int of shared memory.
// Returns 0 or the 1-based column of a zero pivot.
__device__ int blk_gj_solve_smem(int n, int nrhs, cplx* M, int ld, cplx* scratch, int* sp) {
    cplx* rowv = scratch;
    cplx* colv = scratch + n + nrhs;
    cplx* sd = colv + n + nrhs;
    __syncthreads();
    for (int k = 0; k < n; ++k)
        if (!gj_step<false>(n, n + nrhs, M, ld, k, rowv, colv, sp, sd)) return k + 1;
    return 0;
}

// A (n x n, shared, ld) <- A^-1 in place by Gauss-Jordan with partial pivoting
// (rows swapped during the sweep, the inverse's columns swapped back after it).
// scratch: 2 n + 1 complex; piv: n ints of shared memory.
__device__ int blk_gj_inverse_smem(int n, cplx* A, int ld, cplx* scratch, int* piv, int* sp) {
    const int tid = threadIdx.x, nt = blockDim.x;
    cplx* rowv = scratch;
    cplx* colv = scratch + n;
    cplx* sd = colv + n;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (!gj_step<true>(n, n, A, ld, k, rowv, colv, sp, sd)) return k + 1;
        if (tid == 0) piv[k] = *sp;
    }
    __syncthreads();
    for (int k = n - 1; k >= 0; --k) {
        const int p = piv[k];
        if (p != k)
            for (int i = tid; i < n; i += nt) {
                const cplx t = A[i * ld + k];
                A[i * ld + k] = A[i * ld + p];
                A[i * ld + p] = t;
            }
        __syncthreads();
    }
    return 0;
}

// B (n x nrhs) <- A^{-1} B from the factors of blk_lu / blk_lu_blocked, by
// block rows: a small triangular solve per block (one thread per RHS column)
// and a blk_gemm update of the remaining rows. stage: >= LNB*LNB complex.
__device__ void blk_lu_solve_blocked(int n, const cplx* LU, int lda, const int* piv, int nrhs, cplx* B, int ldb,
                                     cplx* stage, GemmSmem* gs) {
    const int tid = threadIdx.x, nt = blockDim.x;
    cplx* Tkk = stage;
    __syncthreads();
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
    // forward: unit lower
    for (int k0 = 0; k0 < n; k0 += LNB) {
        const int kb = min(LNB, n - k0);
        for (int e = tid; e < kb * kb; e += nt) Tkk[e] = LU[(size_t)(k0 + e / kb) * lda + k0 + e % kb];
        __syncthreads();
        trsm_unit_lower_cols(kb, Tkk, B + (size_t)k0 * ldb, ldb, 0, nrhs);
        __syncthreads();
        const int r0 = k0 + kb;
        if (r0 < n)
            blk_gemm(n - r0, nrhs, kb, C(-1.0, 0.0), LU + (size_t)r0 * lda + k0, lda, B + (size_t)k0 * ldb, ldb,
                     C(1.0, 0.0), B + (size_t)r0 * ldb, ldb, gs);
    }
    // backward: upper (with diagonal)
    const int nblk = (n + LNB - 1) / LNB;
    for (int bI = nblk - 1; bI >= 0; --bI) {
        const int k0 = bI * LNB, kb = min(LNB, n - k0);
        for (int e = tid; e < kb * kb; e += nt) Tkk[e] = LU[(size_t)(k0 + e / kb) * lda + k0 + e % kb];
        __syncthreads();
        trsm_upper_cols(kb, Tkk, B + (size_t)k0 * ldb, ldb, 0, nrhs);
        __syncthreads();
        if (k0 > 0)
            blk_gemm(k0, nrhs, kb, C(-1.0, 0.0), LU + k0, lda, B + (size_t)k0 * ldb, ldb, C(1.0, 0.0), B, ldb, gs);
    }
}

// ---- Hessenberg reduction ------------------------------------------------------------
// H (n x n) <- Q^H H Q upper Hessenberg by Householder reflectors
// P_k = I - beta v v^H (beta real, P_k Hermitian and unitary), applied from
// both sides one column at a time.
// Reflector k (v_k of length m = n-k-1, beta_k;
// beta_k = 0 where column k needed none) is recorded in row k of `refl`
// (n x n, global): v_k in [0, m), beta_k in the real part of entry n-1.
// blk_form_q builds Q from these afterwards. For a shared-memory H this keeps
// every per-column pass in shared memory (the forward accumulation of Z is a
// matrix-vector product and a rank-1 update of an n x n global matrix per
// column).
__device__ void blk_hessenberg_refl(int n, cplx* H, int ldh, cplx* refl, cplx* v, cplx* w, RedScratch* rs) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nwarp = nt >> 5;
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        cplx* rk = refl + (size_t)k * n;
        double s = 0.0;
        for (int i = tid; i < m; i += nt) s += cnorm2(H[(size_t)(k + 1 + i) * ldh + k]);
        const double xnorm2 = blk_sum(s, rs);
        const cplx x0 = H[(size_t)(k + 1) * ldh + k];
        const double tail = xnorm2 - cnorm2(x0);
        if (tail <= 0.0) {  // already zero below the subdiagonal
            if (tid == 0) rk[n - 1] = C(0.0, 0.0);
            __syncthreads();
            continue;
        }
        const double xn = sqrt(xnorm2);
        const double ax0 = cabs(x0);
        const cplx ph = ax0 > 0.0 ? cscale(x0, 1.0 / ax0) : C(1.0, 0.0);
        const cplx alpha = cscale(ph, -xn);
        const cplx v0 = csub(x0, alpha);
        const double beta = 2.0 / (tail + cnorm2(v0));
        for (int i = tid; i < m; i += nt) {
            const cplx vi = (i == 0) ? v0 : H[(size_t)(k + 1 + i) * ldh + k];
            v[i] = vi;
            rk[i] = vi;
        }
        if (tid == 0) rk[n - 1] = C(beta, 0.0);
        __syncthreads();
        for (int j = k + 1 + tid; j < n; j += nt) {
            const cplx* col = H + (size_t)(k + 1) * ldh + j;
            cplx acc[4] = {C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0)};
            int i = 0;
            for (; i + 8 <= m; i += 8) {
                cplx h[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) h[u] = col[(size_t)(i + u) * ldh];
#pragma unroll
                for (int u = 0; u < 8; ++u) acc[u & 3] = cfma(cconj(v[i + u]), h[u], acc[u & 3]);
            }
            for (; i < m; ++i) acc[0] = cfma(cconj(v[i]), col[(size_t)i * ldh], acc[0]);
            w[j] = cscale(cadd(cadd(acc[0], acc[1]), cadd(acc[2], acc[3])), beta);
        }
        __syncthreads();
        blk_rank1<false>(m, n - k - 1, H + (size_t)(k + 1) * ldh + k + 1, ldh, v, w + k + 1);
        for (int i = tid; i < m; i += nt) H[(size_t)(k + 1 + i) * ldh + k] = (i == 0) ? alpha : C(0.0, 0.0);
        __syncthreads();
        if (m <= 48) {
            // short rows: one thread per row, no shuffle reduction on the chain
            for (int i = tid; i < n; i += nt) {
                const cplx* row = H + (size_t)i * ldh + k + 1;
                cplx acc[4] = {C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0)};
                int j = 0;
                for (; j + 4 <= m; j += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[u] = cfma(row[j + u], v[j + u], acc[u]);
                }
                for (; j < m; ++j) acc[0] = cfma(row[j], v[j], acc[0]);
                w[i] = cscale(cadd(cadd(acc[0], acc[1]), cadd(acc[2], acc[3])), beta);
            }
        } else {
            blk_matvec_rows(n, m, H + k + 1, ldh, v, w, beta, warp, lane, nwarp);
        }
        __syncthreads();
        blk_rank1<true>(n, m, H + k + 1, ldh, w, v);
        __syncthreads();
    }
}

// Q = P_0 P_1 ... P_{n-3} from the reflectors of blk_hessenberg_refl, formed
// backward in Z (n x n, shared): Z = I, then Z <- P_k Z for k = n-3 .. 0.
// Before step k, Z is the identity outside its trailing block from k+2, so P_k
// changes only Z[k+1:, k+1:] (LAPACK's xUNGHR order). v, w: scratch of length n.
__device__ void blk_form_q(int n, cplx* Z, int ldz, const cplx* refl, cplx* v, cplx* w) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < n * n; e += nt) {
        const int i = e / n, j = e % n;
        Z[(size_t)i * ldz + j] = C(i == j ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int k = n - 3; k >= 0; --k) {
        const int m = n - k - 1;
        const cplx* rk = refl + (size_t)k * n;
        const double beta = rk[n - 1].x;
        if (beta == 0.0) continue;  // the same value in every thread
        for (int i = tid; i < m; i += nt) v[i] = rk[i];
        __syncthreads();
        // w[j] = beta * sum_i conj(v[i]) Z[k+1+i][k+1+j]
        for (int j = tid; j < m; j += nt) {
            const cplx* col = Z + (size_t)(k + 1) * ldz + k + 1 + j;
            cplx acc[4] = {C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0), C(0.0, 0.0)};
            int i = 0;
            for (; i + 8 <= m; i += 8) {
                cplx h[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) h[u] = col[(size_t)(i + u) * ldz];
#pragma unroll
                for (int u = 0; u < 8; ++u) acc[u & 3] = cfma(cconj(v[i + u]), h[u], acc[u & 3]);
            }
            for (; i < m; ++i) acc[0] = cfma(cconj(v[i]), col[(size_t)i * ldz], acc[0]);
            w[j] = cscale(cadd(cadd(acc[0], acc[1]), cadd(acc[2], acc[3])), beta);
        }
        __syncthreads();
        blk_rank1<false>(m, m, Z + (size_t)(k + 1) * ldz + k + 1, ldz, v, w);
        __syncthreads();
    }
}

// Blocked Householder reduction (panels of LNB columns, compact WY form).
// Reflector P_j = I - b_j v_j v_j^H (b_j real, P_j Hermitian) as in
// blk_hessenberg_refl; a panel's product is Q = I - V T V^H with T upper triangular.
// For each panel column the right update by the earlier reflectors uses
// Y = A V T (A at the panel start), the left update applies Q_prev^H to that
// column only, and Y gains A v_j by one matrix-vector product over the columns
// right of it (untouched within the panel). After the panel the trailing
// columns get A <- A - Y V^H, then A <- (I - V T^H V^H) A, and Z <- Z - (Z V T) V^H,
// all by blk_gemm. Memory traffic per column is one read of the trailing
// matrix (the product A v_j) plus 1/LNB of a few passes for the GEMMs, against
// ~8 passes for rank-1 updates.
// scratch (global, >= 5 * LNB * n complex); stage (shared, >= n + LNB^2 + 2 LNB complex).
// prof (optional): clock64 sums [0] column steps without the matrix-vector
// product, [1] the products A v_j, [2] the trailing and Z updates.
__device__ void blk_hessenberg_blocked(int n, cplx* H, int ldh, cplx* Z, int ldz, cplx* scratch, cplx* stage,
                                       RedScratch* rs, GemmSmem* gs, long long* prof = nullptr) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nwarp = nt >> 5;
    constexpr int NB = LNB;
    cplx* V = scratch;                    // [m x NB] (row r <-> index k+1+r)
    cplx* VH = V + (size_t)NB * n;        // [NB x n]: conj(V)^T, leading dimension n
    cplx* Y = VH + (size_t)NB * n;        // [n x NB]
    cplx* Wt = Y + (size_t)NB * n;        // [NB x n]
    cplx* P = Wt + (size_t)NB * n;        // [n x NB]
    cplx* v = stage;                      // [n] current reflector (index i+1 .. n-1)
    cplx* Tm = stage + n;                 // [NB x NB]
    cplx* u = Tm + NB * NB;               // [NB]
    cplx* wv = u + NB;                    // [NB]
    for (int e = tid; e < n * n; e += nt) {
        const int i = e / n, j = e % n;
        Z[(size_t)i * ldz + j] = C(i == j ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int k = 0; k + 2 < n; k += NB) {
        const int kb = min(NB, n - 2 - k);
        const int m = n - k - 1;
        for (int e = tid; e < m * NB; e += nt) V[e] = C(0.0, 0.0);
        for (int e = tid; e < NB * NB; e += nt) Tm[e] = C(0.0, 0.0);
        __syncthreads();
        const long long tc0 = clock64();
        for (int j = 0; j < kb; ++j) {
            const int i = k + j;
            if (j > 0) {
                // (1) column i <- column i of A Q_prev:  H[:, i] -= Y[:, :j] conj(V[j-1, :j])
                for (int r = tid; r < n; r += nt) {
                    cplx s = H[(size_t)r * ldh + i];
                    for (int l = 0; l < j; ++l) s = csub(s, cmul(Y[(size_t)r * NB + l], cconj(V[(size_t)(j - 1) * NB + l])));
                    H[(size_t)r * ldh + i] = s;
                }
                __syncthreads();
                // (2) rows k+1.. of column i <- Q_prev^H b = b - V T^H (V^H b)
                for (int l = warp; l < j; l += nwarp) {
                    cplx s = C(0.0, 0.0);
                    for (int r = l + lane; r < m; r += 32)
                        s = cfma(cconj(V[(size_t)r * NB + l]), H[(size_t)(k + 1 + r) * ldh + i], s);
                    for (int o = 16; o > 0; o >>= 1) {
                        s.x += __shfl_down_sync(0xffffffffu, s.x, o);
                        s.y += __shfl_down_sync(0xffffffffu, s.y, o);
                    }
                    if (lane == 0) u[l] = s;
                }
                __syncthreads();
                if (tid < j) {  // wv = T^H u (T upper: (T^H)[l][p] = conj(T[p][l]), p <= l)
                    cplx s = C(0.0, 0.0);
                    for (int p = 0; p <= tid; ++p) s = cfma(cconj(Tm[p * NB + tid]), u[p], s);
                    wv[tid] = s;
                }
                __syncthreads();
                for (int r = tid; r < m; r += nt) {
                    cplx s = H[(size_t)(k + 1 + r) * ldh + i];
                    for (int l = 0; l < j; ++l) s = csub(s, cmul(V[(size_t)r * NB + l], wv[l]));
                    H[(size_t)(k + 1 + r) * ldh + i] = s;
                }
                __syncthreads();
            }
            // (3) reflector from x = H[i+1:, i]
            const int mx = n - i - 1;
            double s2 = 0.0;
            for (int r = tid; r < mx; r += nt) s2 += cnorm2(H[(size_t)(i + 1 + r) * ldh + i]);
            const double xnorm2 = blk_sum(s2, rs);
            const cplx x0 = H[(size_t)(i + 1) * ldh + i];
            const double tail = xnorm2 - cnorm2(x0);
            double beta = 0.0;
            cplx alpha = x0, v0 = C(0.0, 0.0);
            if (tail > 0.0) {
                const double xn = sqrt(xnorm2), ax0 = cabs(x0);
                const cplx ph = ax0 > 0.0 ? cscale(x0, 1.0 / ax0) : C(1.0, 0.0);
                alpha = cscale(ph, -xn);
                v0 = csub(x0, alpha);
                beta = 2.0 / (tail + cnorm2(v0));
            }
            for (int r = tid; r < mx; r += nt) {
                const cplx vr = beta == 0.0 ? C(0.0, 0.0) : (r == 0 ? v0 : H[(size_t)(i + 1 + r) * ldh + i]);
                v[r] = vr;
                V[(size_t)(j + r) * NB + j] = vr;
            }
            __syncthreads();
            for (int r = tid; r < mx; r += nt) H[(size_t)(i + 1 + r) * ldh + i] = (r == 0) ? alpha : C(0.0, 0.0);
            // (4) u = V_prev^H v_j; Y[:, j] = beta (A v_j - Y_prev u); T[:j, j] = -beta T_prev u
            for (int l = warp; l < j; l += nwarp) {
                cplx s = C(0.0, 0.0);
                for (int r = j + lane; r < m; r += 32) s = cfma(cconj(V[(size_t)r * NB + l]), v[r - j], s);
                for (int o = 16; o > 0; o >>= 1) {
                    s.x += __shfl_down_sync(0xffffffffu, s.x, o);
                    s.y += __shfl_down_sync(0xffffffffu, s.y, o);
                }
                if (lane == 0) u[l] = s;
            }
            const long long tm0 = clock64();
            blk_matvec_rows(n, mx, H + i + 1, ldh, v, P, 1.0, warp, lane, nwarp);  // P[:n] as a vector
            __syncthreads();
            if (prof && tid == 0) prof[1] += clock64() - tm0;
            if (tid < j) {
                cplx s = C(0.0, 0.0);
                for (int p = tid; p < j; ++p) s = cfma(Tm[tid * NB + p], u[p], s);
                wv[tid] = cscale(s, -beta);
            }
            for (int r = tid; r < n; r += nt) {
                cplx s = P[r];
                for (int l = 0; l < j; ++l) s = csub(s, cmul(Y[(size_t)r * NB + l], u[l]));
                Y[(size_t)r * NB + j] = cscale(s, beta);
            }
            __syncthreads();
            if (tid < j) Tm[tid * NB + j] = wv[tid];
            if (tid == 0) Tm[j * NB + j] = C(beta, 0.0);
            __syncthreads();
        }
        if (prof && tid == 0) prof[0] += clock64() - tc0;
        const long long tg0 = clock64();
        for (int e = tid; e < NB * m; e += nt) {
            const int l = e / m, r = e % m;
            VH[(size_t)l * n + r] = l < kb ? cconj(V[(size_t)r * NB + l]) : C(0.0, 0.0);
        }
        // (5) trailing columns c >= k+kb  (V row kb-1 <-> index k+kb)
        const int c0 = k + kb, nc = n - c0;
        if (nc > 0) {
            blk_gemm(n, nc, kb, C(-1.0, 0.0), Y, NB, VH + (kb - 1), n, C(1.0, 0.0), H + c0, ldh, gs);  // A -= Y V^H
            blk_gemm(kb, nc, m, C(1.0, 0.0), VH, n, H + (size_t)(k + 1) * ldh + c0, ldh, C(0.0, 0.0), Wt, n, gs);
            for (int c = tid; c < nc; c += nt) {  // Wt <- T^H Wt, rows from the bottom up
                for (int l = kb - 1; l >= 0; --l) {
                    cplx s = C(0.0, 0.0);
                    for (int p = 0; p <= l; ++p) s = cfma(cconj(Tm[p * NB + l]), Wt[(size_t)p * n + c], s);
                    Wt[(size_t)l * n + c] = s;
                }
            }
            blk_gemm(m, nc, kb, C(-1.0, 0.0), V, NB, Wt, n, C(1.0, 0.0), H + (size_t)(k + 1) * ldh + c0, ldh, gs);
        }
        // Z[:, k+1:] <- Z[:, k+1:] - (Z V T) V^H
        blk_gemm(n, kb, m, C(1.0, 0.0), Z + k + 1, ldz, V, NB, C(0.0, 0.0), P, NB, gs);
        for (int r = tid; r < n; r += nt) {  // P <- P T, columns from the right
            for (int l = kb - 1; l >= 0; --l) {
                cplx s = C(0.0, 0.0);
                for (int p = 0; p <= l; ++p) s = cfma(P[(size_t)r * NB + p], Tm[p * NB + l], s);
                P[(size_t)r * NB + l] = s;
            }
        }
        blk_gemm(n, m, kb, C(-1.0, 0.0), P, NB, VH, n, C(1.0, 0.0), Z + k + 1, ldz, gs);
        if (prof && tid == 0) prof[2] += clock64() - tg0;
    }
}

// ---- complex Schur by shifted QR ------------------------------------------------------
// Givens G = [[c, s], [-conj(s), c]] with G [a; b] = [r; 0], c real.
// c = |a| / r, s = a conj(b) / (|a| r), r = sqrt(|a|^2 + |b|^2), formed with
// two reciprocal square roots (entries here are far from over/underflow).
__device__ __forceinline__ void givens(cplx a, cplx b, double& c, cplx& s) {
    const double na = cnorm2(a), nb = cnorm2(b);
    if (nb == 0.0) {
        c = 1.0;
        s = C(0.0, 0.0);
        return;
    }
    if (na == 0.0) {
        c = 0.0;
        s = cscale(cconj(b), rsqrt(nb));
        return;
    }
    const double ia = rsqrt(na), ir = rsqrt(na + nb);
    c = na * ia * ir;
    s = cscale(cmul(a, cconj(b)), ia * ir);
}

// eigenvalue of [[a, b], [c, d]] closest to d
__device__ __forceinline__ cplx wilkinson(cplx a, cplx b, cplx c, cplx d) {
    const cplx half = cscale(csub(a, d), 0.5);
    const cplx disc = csqrt_p(cfma(half, half, cmul(b, c)));
    const cplx mid = cscale(cadd(a, d), 0.5);
    const cplx e1 = cadd(mid, disc), e2 = csub(mid, disc);
    return cabs1(csub(e1, d)) <= cabs1(csub(e2, d)) ? e1 : e2;
}

constexpr int kMaxN = 2048;  // largest matrix order (deflation flags are per row; 2N <= 1922 for M <= 15)

// ---- eigenvectors of the triangular Schur factor ----------------------------------------
// X (n x n, row-major) <- right eigenvectors of upper-triangular T: column k
// solves (T - t_kk I) x = 0 with x_k = 1, x_i = 0 for i > k (ztrevc's back
// substitution, with tiny denominators replaced by smin = max(eps |t_kk|, tiny)).
// Rows are solved bottom-up in blocks of TB: the coupling of a block to the rows
// below it, S = T[block, below] X[below, below], is one GEMM (tensor cores);
// inside the block one thread per column k finishes the substitution with its
// own shift t_kk. Columns are then scaled to unit max |re|+|im|.
// S: scratch of TB x n complex (global).
constexpr int TB = 64;
__device__ void blk_trevc(int n, const cplx* T, int ldt, cplx* X, int ldx, cplx* S, GemmSmem* gs) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const double eps = 2.220446049250313e-16;
    const double tiny = 2.2250738585072014e-308 / eps;
    for (int e = tid; e < n * n; e += nt) {
        const int i = e / n, k = e % n;
        X[(size_t)i * ldx + k] = C(i == k ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int r0 = ((n - 1) / TB) * TB; r0 >= 0; r0 -= TB) {
        const int r1 = min(n, r0 + TB);
        const bool below = r1 < n;
        // S[i - r0][k - r1] = sum_{j >= r1} T[i][j] X[j][k]   (k >= r1; zero for k < r1)
        if (below)
            blk_gemm(r1 - r0, n - r1, n - r1, C(1.0, 0.0), T + (size_t)r0 * ldt + r1, ldt, X + (size_t)r1 * ldx + r1,
                     ldx, C(0.0, 0.0), S, n, gs);
        for (int k = r0 + 1 + tid; k < n; k += nt) {
            const cplx lam = T[(size_t)k * ldt + k];
            const double smin = fmax(eps * cabs1(lam), tiny);
            const int jmax = min(r1 - 1, k);
            for (int i = min(r1, k) - 1; i >= r0; --i) {
                cplx acc = (below && k >= r1) ? S[(size_t)(i - r0) * n + (k - r1)] : C(0.0, 0.0);
                for (int j = i + 1; j <= jmax; ++j) acc = cfma(T[(size_t)i * ldt + j], X[(size_t)j * ldx + k], acc);
                cplx den = csub(T[(size_t)i * ldt + i], lam);
                if (cabs1(den) < smin) den = C(smin, 0.0);
                X[(size_t)i * ldx + k] = cneg(cdiv(acc, den));
            }
        }
        __syncthreads();
    }
    for (int k = tid; k < n; k += nt) {
        double xmax = 0.0;
        for (int j = 0; j <= k; ++j) xmax = fmax(xmax, cabs1(X[(size_t)j * ldx + k]));
        const double sc = 1.0 / xmax;
        for (int j = 0; j <= k; ++j) X[(size_t)j * ldx + k] = cscale(X[(size_t)j * ldx + k], sc);
    }
    __syncthreads();
}

}  // namespace cb
