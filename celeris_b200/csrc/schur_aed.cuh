// Complex Schur decomposition for large n (one CTA per cell): small-bulge
// multishift QR with aggressive early deflation (AED), the scheme of LAPACK's
// xLAQR0/xLAQR3/xLAQR5 restated for one thread block:
//
//  * AED: the trailing NW x NW window of the active block is brought to Schur
//    form in shared memory (one warp, single-shift QR, unitary U accumulated).
//    Eigenvalues whose spike entry s * conj(U[0][j]) is negligible deflate;
//    the others are moved to the top of the window by adjacent swaps, the spike
//    is reflected back to a multiple of e1 and the undeflated part is reduced
//    to Hessenberg form again. The undeflated eigenvalues become the shifts.
//  * Sweep: up to NSH single-shift bulges are chased down the active block as
//    a chain (bulges two rows apart, all moved one row per step: first every
//    row rotation, then every column rotation, one warp per bulge). The chain
//    advances through windows of at most WMAX rows/columns held in shared
//    memory; each window's rotations are accumulated into one unitary U.
//  * Every window (AED, sweep or a whole small block) reaches the rest of the
//    matrix once, as dense products with U (rows right of the window,
//    columns above it, and Z), tiled through shared memory.
//
// The rows and columns outside the window are therefore read and written once
// per window instead of once per rotation block of a single-shift sweep; the
// work moves from memory-bound rotations to compute-bound small products.
#pragma once

#include "cblas_block.cuh"

namespace cb {

// WMAX = 56 keeps the shared block near 104 KB, so two cells share an SM and
// one cell's latency-bound phases (AED, rotation steps) overlap the other's
// products; with 16 shifts a window still advances the chain by 23 rows.
constexpr int WMAX = 56;     // window size (rows/columns)
constexpr int NSH = 16;      // shifts per sweep
constexpr int NWIN = 24;     // AED window
constexpr int NSMALL = WMAX; // active blocks up to this size are finished in shared memory
constexpr int FT = 24;       // far-update tile (rows or columns), a multiple of the 8-wide DMMA tile
// Threads of the Schur kernel: two CTAs of 256 threads and <= 128 registers
// share an SM; WMAX / 8 = 7 warps carry the far-update products.
constexpr int kSchurThreads = 256;

struct AedShared {
    cplx B[WMAX][WMAX + 1];  // window; during far updates two tile buffers of WMAX * FT
    cplx U[WMAX][WMAX + 1];  // accumulated unitary of the window (+1: column walks spread over the banks)
    cplx sh[NWIN];           // undeflated eigenvalues of the last AED
    cplx vec[WMAX];          // Householder vector
    double rc[NSH];          // rotations of one chain step, per bulge
    cplx rs[NSH];
    int pos[NSH];            // bulge positions (-2 not introduced, -1 gone)
    unsigned char flag[kMaxN];
    int lo, hi, done, info, nsweep, nsu, nd, nshift, nxt, win_end, ws, we, it;
    cplx shift[NSH];
    unsigned umask[WMAX / 8];  // bit q of umask[c]: block U[4q..4q+3][8c..8c+7] has a non-zero
    double qc[WMAX];           // rotations of one small-QR sweep (deferred column rotations)
    cplx qs[WMAX];
};

// ---- warp-level helpers on shared matrices ------------------------------------------------
// rows r, r+1 over columns [c0, c1): G = [[c, s], [-conj s, c]] from the left
__device__ __forceinline__ void wrot_rows(cplx* B, int ld, int r, double c, cplx s, int c0, int c1, int lane) {
    const cplx ms = cneg(cconj(s));
    for (int col = c0 + lane; col < c1; col += 32) {
        const cplx x = B[r * ld + col], y = B[(r + 1) * ld + col];
        B[r * ld + col] = cfma(s, y, cscale(x, c));
        B[(r + 1) * ld + col] = cfma(ms, x, cscale(y, c));
    }
}
// columns k, k+1 over rows [r0, r1): M <- M G^H
__device__ __forceinline__ void wrot_cols(cplx* B, int ld, int k, double c, cplx s, int r0, int r1, int lane) {
    const cplx cs = cconj(s), ns = cneg(s);
    for (int row = r0 + lane; row < r1; row += 32) {
        const cplx x = B[row * ld + k], y = B[row * ld + k + 1];
        B[row * ld + k] = cfma(cs, y, cscale(x, c));
        B[row * ld + k + 1] = cfma(ns, x, cscale(y, c));
    }
}

// The same rotations by a group of `nl` lanes (lane index l in the group).
__device__ __forceinline__ void grot_rows(cplx* B, int ld, int r, double c, cplx s, int c0, int c1, int l, int nl) {
    const cplx ms = cneg(cconj(s));
    for (int col = c0 + l; col < c1; col += nl) {
        const cplx x = B[r * ld + col], y = B[(r + 1) * ld + col];
        B[r * ld + col] = cfma(s, y, cscale(x, c));
        B[(r + 1) * ld + col] = cfma(ms, x, cscale(y, c));
    }
}
__device__ __forceinline__ void grot_cols(cplx* B, int ld, int k, double c, cplx s, int r0, int r1, int l, int nl) {
    const cplx cs = cconj(s), ns = cneg(s);
    for (int row = r0 + l; row < r1; row += nl) {
        const cplx x = B[row * ld + k], y = B[row * ld + k + 1];
        B[row * ld + k] = cfma(cs, y, cscale(x, c));
        B[row * ld + k + 1] = cfma(ns, x, cscale(y, c));
    }
}

// Single-shift QR of a Hessenberg block B (m x m, m <= 64, shared) with the
// rotations accumulated into U (mu x m, mu <= 64). The bulge chase of a sweep
// (rotations k = l .. hi-1) needs only the band around the diagonal: rotation
// k + 1 is a function of the 2 x 2 block at k, the subdiagonal below it and
// the bulge, so warp 0 keeps that band in registers (the same values in every
// lane) and derives each rotation without a shared-memory round trip. Its
// lanes also carry the columns right of the band (lane j % 32): row rotation
// k mixes the running B[k][j] (a register) with the untouched B[k+1][j],
// stores the final B[k][j], and column k + 2 enters the band by a shuffle of
// its running value. Nothing in the chase reads the rows above the band or
// U, so their column rotations are deferred: warp 0 records the sweep's
// rotations, and then every thread carries one row of B (from the rotation
// after it left the band) or of U through all of them. Each element sees the
// same rotations, in the same order and with the same arithmetic, as the plain
// sweep (rows k, k+1 over columns >= k-1, then columns k, k+1 over rows <= k+2).
__device__ __forceinline__ void rot_rows2(cplx x, cplx y, double c, cplx s, cplx ms, cplx& xo, cplx& yo) {
    xo = cfma(s, y, cscale(x, c));
    yo = cfma(ms, x, cscale(y, c));
}
__device__ __forceinline__ void rot_cols2(cplx x, cplx y, double c, cplx cs, cplx ns, cplx& xo, cplx& yo) {
    xo = cfma(cs, y, cscale(x, c));
    yo = cfma(ns, x, cscale(y, c));
}
// givens() without branches (the same c, s in every case), so that the chase
// step below stays one block the compiler can schedule as a whole.
__device__ __forceinline__ void givens_sel(cplx a, cplx b, double& c, cplx& s) {
    const double na = cnorm2(a), nb = cnorm2(b);
    const double ia = rsqrt(na), ir = rsqrt(na + nb);
    const cplx sg = cscale(cmul(a, cconj(b)), ia * ir), s0 = cscale(cconj(b), ir);
    c = nb == 0.0 ? 1.0 : (na == 0.0 ? 0.0 : na * ia * ir);
    s = nb == 0.0 ? C(0.0, 0.0) : (na == 0.0 ? s0 : sg);
}
// The chase of one sweep by warp 0 (NS: column slots per lane, m <= 32 NS).
// Records rotation k in qc/qs[k - l]; leaves B[k][k+1] holding row k's value
// after column rotation k (the start of its deferred chain).
template <int NS>
__device__ void qr_chase(int m, cplx* B, int ld, int l, int hi, cplx shift, double* qc, cplx* qs, int lane) {
    const cplx Z0 = C(0.0, 0.0);
    cplx P = B[l * ld + l], Q = B[l * ld + l + 1], R = B[(l + 1) * ld + l], S = B[(l + 1) * ld + l + 1];
    cplx T = (l + 2 <= hi) ? B[(l + 2) * ld + l + 1] : Z0;
    cplx a = csub(P, shift), bb = R;
    cplx cc[NS];  // running values of columns lane + 32 t right of the band
    int ci[NS];   // those columns, clamped into the matrix for the loads
#pragma unroll
    for (int t = 0; t < NS; ++t) {
        const int i = lane + 32 * t;
        ci[t] = min(i, m - 1);
        cc[t] = (i >= l + 2 && i < m) ? B[l * ld + i] : Z0;
    }
    for (int k = l; k < hi; ++k) {
        // loads first: row k+1 right of the band and the next band entries
        // are untouched by this sweep so far
        cplx yr[NS];
#pragma unroll
        for (int t = 0; t < NS; ++t) yr[t] = B[(k + 1) * ld + ci[t]];
        const int j2 = min(k + 2, m - 1), j3 = min(k + 3, m - 1);
        const cplx Sn = B[j2 * ld + j2], Tn = B[j3 * ld + j2];
        double c;
        cplx s;
        givens_sel(a, bb, c, s);
        const cplx ms = cneg(cconj(s)), cs = cconj(s), ns = cneg(s);
        const cplx rn = cfma(s, bb, cscale(a, c));  // B[k][k-1] after the row rotation (k > l)
        cplx xr[NS];
#pragma unroll
        for (int t = 0; t < NS; ++t) {
            cplx yo;
            rot_rows2(cc[t], yr[t], c, s, ms, xr[t], yo);
            if (lane + 32 * t >= k + 2) cc[t] = yo;
        }
        // the band: rows k, k+1 then columns k, k+1 (row k+2 gains the bulge)
        cplx P1, Q1, R1, S1, P2, Q2, R2, S2, bul, Rn;
        rot_rows2(P, R, c, s, ms, P1, R1);
        rot_rows2(Q, S, c, s, ms, Q1, S1);
        rot_cols2(P1, Q1, c, cs, ns, P2, Q2);
        rot_cols2(R1, S1, c, cs, ns, R2, S2);
        rot_cols2(Z0, T, c, cs, ns, bul, Rn);  // T = 0 past the active block
        // column k+2 enters the band (its running value after row rotation k)
        const int j = k + 2;
        const cplx v = (NS == 1 || j < 32) ? cc[0] : cc[NS - 1];
        const cplx Qn = C(__shfl_sync(0xffffffffu, v.x, j & 31), __shfl_sync(0xffffffffu, v.y, j & 31));
#pragma unroll
        for (int t = 0; t < NS; ++t) {
            const int i = lane + 32 * t;
            if (i >= k + 2 && i < m) B[k * ld + i] = xr[t];
        }
        if (lane == 0) {
            qc[k - l] = c;
            qs[k - l] = s;
            if (k > l) {
                B[k * ld + k - 1] = rn;
                B[(k + 1) * ld + k - 1] = Z0;
            }
            B[k * ld + k] = P2;
            B[k * ld + k + 1] = Q2;
            if (k + 1 == hi) {
                B[(k + 1) * ld + k] = R2;
                B[(k + 1) * ld + k + 1] = S2;
            }
        }
        a = R2;
        bb = bul;
        P = S2;
        Q = Qn;
        R = Rn;
        S = Sn;
        T = (k + 3 <= hi) ? Tn : Z0;
        __syncwarp();
    }
#pragma unroll
    for (int t = 0; t < NS; ++t) {
        const int i = lane + 32 * t;
        if (i >= hi + 1 && i < m) B[hi * ld + i] = cc[t];
    }
}

// Single-shift QR of the m x m upper Hessenberg matrix B (shared, ld) to upper
// triangular form, U <- U Q (rows [0, mu)). Called by every thread of the
// block; warp 0 chases, all threads apply the deferred column rotations.
// Returns 0, or the (1-based) row where the iteration cap ran out (the same
// value in every thread).
// tprof (optional): clock64 sums of [0] the chases (warp 0) and [1] the
// deferred rotations (thread 0).
__device__ __noinline__ int blk_schur_small(int m, cplx* B, int ld, cplx* U, int ldu, int mu, AedShared* sh,
                               long long* nrot = nullptr, int iter_cap = 0, long long* tprof = nullptr) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const double eps = 2.220446049250313e-16;
    const double smallnum = 2.2250738585072014e-308 * (m / eps);
    int hi = m - 1, it = 0, total = 0;
    long long rot_count = 0;  // written to *nrot once: a global update per sweep stalls the chase
    const int max_total = iter_cap > 0 ? min(iter_cap, 30 * m) : 30 * m;
    while (hi > 0) {
        // l = largest index in [1, hi] with a negligible subdiagonal (0 if
        // none); every warp reads the same B and finds the same l
        int l = 0;
        for (int base = hi; base >= 1 && l == 0; base -= 32) {
            const int i = base - lane;
            bool f = false;
            if (i >= 1) {
                const double tst = cabs1(B[(i - 1) * ld + i - 1]) + cabs1(B[i * ld + i]);
                f = cabs1(B[i * ld + i - 1]) <= fmax(eps * tst, smallnum);
            }
            const unsigned msk = __ballot_sync(0xffffffffu, f);
            if (msk) l = base - (__ffs(msk) - 1);
        }
        cplx shift = C(0.0, 0.0);
        const bool deflated = l == hi;
        if (!deflated) {
            if (it + 1 == 10 || it + 1 == 20) {
                shift = cadd(B[hi * ld + hi],
                             C(0.75 * fabs(B[hi * ld + hi - 1].x) + fabs(B[hi * ld + hi - 1].y), 0.0));
            } else {
                shift = wilkinson(B[(hi - 1) * ld + hi - 1], B[(hi - 1) * ld + hi], B[hi * ld + hi - 1],
                                  B[hi * ld + hi]);
            }
        }
        __syncthreads();  // every read of this step's deflation test and shift is done
        if (l > 0 && tid == 0) B[l * ld + l - 1] = C(0.0, 0.0);
        if (deflated) {
            --hi;
            it = 0;
            __syncthreads();
            continue;
        }
        if (++total > max_total) {
            if (nrot && tid == 0) *nrot += rot_count;
            return hi + 1;
        }
        ++it;
        rot_count += hi - l;
        if (warp == 0) {
            const long long tc0 = clock64();
            if (m <= 32)
                qr_chase<1>(m, B, ld, l, hi, shift, sh->qc, sh->qs, lane);
            else
                qr_chase<2>(m, B, ld, l, hi, shift, sh->qc, sh->qs, lane);
            if (tprof && lane == 0) tprof[0] += clock64() - tc0;
        }
        __syncthreads();
        const long long td0 = clock64();
        // deferred column rotations: row r of B from the rotation after it
        // left the band (rows above the block from l), every row of U from l
        for (int q = tid; q < hi + mu; q += nt) {
            const bool isu = q >= hi;
            const int r = isu ? q - hi : q;
            cplx* row = isu ? U + r * ldu : B + r * ld;
            const int k0 = isu ? l : max(l, r + 1);
            cplx carry = row[k0];
            for (int k = k0; k < hi; ++k) {
                const double c = sh->qc[k - l];
                const cplx s = sh->qs[k - l];
                cplx xo, yo;
                rot_cols2(carry, row[k + 1], c, cconj(s), cneg(s), xo, yo);
                row[k] = xo;
                carry = yo;
            }
            row[hi] = carry;
        }
        __syncthreads();
        if (tprof && tid == 0) tprof[1] += clock64() - td0;
    }
    if (nrot && tid == 0) *nrot += rot_count;
    return 0;
}

// Householder reflector from x (length len, shared) : returns beta (0 when x is
// already a multiple of e1) and leaves v in x (v0 = x0 - alpha), alpha out.
// P = I - beta v v^H is Hermitian and unitary with P x = alpha e1. One warp.
__device__ double warp_reflector(cplx* x, int len, cplx& alpha, int lane) {
    double s2 = 0.0;
    for (int i = lane; i < len; i += 32) s2 += cnorm2(x[i]);
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    const cplx x0 = x[0];
    const double tail = s2 - cnorm2(x0);
    __syncwarp();
    if (!(tail > 0.0)) {
        alpha = x0;
        return 0.0;
    }
    const double xn = sqrt(s2), ax0 = cabs(x0);
    const cplx ph = ax0 > 0.0 ? cscale(x0, 1.0 / ax0) : C(1.0, 0.0);
    alpha = cscale(ph, -xn);
    const cplx v0 = csub(x0, alpha);
    if (lane == 0) x[0] = v0;
    __syncwarp();
    return 2.0 / (tail + cnorm2(v0));
}

// M[r0:r0+len, c0:c1] <- P M (P = I - beta v v^H), lanes over columns
__device__ __forceinline__ void wrefl_left(cplx* M, int ld, int r0, int len, int c0, int c1, const cplx* v,
                                           double beta, int lane) {
    for (int col = c0 + lane; col < c1; col += 32) {
        cplx w = C(0.0, 0.0);
        for (int i = 0; i < len; ++i) w = cfma(cconj(v[i]), M[(r0 + i) * ld + col], w);
        w = cscale(w, beta);
        for (int i = 0; i < len; ++i) M[(r0 + i) * ld + col] = cfms(v[i], w, M[(r0 + i) * ld + col]);
    }
}
// M[r0:r1, c0:c0+len] <- M P, lanes over rows
__device__ __forceinline__ void wrefl_right(cplx* M, int ld, int r0, int r1, int c0, int len, const cplx* v,
                                            double beta, int lane) {
    for (int row = r0 + lane; row < r1; row += 32) {
        cplx w = C(0.0, 0.0);
        for (int i = 0; i < len; ++i) w = cfma(M[row * ld + c0 + i], v[i], w);
        w = cscale(w, beta);
        for (int i = 0; i < len; ++i) M[row * ld + c0 + i] = cfms(w, cconj(v[i]), M[row * ld + c0 + i]);
    }
}

// ---- far updates: the window's unitary applied to the rest of the matrix ------------------
// Tiles of FT rows or columns stream through two shared buffers with cp.async
// (16-byte copies, zero-filled past the edge): the next tile is in flight
// while the current one is multiplied. The buffers overlay the window B, which
// is dead during the far updates.
constexpr int FBUF = WMAX * FT;  // complex entries per tile buffer

// X[r0:r0+w, c0:c1] <- U^H X  (U w x w in shared memory). Tile t holds columns
// c0 + t*FT .. as [w][FT] (k-major: a warp reads 8 consecutive entries).
__device__ void far_left(cplx* X, int ld, int r0, int w, int c0, int c1, const cplx (*U)[WMAX + 1], cplx* buf,
                         const unsigned* umask) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int ntile = (c1 - c0 + FT - 1) / FT;
    auto issue = [&](int t) {
        const int cb = c0 + t * FT, nc = min(FT, c1 - cb);
        cplx* dst = buf + (t & 1) * FBUF;
        for (int e = tid; e < w * FT; e += nt) {
            const int k = e / FT, c = e % FT;
            cp_async16(dst + e, X + (size_t)(r0 + k) * ld + cb + (c < nc ? c : 0), c < nc);
        }
        cp_async_commit();
    };
    issue(0);
    for (int t = 0; t < ntile; ++t) {
        if (t + 1 < ntile) {
            issue(t + 1);
            cp_async_wait1();
        } else {
            cp_async_wait0();
        }
        __syncthreads();
        const cplx* tile = buf + (t & 1) * FBUF;
        const int cb = c0 + t * FT, nc = min(FT, c1 - cb);
        // DMMA: warp i < WMAX/8 owns output rows 8i..8i+7 and all FT/8 column
        // tiles; A = U^H (A[g][t] = conj U[k][8i+g]), B = the staged tile
        const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
        if (warp < WMAX / 8 && 8 * warp < w) {
            const int row = 8 * warp + g;
            const unsigned mk = umask[warp];
            double cr[FT / 8][2], ci[FT / 8][2];
#pragma unroll
            for (int j = 0; j < FT / 8; ++j) cr[j][0] = cr[j][1] = ci[j][0] = ci[j][1] = 0.0;
            for (int ks = 0; ks < w; ks += 4) {
                if (!((mk >> (ks >> 2)) & 1u)) continue;  // this 8 x 4 block of U is zero
                const int kk = ks + t4;
                const cplx uv = (kk < w && row < w) ? U[kk][row] : C(0.0, 0.0);
                const double ar = uv.x, ai = -uv.y, nai = uv.y;  // conj(U)
#pragma unroll
                for (int j = 0; j < FT / 8; ++j) {
                    const cplx bv = kk < w ? tile[kk * FT + 8 * j + g] : C(0.0, 0.0);
                    dmma(cr[j][0], cr[j][1], ar, bv.x);
                    dmma(cr[j][0], cr[j][1], nai, bv.y);
                    dmma(ci[j][0], ci[j][1], ar, bv.y);
                    dmma(ci[j][0], ci[j][1], ai, bv.x);
                }
            }
            if (row < w) {
#pragma unroll
                for (int j = 0; j < FT / 8; ++j)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int c = 8 * j + 2 * t4 + h;
                        if (c < nc) X[(size_t)(r0 + row) * ld + cb + c] = C(cr[j][h], ci[j][h]);
                    }
            }
        }
        __syncthreads();
    }
}

// X[r0:r1, c0:c0+w] <- X U. Tile t holds rows r0 + t*FT .. as [FT][w] with
// row stride TS = WMAX + 1: WMAX complex is a multiple of 128 bytes, so without
// the pad the rows a warp reads at once would sit in the same banks.
constexpr int TS = WMAX + 1;
constexpr int FBUF_R = FT * TS;
__device__ void far_right(cplx* X, int ld, int r0, int r1, int c0, int w, const cplx (*U)[WMAX + 1], cplx* buf,
                          const unsigned* umask) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int ntile = (r1 - r0 + FT - 1) / FT;
    auto issue = [&](int t) {
        const int rb = r0 + t * FT, nr = min(FT, r1 - rb);
        cplx* dst = buf + (t & 1) * FBUF_R;
        for (int e = tid; e < FT * w; e += nt) {
            const int r = e / w, k = e % w;
            cp_async16(dst + r * TS + k, X + (size_t)(rb + (r < nr ? r : 0)) * ld + c0 + k, r < nr);
        }
        cp_async_commit();
    };
    issue(0);
    for (int t = 0; t < ntile; ++t) {
        if (t + 1 < ntile) {
            issue(t + 1);
            cp_async_wait1();
        } else {
            cp_async_wait0();
        }
        __syncthreads();
        const cplx* tile = buf + (t & 1) * FBUF_R;
        const int rb = r0 + t * FT, nr = min(FT, r1 - rb);
        // DMMA: warp j < WMAX/8 owns output columns 8j..8j+7 and all FT/8 row
        // tiles; A = the staged rows, B = U
        const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
        if (warp < WMAX / 8 && 8 * warp < w) {
            const int col = 8 * warp + g;
            const unsigned mk = umask[warp];
            double cr[FT / 8][2], ci[FT / 8][2];
#pragma unroll
            for (int i = 0; i < FT / 8; ++i) cr[i][0] = cr[i][1] = ci[i][0] = ci[i][1] = 0.0;
            for (int ks = 0; ks < w; ks += 4) {
                if (!((mk >> (ks >> 2)) & 1u)) continue;  // this 4 x 8 block of U is zero
                const int kk = ks + t4;
                const cplx uv = (kk < w && col < w) ? U[kk][col] : C(0.0, 0.0);
#pragma unroll
                for (int i = 0; i < FT / 8; ++i) {
                    const cplx av = kk < w ? tile[(8 * i + g) * TS + kk] : C(0.0, 0.0);
                    dmma(cr[i][0], cr[i][1], av.x, uv.x);
                    dmma(cr[i][0], cr[i][1], -av.y, uv.y);
                    dmma(ci[i][0], ci[i][1], av.x, uv.y);
                    dmma(ci[i][0], ci[i][1], av.y, uv.x);
                }
            }
#pragma unroll
            for (int i = 0; i < FT / 8; ++i) {
                const int r = 8 * i + g;
                if (r >= nr) continue;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = 8 * warp + 2 * t4 + h;
                    if (c < w) X[(size_t)(rb + r) * ld + c0 + c] = C(cr[i][h], ci[i][h]);
                }
            }
        }
        __syncthreads();
    }
}

// Window [ws, we) of H <- U^H (.) U everywhere outside the window, given that
// the window itself was already transformed in shared memory: rows ws..we-1 to
// the right (columns we..n-1), columns ws..we-1 above (rows 0..ws-1), and Z.
// The tile buffers overlay B: the window must be stored before the call.
// The window unitary of a sweep is banded (a chain of adjacent-column rotations
// that moves down the window): a bitmap of its non-zero 4 x 8 blocks lets the
// products skip the zero ones (rotations keep structural zeros exactly zero).
// banded: the window comes from a sweep (AED and small-block windows are dense).
__device__ void far_all(int n, cplx* H, int ldh, cplx* Z, int ldz, int ws, int we, AedShared* sh,
                        bool banded = false) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int w = we - ws;
    cplx* buf = &sh->B[0][0];
    if (tid < WMAX / 8) sh->umask[tid] = banded ? 0u : ~0u;
    __syncthreads();
    const int nkq = (w + 3) / 4, njc = (w + 7) / 8;
    for (int e = tid; banded && e < nkq * njc; e += nt) {
        const int kq = e / njc, jc = e % njc;
        bool nz = false;
        for (int r = 4 * kq; r < min(4 * kq + 4, w); ++r)
            for (int c = 8 * jc; c < min(8 * jc + 8, w); ++c) {
                const cplx u = sh->U[r][c];
                nz = nz || u.x != 0.0 || u.y != 0.0;
            }
        if (nz) atomicOr(&sh->umask[jc], 1u << kq);
    }
    __syncthreads();
    if (we < n) far_left(H, ldh, ws, w, we, n, sh->U, buf, sh->umask);
    if (ws > 0) far_right(H, ldh, 0, ws, ws, w, sh->U, buf, sh->umask);
    far_right(Z, ldz, 0, n, ws, w, sh->U, buf, sh->umask);
}

__device__ void load_window(const cplx* H, int ldh, int ws, int w, AedShared* sh) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < w * w; e += nt) {
        const int r = e / w, c = e % w;
        sh->B[r][c] = H[(size_t)(ws + r) * ldh + ws + c];
        sh->U[r][c] = C(r == c ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
}

// mask: write exact zeros below the subdiagonal (a finished Hessenberg or
// triangular window); a sweep window is stored as it is (it holds bulges).
__device__ void store_window(cplx* H, int ldh, int ws, int w, const AedShared* sh, bool mask) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < w * w; e += nt) {
        const int r = e / w, c = e % w;
        H[(size_t)(ws + r) * ldh + ws + c] = (mask && r > c + 1) ? C(0.0, 0.0) : sh->B[r][c];
    }
}

// ---- aggressive early deflation ---------------------------------------------------------------
// Window [kwtop, hi] of the active block [lo, hi]. Sets sh->nd (deflated count)
// and sh->nsu / sh->sh[0..nsu) (undeflated eigenvalues, the shifts).
__device__ void aed(int n, cplx* H, int ldh, cplx* Z, int ldz, int lo, int hi, AedShared* sh, long long* prof) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long t0 = clock64();
    const double eps = 2.220446049250313e-16;
    const double smallnum = 2.2250738585072014e-308 * (n / eps);
    const int kwtop = max(lo, hi - NWIN + 1), jw = hi - kwtop + 1;
    const cplx s = kwtop > lo ? H[(size_t)kwtop * ldh + kwtop - 1] : C(0.0, 0.0);
    load_window(H, ldh, kwtop, jw, sh);
    cplx* B = &sh->B[0][0];
    cplx* U = &sh->U[0][0];
    constexpr int ldb = WMAX + 1, ldu = WMAX + 1;
    const long long ts0 = clock64();
    const int info = blk_schur_small(jw, B, ldb, U, ldu, jw, sh, prof ? prof + 8 : nullptr, 0,
                                     prof ? prof + 12 : nullptr);
    if (warp == 0) {
        if (prof && lane == 0) prof[5] += clock64() - ts0;
        int nsu = jw, ilst = 0;
        if (info == 0) {
            while (nsu > ilst) {
                double foo = cabs1(B[(nsu - 1) * ldb + nsu - 1]);
                if (foo == 0.0) foo = cabs1(s);
                if (cabs1(s) * cabs1(U[nsu - 1]) <= fmax(smallnum, eps * foo)) {
                    --nsu;  // deflatable: stays at the bottom
                } else {
                    for (int k = nsu - 2; k >= ilst; --k) {  // move it up to ilst
                        double c;
                        cplx sn;
                        givens(B[k * ldb + k + 1], csub(B[(k + 1) * ldb + k + 1], B[k * ldb + k]), c, sn);
                        __syncwarp();
                        wrot_rows(B, ldb, k, c, sn, k, jw, lane);
                        __syncwarp();
                        wrot_cols(B, ldb, k, c, sn, 0, k + 2, lane);
                        wrot_cols(U, ldu, k, c, sn, 0, jw, lane);
                        __syncwarp();
                        if (lane == 0) B[(k + 1) * ldb + k] = C(0.0, 0.0);
                        __syncwarp();
                    }
                    ++ilst;
                }
                __syncwarp();
            }
        }
        for (int i = lane; i < nsu; i += 32) sh->sh[i] = B[i * ldb + i];
        if (lane == 0) {
            sh->nsu = nsu;
            sh->nd = jw - nsu;
        }
        __syncwarp();
        if (s.x != 0.0 || s.y != 0.0) {
            if (nsu > 0) {
                // spike w = s conj(U[0, :nsu]) -> alpha e1
                for (int i = lane; i < nsu; i += 32) sh->vec[i] = cmul(s, cconj(U[i]));
                __syncwarp();
                cplx alpha;
                const double beta = warp_reflector(sh->vec, nsu, alpha, lane);
                if (beta != 0.0) {
                    wrefl_left(B, ldb, 0, nsu, 0, jw, sh->vec, beta, lane);
                    __syncwarp();
                    wrefl_right(B, ldb, 0, nsu, 0, nsu, sh->vec, beta, lane);
                    wrefl_right(U, ldu, 0, jw, 0, nsu, sh->vec, beta, lane);
                    __syncwarp();
                }
                // back to Hessenberg: columns 0 .. nsu-3 of the undeflated block
                for (int j = 0; j + 2 < nsu; ++j) {
                    const int len = nsu - j - 1;
                    for (int i = lane; i < len; i += 32) sh->vec[i] = B[(j + 1 + i) * ldb + j];
                    __syncwarp();
                    cplx al;
                    const double bt = warp_reflector(sh->vec, len, al, lane);
                    if (bt != 0.0) {
                        wrefl_left(B, ldb, j + 1, len, j + 1, jw, sh->vec, bt, lane);
                        __syncwarp();
                        for (int i = lane; i < len; i += 32) B[(j + 1 + i) * ldb + j] = i == 0 ? al : C(0.0, 0.0);
                        wrefl_right(B, ldb, 0, nsu, j + 1, len, sh->vec, bt, lane);
                        wrefl_right(U, ldu, 0, jw, j + 1, len, sh->vec, bt, lane);
                    }
                    __syncwarp();
                }
            }
        }
    }
    __syncthreads();
    const long long t1 = clock64();
    const int nsu = sh->nsu;
    store_window(H, ldh, kwtop, jw, sh, true);
    if (kwtop > lo) {
        for (int i = tid; i < jw; i += blockDim.x)
            H[(size_t)(kwtop + i) * ldh + kwtop - 1] = (i == 0 && nsu > 0) ? cmul(s, cconj(sh->U[0][0])) : C(0.0, 0.0);
    }
    far_all(n, H, ldh, Z, ldz, kwtop, hi + 1, sh);
    if (prof && tid == 0) {
        prof[0] += t1 - t0;
        prof[1] += clock64() - t1;
    }
}

// ---- one multishift sweep over the active block [lo, hi] with nsh shifts ----------------------
// All bulges move in lockstep, so the moves of every step follow from the
// positions at the start of a window: in the first window (ws = lo) bulge b is
// introduced at step 2b and sits at lo + t - 2b before step t > 2b; later
// windows introduce nothing and bulge b sits at pos[b] + t until it leaves the
// block (its last move starts at hi - 1). A window runs while the leading
// bulge's move stays inside it (its rows reach p + 2 <= we - 1), or, in the
// window that ends at hi, until every bulge has left.
static_assert(WMAX - 2 > 2 * (NSH - 1), "the first window introduces every bulge");
static_assert(2 * WMAX * FT <= WMAX * (WMAX + 1) && 2 * FBUF_R <= WMAX * (WMAX + 1),
              "tile buffers overlay the window");
static_assert(WMAX % 8 == 0 && FT % 8 == 0 && WMAX / 8 <= kSchurThreads / 32 && WMAX / 4 <= 32,
              "far-update DMMA tiles and block bitmap");

__device__ void chain_sweep(int n, cplx* H, int ldh, cplx* Z, int ldz, int lo, int hi, int nsh, AedShared* sh,
                            long long* prof) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    constexpr int ldb = WMAX + 1, ldu = WMAX + 1;
    cplx* B = &sh->B[0][0];
    cplx* U = &sh->U[0][0];
    if (tid == 0) {
        for (int b = 0; b < nsh; ++b) sh->pos[b] = -2;
        sh->nxt = 0;
        sh->ws = lo;
        sh->we = min(lo + WMAX, hi + 1);
    }
    __syncthreads();
    for (int guard = 0; guard < n / 4 + 32; ++guard) {  // a sweep takes about n / 30 windows
        const int ws = sh->ws, we = sh->we, w = we - ws;
        const bool first = sh->nxt == 0;
        int S;
        if (first) {
            S = we - 2 - lo;  // we < hi + 1 here: the block is longer than a window
        } else {
            int plead = -1, plast = 1 << 30;
            for (int b = 0; b < nsh; ++b) {
                const int p = sh->pos[b];
                if (p >= 0) {
                    plead = max(plead, p);
                    plast = min(plast, p);
                }
            }
            S = (we == hi + 1) ? hi - plast : we - 2 - plead;
        }
        const long long t0 = clock64();
        load_window(H, ldh, ws, w, sh);
        // Each warp carries bulges b and b + nwarp, one per half-warp, so their
        // rotations run side by side (bulges 2 rows apart touch disjoint rows in
        // phase 1 and disjoint columns in phase 2).
        const int hl = lane & 15;
        for (int t = 0; t < S; ++t) {
            // phase 1: row rotations
            for (int b0 = warp; b0 < nsh; b0 += 2 * nwarp) {
                const int b = b0 + (lane >> 4) * nwarp;
                int p = 0;
                bool intro = false, act = b < nsh;
                if (act) {
                    if (first) {
                        act = t >= 2 * b;
                        intro = t == 2 * b;
                        p = intro ? lo : lo + t - 2 * b;
                    } else {
                        const int p0 = sh->pos[b];
                        p = p0 + t;
                        act = p0 >= 0 && p <= hi - 1;
                    }
                }
                const int k = p - ws;
                double c = 1.0;
                cplx s = C(0.0, 0.0);
                if (act) {
                    cplx a, bb;
                    if (intro) {
                        a = csub(B[k * ldb + k], sh->shift[b]);
                        bb = B[(k + 1) * ldb + k];
                    } else {
                        a = B[k * ldb + k - 1];
                        bb = B[(k + 1) * ldb + k - 1];
                    }
                    givens(a, bb, c, s);
                }
                __syncwarp();
                if (act) grot_rows(B, ldb, k, c, s, intro ? k : k - 1, w, hl, 16);
                __syncwarp();
                if (act && hl == 0) {
                    if (!intro) B[(k + 1) * ldb + k - 1] = C(0.0, 0.0);
                    sh->rc[b] = c;
                    sh->rs[b] = s;
                }
            }
            __syncthreads();
            // phase 2: column rotations
            for (int b0 = warp; b0 < nsh; b0 += 2 * nwarp) {
                const int b = b0 + (lane >> 4) * nwarp;
                int p = 0;
                bool act = b < nsh;
                if (act) {
                    if (first) {
                        act = t >= 2 * b;
                        p = t == 2 * b ? lo : lo + t - 2 * b;
                    } else {
                        const int p0 = sh->pos[b];
                        p = p0 + t;
                        act = p0 >= 0 && p <= hi - 1;
                    }
                }
                if (act) {
                    const int k = p - ws;
                    const double c = sh->rc[b];
                    const cplx s = sh->rs[b];
                    grot_cols(B, ldb, k, c, s, 0, min(p + 2, hi) - ws + 1, hl, 16);
                    grot_cols(U, ldu, k, c, s, 0, w, hl, 16);
                }
            }
            __syncthreads();
        }
        const long long t1 = clock64();
        store_window(H, ldh, ws, w, sh, false);
        far_all(n, H, ldh, Z, ldz, ws, we, sh, true);  // begins and ends with barriers
        if (prof && tid == 0) {
            prof[2] += t1 - t0;
            prof[3] += clock64() - t1;
            prof[7] += S;
        }
        if (tid == 0) {
            int plast = 1 << 30;
            for (int b = 0; b < nsh; ++b) {
                int p;
                if (first) {
                    p = 2 * b < S ? lo + S - 2 * b : -2;
                } else {
                    p = sh->pos[b] >= 0 ? sh->pos[b] + S : -1;
                }
                if (p > hi - 1) p = -1;
                sh->pos[b] = p;
                if (p >= 0) plast = min(plast, p);
            }
            sh->nxt = nsh;
            if (plast == 1 << 30) {
                sh->win_end = 1;
            } else {
                sh->win_end = 0;
                sh->ws = plast - 1;
                sh->we = min(plast - 1 + WMAX, hi + 1);
            }
        }
        __syncthreads();
        if (sh->win_end) break;
    }
}

// prof (optional, per cell): clock64 sums of [AED local, AED far, sweep local,
// sweep far, small blocks, AED QR], [7] chain steps, [8] AED QR rotations,
// [12, 13] the AED window QR's chases and deferred rotations, [14, 15] those of
// the final blocks.
__device__ int blk_schur_aed(int n, cplx* H, int ldh, cplx* Z, int ldz, AedShared* sh, long long* prof,
                             int iter_cap = 0) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const double eps = 2.220446049250313e-16;
    const double smallnum = 2.2250738585072014e-308 * (n / eps);
    if (tid == 0) {
        sh->hi = n - 1;
        sh->lo = 0;
        sh->done = 0;
        sh->info = 0;
        sh->nsweep = 0;
        sh->it = 0;
    }
    __syncthreads();
    // AED + sweep iterations (about n / 4 are typical); iter_cap > 0 lowers the
    // cap (failure-path tests of the non-convergence report)
    const int max_iter = iter_cap > 0 ? min(iter_cap, 2 * n + 100) : 2 * n + 100;
    for (int iter = 0; iter < max_iter; ++iter) {
        const int hi0 = sh->hi;
        for (int i = 1 + tid; i <= hi0; i += nt) {
            const double tst = cabs1(H[(size_t)(i - 1) * ldh + i - 1]) + cabs1(H[(size_t)i * ldh + i]);
            sh->flag[i] = cabs1(H[(size_t)i * ldh + i - 1]) <= fmax(eps * tst, smallnum) ? 1 : 0;
        }
        __syncthreads();
        if (tid == 0) {
            int hi = hi0;
            while (hi > 0 && sh->flag[hi]) {
                H[(size_t)hi * ldh + hi - 1] = C(0.0, 0.0);
                --hi;
                sh->it = 0;
            }
            int lo = hi;
            while (lo > 0 && !sh->flag[lo]) --lo;
            if (lo > 0) H[(size_t)lo * ldh + lo - 1] = C(0.0, 0.0);
            sh->hi = hi;
            sh->lo = lo;
            sh->done = hi <= 0 ? 1 : 0;
        }
        __syncthreads();
        if (sh->done) break;
        const int lo = sh->lo, hi = sh->hi, L = hi - lo + 1;
        if (L <= NSMALL) {
            // the whole block in shared memory
            const long long t0 = clock64();
            load_window(H, ldh, lo, L, sh);
            const int info = blk_schur_small(L, &sh->B[0][0], WMAX + 1, &sh->U[0][0], WMAX + 1, L, sh, nullptr,
                                             iter_cap, prof ? prof + 14 : nullptr);
            if (tid == 0 && info) sh->info = lo + info;
            __syncthreads();
            store_window(H, ldh, lo, L, sh, true);
            far_all(n, H, ldh, Z, ldz, lo, hi + 1, sh);
            if (prof && tid == 0) prof[4] += clock64() - t0;
            if (tid == 0) {
                sh->hi = lo - 1;
                sh->it = 0;
                sh->nsweep += 1;
                if (sh->info) sh->done = 1;
            }
            __syncthreads();
            if (sh->done) break;
            if (sh->hi <= 0) break;
            continue;
        }
        aed(n, H, ldh, Z, ldz, lo, hi, sh, prof);
        if (tid == 0) {
            const int nd = sh->nd;
            sh->hi = hi - nd;
            sh->it = nd > 0 ? 0 : sh->it + 1;
            sh->nsweep += 1;
            // sweep unless AED deflated at least 14% of its window
            int nsh = 0;
            const int L2 = sh->hi - lo + 1;
            if ((nd == 0 || 100 * nd <= 14 * NWIN) && L2 > NSMALL) {
                const int nsu = sh->nsu;
                if (sh->it > 0 && sh->it % 6 == 0) {  // exceptional shifts
                    nsh = NSH;
                    for (int i = 0; i < nsh; ++i) {
                        const int r = sh->hi - i;
                        const cplx sub = H[(size_t)r * ldh + r - 1];
                        sh->shift[i] = cadd(H[(size_t)r * ldh + r], C(0.75 * cabs1(sub), 0.0));
                    }
                } else if (nsu >= 2) {
                    nsh = min(NSH, nsu);
                    for (int i = 0; i < nsh; ++i) sh->shift[i] = sh->sh[i];
                } else {
                    nsh = 2;
                    for (int i = 0; i < nsh; ++i) sh->shift[i] = H[(size_t)(sh->hi - i) * ldh + sh->hi - i];
                }
            }
            sh->nshift = nsh;  // reused as the shift count of the sweep
        }
        __syncthreads();
        const int nsh = sh->nshift;
        if (nsh > 0) chain_sweep(n, H, ldh, Z, ldz, lo, sh->hi, nsh, sh, prof);
        if (iter == max_iter - 1 && tid == 0) sh->info = sh->hi + 1;
        __syncthreads();
    }
    const int info = sh->info;
    __syncthreads();
    return info;
}

}  // namespace cb
