/*
 * ORACLE - test infrastructure only. Never linked into, or called by, the
 * celeris_b200 product path; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it, as the checker.
 *
 * CPU restatement of the reference's FP64 Rayleigh-Sommerfeld loops, returning
 * the complex field E as well as |E|^2:
 *   - rs_field / rs_pixels follow src/celeris/analysis/focal.cpp:223-236
 *     (propagate_pillars CPU loop): fx = cx - W + i*step, fy = cy - W + j*step,
 *     R = sqrt((fx-x)^2 + (fy-y)^2 + z^2), E += t * polar(1/R, k R), same
 *     summation order over pillars, intensity = norm(E).
 *   - rs_zx follows src/celeris/analysis/throughfocus.cpp:105-118.
 *   - rs_adjoint is the conjugate-transpose of rs_field (pixel -> pillar):
 *     out_j = sum_p conj(exp(i k R_pj)/R_pj) v_p, pixels in row-major order.
 * Complex arrays are interleaved (re, im) doubles. Rows (or pillars) are split
 * over pthreads like parallel_rows (focal.cpp:19-29): worker w takes items
 * w, w + W, ...; each output is summed by one thread in a fixed order, so
 * results do not depend on the thread count. ORACLE_THREADS overrides the
 * thread count (default: online cores).
 */
#include <math.h>
#include <pthread.h>
#include <stddef.h>
#include <stdlib.h>
#include <unistd.h>

typedef void (*item_fn)(void* ctx, int item);
typedef struct {
    item_fn fn;
    void* ctx;
    int lo, hi, w, nw;
} job_t;

static void* worker(void* a) {
    job_t* j = (job_t*)a;
    for (int i = j->lo + j->w; i < j->hi; i += j->nw) j->fn(j->ctx, i);
    return NULL;
}

int oracle_threads(void) {
    const char* e = getenv("ORACLE_THREADS");
    if (e && atoi(e) > 0) return atoi(e);
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

static void parallel_items(int lo, int hi, item_fn fn, void* ctx) {
    int nw = oracle_threads();
    if (nw > hi - lo) nw = hi - lo;
    if (nw <= 1) {
        for (int i = lo; i < hi; ++i) fn(ctx, i);
        return;
    }
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nw);
    job_t* jb = (job_t*)malloc(sizeof(job_t) * nw);
    for (int w = 0; w < nw; ++w) {
        jb[w].fn = fn;
        jb[w].ctx = ctx;
        jb[w].lo = lo;
        jb[w].hi = hi;
        jb[w].w = w;
        jb[w].nw = nw;
        pthread_create(&th[w], NULL, worker, &jb[w]);
    }
    for (int w = 0; w < nw; ++w) pthread_join(th[w], NULL);
    free(th);
    free(jb);
}

/* t * polar(rho, theta) accumulated into (er, ei) exactly as
 * E += c.t * std::polar(1.0 / R, k * R) (focal.cpp:232). */
static inline void acc_term(double tr, double ti, double R, double k, double* er, double* ei) {
    const double rho = 1.0 / R;
    const double th = k * R;
    const double pr = rho * cos(th);
    const double pim = rho * sin(th);
    *er += tr * pr - ti * pim;
    *ei += tr * pim + ti * pr;
}

static void one_pixel(const double* px, const double* py, const double* pt, int npil, double fx,
                      double fy, double z, double k, double* er, double* ei) {
    double sr = 0.0, si = 0.0;
    for (int p = 0; p < npil; ++p) {
        const double R = sqrt((fx - px[p]) * (fx - px[p]) + (fy - py[p]) * (fy - py[p]) + z * z);
        acc_term(pt[2 * p], pt[2 * p + 1], R, k, &sr, &si);
    }
    *er = sr;
    *ei = si;
}

typedef struct {
    const double *px, *py, *pt;
    int npil, n, nx, nz;
    double cx, cy, z, k, half_window, step;
    double xmin, xmax, zmin, zmax;
    const int* idx;
    const double* v;
    double *field, *intensity, *out;
} ctx_t;

static void field_row(void* c_, int j) {
    ctx_t* c = (ctx_t*)c_;
    const double fy = c->cy - c->half_window + j * c->step;
    for (int i = 0; i < c->n; ++i) {
        const double fx = c->cx - c->half_window + i * c->step;
        double er, ei;
        one_pixel(c->px, c->py, c->pt, c->npil, fx, fy, c->z, c->k, &er, &ei);
        const size_t q = (size_t)j * c->n + i;
        if (c->field) {
            c->field[2 * q] = er;
            c->field[2 * q + 1] = ei;
        }
        if (c->intensity) c->intensity[q] = er * er + ei * ei;
    }
}

/* Rows [row_lo, row_hi) of the n x n grid. field (2*n*n) and intensity (n*n)
 * are indexed by the full-grid pixel index; either may be NULL. */
void rs_field(const double* px, const double* py, const double* pt, int npil, double cx,
              double cy, double z, double k, int n, double half_window, int row_lo, int row_hi,
              double* field, double* intensity) {
    ctx_t c = {0};
    c.px = px;
    c.py = py;
    c.pt = pt;
    c.npil = npil;
    c.n = n;
    c.cx = cx;
    c.cy = cy;
    c.z = z;
    c.k = k;
    c.half_window = half_window;
    c.step = 2.0 * half_window / (n - 1);
    c.field = field;
    c.intensity = intensity;
    parallel_items(row_lo, row_hi, field_row, &c);
}

static void pixel_item(void* c_, int s) {
    ctx_t* c = (ctx_t*)c_;
    const int j = c->idx[s] / c->n, i = c->idx[s] % c->n;
    const double fy = c->cy - c->half_window + j * c->step;
    const double fx = c->cx - c->half_window + i * c->step;
    one_pixel(c->px, c->py, c->pt, c->npil, fx, fy, c->z, c->k, &c->out[2 * s], &c->out[2 * s + 1]);
}

/* Selected pixels of the n x n grid: out (2*ns) receives E at idx[s]. */
void rs_pixels(const double* px, const double* py, const double* pt, int npil, double cx,
               double cy, double z, double k, int n, double half_window, const int* idx, int ns,
               double* out) {
    ctx_t c = {0};
    c.px = px;
    c.py = py;
    c.pt = pt;
    c.npil = npil;
    c.n = n;
    c.cx = cx;
    c.cy = cy;
    c.z = z;
    c.k = k;
    c.half_window = half_window;
    c.step = 2.0 * half_window / (n - 1);
    c.idx = idx;
    c.out = out;
    parallel_items(0, ns, pixel_item, &c);
}

static void zx_row(void* c_, int iz) {
    ctx_t* c = (ctx_t*)c_;
    const double z = c->zmin + (c->zmax - c->zmin) * iz / (c->nz - 1);
    for (int ix = 0; ix < c->nx; ++ix) {
        const double fx = c->xmin + (c->xmax - c->xmin) * ix / (c->nx - 1);
        double er = 0.0, ei = 0.0;
        for (int p = 0; p < c->npil; ++p) {
            const double r = sqrt((fx - c->px[p]) * (fx - c->px[p]) + c->py[p] * c->py[p] + z * z);
            acc_term(c->pt[2 * p], c->pt[2 * p + 1], r, c->k, &er, &ei);
        }
        c->out[(size_t)iz * c->nx + ix] = er * er + ei * ei;
    }
}

/* Caustic in the y = 0 plane: out[iz*nx + ix] = |E|^2 (throughfocus.cpp:105-118). */
void rs_zx(const double* px, const double* py, const double* pt, int npil, double xmin,
           double xmax, int nx, double zmin, double zmax, int nz, double k, double* out) {
    ctx_t c = {0};
    c.px = px;
    c.py = py;
    c.pt = pt;
    c.npil = npil;
    c.k = k;
    c.xmin = xmin;
    c.xmax = xmax;
    c.nx = nx;
    c.zmin = zmin;
    c.zmax = zmax;
    c.nz = nz;
    c.out = out;
    parallel_items(0, nz, zx_row, &c);
}

static void adj_item(void* c_, int p) {
    ctx_t* c = (ctx_t*)c_;
    double gr = 0.0, gi = 0.0;
    for (int j = 0; j < c->n; ++j) {
        const double fy = c->cy - c->half_window + j * c->step;
        for (int i = 0; i < c->n; ++i) {
            const double fx = c->cx - c->half_window + i * c->step;
            const double R = sqrt((fx - c->px[p]) * (fx - c->px[p]) +
                                  (fy - c->py[p]) * (fy - c->py[p]) + c->z * c->z);
            const double rho = 1.0 / R;
            const double cs = rho * cos(c->k * R), sn = rho * sin(c->k * R);
            const size_t q = (size_t)j * c->n + i;
            gr += cs * c->v[2 * q] + sn * c->v[2 * q + 1];
            gi += cs * c->v[2 * q + 1] - sn * c->v[2 * q];
        }
    }
    c->out[2 * p] = gr;
    c->out[2 * p + 1] = gi;
}

/* Adjoint: out_j = sum_p conj(g_pj) v_p over the n x n grid (row-major p). */
void rs_adjoint(const double* px, const double* py, int npil, double cx, double cy, double z,
                double k, int n, double half_window, const double* v, double* out) {
    ctx_t c = {0};
    c.px = px;
    c.py = py;
    c.npil = npil;
    c.n = n;
    c.cx = cx;
    c.cy = cy;
    c.z = z;
    c.k = k;
    c.half_window = half_window;
    c.step = 2.0 * half_window / (n - 1);
    c.v = v;
    c.out = out;
    parallel_items(0, npil, adj_item, &c);
}
