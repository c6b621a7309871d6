/*
 * cuphu_oracle.c -- CPU restatement of cuPHU's data-parallel unwrapping path.
 *
 * TEST INFRASTRUCTURE ONLY (see cuphu_oracle.h).  Restates, in plain C, the
 * arithmetic of the reference files named beside each function, so that the
 * B200 kernels can be checked against it bit for bit.  Compiled with
 * -ffp-contract=off: every fused multiply-add below is explicit and mirrors
 * a contraction that nvcc performs in the reference kernel it restates.
 *
 * Deliberate extensions over the reference (documented, shared with the GPU
 * kernels):
 *  - mirror padding reflects repeatedly when the half-window exceeds the
 *    array extent (the reference reads out of bounds there,
 *    cuphu_util.cu:172-177);
 *  - residues (no cuPHU code exists) use the elementary-loop definition
 *    right, down, left, up over the A2 wrapped differences;
 *  - the Laplace solve here is the FP64 restatement of the reference FP32
 *    Jacobi-PCG + IRLS (cuphu_laplace.cu:352-549) with a fixed reduction
 *    tree, and is the "FP64 oracle" for the GPU solvers.
 */
#include "cuphu_oracle.h"

#include <math.h>
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define TWOPI_F      6.28318548202514648f    /* 2*CUDART_PI_F, cuphu_util.cu:23 */
#define INV_TWOPI_F  0.15915494309189534561f /* cuphu_laplace.cu:60 */
#define LAP_EPS_F    1e-12f                  /* cuphu_laplace.cu:61 */
#define LARGESIGSQ   32000                   /* cuphu_laplace.cu:62 */
#define LARGESHORT   32000

/* PTX cvt.rzi.s32.f64 (C cast in device code): NaN -> 0, saturating. */
static inline int cvt_rzi(double v)
{
    if (v != v) return 0;
    if (v >= 2147483647.0) return INT_MAX;
    if (v <= -2147483648.0) return INT_MIN;
    return (int)v;
}

/* __double2int_rn: round to nearest even, NaN -> 0, saturating. */
static inline int cvt_rni(double v)
{
    if (v != v) return 0;
    double r = nearbyint(v);
    if (r >= 2147483647.0) return INT_MAX;
    if (r <= -2147483648.0) return INT_MIN;
    return (int)r;
}

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* ── A1: phase ─────────────────────────────────────────────────────────────
 * Host atan2 shifted to [0,2pi) (cuphu_solver.cpp:1706-1712), then the
 * device re-wrap p - 2pi*floor(p/2pi) (cuphu_util.cu:33-36, launched at
 * cuphu_solver.cpp:397). */
static inline float rewrap(float p)
{
    return fmaf(-TWOPI_F, floorf(p / TWOPI_F), p);
}

void orc_phase_from_igram(const float *re, const float *im, long n, float *phase)
{
    #pragma omp parallel for schedule(static)
    for (long k = 0; k < n; ++k) {
        float phi = atan2f(im[k], re[k]);
        if (phi < 0.0f) phi += 6.28318530717958648f;
        phase[k] = rewrap(phi);
    }
}

void orc_phase_from_c64(const float *c64, long n, float *phase)
{
    #pragma omp parallel for schedule(static)
    for (long k = 0; k < n; ++k) {
        float phi = atan2f(c64[2 * k + 1], c64[2 * k]);
        if (phi < 0.0f) phi += 6.28318530717958648f;
        phase[k] = rewrap(phi);
    }
}

void orc_wrap_phase(float *p, long n)
{
    for (long k = 0; k < n; ++k) p[k] = rewrap(p[k]);
}

/* ── A2: wrapped differences in cycles (cuphu_util.cu:27-30, 54-92) ─────── */
static inline float wrap_cycles(float d) { return d - floorf(d + 0.5f); }

void orc_phase_diffs(const float *phase, int nrow, int ncol, float *rng, float *az)
{
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol - 1; ++c)
            rng[(size_t)r * (ncol - 1) + c] = wrap_cycles(
                (phase[(size_t)r * ncol + c + 1] - phase[(size_t)r * ncol + c]) / TWOPI_F);
    for (int r = 0; r < nrow - 1; ++r)
        for (int c = 0; c < ncol; ++c)
            az[(size_t)r * ncol + c] = wrap_cycles(
                (phase[(size_t)r * ncol + c] - phase[(size_t)(r + 1) * ncol + c]) / TWOPI_F);
}

/* ── A3: mirror-padded separable boxcar (cuphu_util.cu:104-181, 237-287) ── */
static inline int reflect_index(int i, int n)
{
    if (n <= 1) return 0;
    int period = 2 * (n - 1);
    int j = i % period;
    if (j < 0) j += period;
    if (j > n - 1) j = period - j;
    return j;
}

void orc_boxcar2d(const float *src, float *dst, int nrow, int ncol, int kr, int kc)
{
    if (nrow <= 0 || ncol <= 0) return;
    int prow = nrow + 2 * kr;
    int wlc = 2 * kc + 1, wlr = 2 * kr + 1;
    float *tmp = (float *)malloc((size_t)prow * ncol * sizeof(float));
    /* row pass over every padded row */
    for (int i = 0; i < prow; ++i) {
        const float *srow = src + (size_t)reflect_index(i - kr, nrow) * ncol;
        for (int c = 0; c < ncol; ++c) {
            float s = 0.0f;
            for (int k = 0; k < wlc; ++k)
                s += srow[reflect_index(c + k - kc, ncol)];
            tmp[(size_t)i * ncol + c] = s / (float)wlc;
        }
    }
    /* column pass */
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol; ++c) {
            float s = 0.0f;
            for (int k = 0; k < wlr; ++k) s += tmp[(size_t)(r + k) * ncol + c];
            dst[(size_t)r * ncol + c] = s / (float)wlr;
        }
    free(tmp);
}

/* ── A4: scalar constants (cuphu_cost.cu:41-59), host arithmetic ─────────── */
void orc_cost_constants(const orc_cost_params *p, double out[9])
{
    double rho0 = p->rhosconst1 / p->ncorrlooks + p->rhosconst2;
    double thresh = p->defothreshfactor * rho0;
    double rhopow = 2.0 * p->cstd1 + p->cstd2 * log(p->ncorrlooks) + p->cstd3 * p->ncorrlooks;
    out[0] = rho0;
    out[1] = thresh;
    out[2] = rhopow;
    out[3] = 2.0 / 12.0;
    out[4] = p->sigsqcorr;
    out[5] = p->nshortcycle;
    out[6] = p->nshortcycle * p->nshortcycle;
    out[7] = p->costscale;
    out[8] = (double)(int)p->sigsqshortmin;
}

/* ── A7: mask -> arc weights (cuphu_solver.cpp:404-426), flat row-then-col */
void orc_arc_weights_from_mask(const unsigned char *mask, int nrow, int ncol, short *w)
{
    size_t nra = (size_t)(nrow - 1) * ncol;
    for (int r = 0; r < nrow - 1; ++r)
        for (int c = 0; c < ncol; ++c)
            w[(size_t)r * ncol + c] =
                (mask[(size_t)r * ncol + c] && mask[(size_t)(r + 1) * ncol + c]) ? 1 : 0;
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol - 1; ++c)
            w[nra + (size_t)r * (ncol - 1) + c] =
                (mask[(size_t)r * ncol + c] && mask[(size_t)r * ncol + c + 1]) ? 1 : 0;
}

/* ── A5/A6: per-arc statistical cost (cuphu_cost.cu:77-323) ───────────────
 * mode 0 = SMOOTH (2 shorts/arc), 1|2 = DEFO/TOPO (4 shorts/arc). */
static void arc_cost(double ca, double cb, float dpsi, float avgdpsi, short w,
                     int mode, const double k[9], double defomax, short *o)
{
    if (w == 0) {
        o[0] = LARGESHORT / 2;
        o[1] = LARGESHORT;
        if (mode) { o[2] = LARGESHORT; o[3] = 0; }
        return;
    }
    double rho = 0.5 * (ca + cb);
    if (rho < k[1]) rho = 0.0;
    double sigsqrho = fma(k[3], pow(1.0 - rho, k[2]), k[4]) * k[6];
    double dp = (double)dpsi, avg = (double)avgdpsi;
    double offset = k[5] * (dp - (rho > 0 ? avg : 0.5 * avg));
    double sigsq_f = sigsqrho / (k[7] * (double)w);
    int sigsq_i = cvt_rzi(sigsq_f);
    int sqmin = (int)k[8];
    if (sigsq_i < sqmin) sigsq_i = sqmin;
    int off_i, dzmax = 0, laycost = 0;
    if (mode) {
        dzmax = cvt_rni(k[5] * defomax);
        dzmax = imax(1, imin(dzmax, SHRT_MAX));
        /* int product wraps on the device; emulate with unsigned */
        int prod = (int)((unsigned)dzmax * (unsigned)sigsq_i);
        laycost = cvt_rzi(sqrt((double)prod));
        laycost = imin(laycost, SHRT_MAX);
        off_i = cvt_rni(offset);
    } else {
        off_i = cvt_rzi(offset);
    }
    off_i = imax(off_i, SHRT_MIN);
    off_i = imin(off_i, SHRT_MAX);
    sigsq_i = imin(sigsq_i, SHRT_MAX);
    o[0] = (short)off_i;
    o[1] = (short)sigsq_i;
    if (mode) { o[2] = (short)dzmax; o[3] = (short)laycost; }
}

int orc_build_costs(const float *phase, const float *corr, const short *weights,
                    int nrow, int ncol, int mode, const orc_cost_params *p,
                    int kperp, int kpar, short *out)
{
    double k[9];
    orc_cost_constants(p, k);
    int es = mode ? 4 : 2;
    size_t nra = (size_t)(nrow - 1) * ncol, nca = (size_t)nrow * (ncol - 1);
    float *rng = (float *)malloc((nca + 1) * sizeof(float));
    float *az = (float *)malloc((nra + 1) * sizeof(float));
    float *arng = (float *)malloc((nca + 1) * sizeof(float));
    float *aaz = (float *)malloc((nra + 1) * sizeof(float));
    orc_phase_diffs(phase, nrow, ncol, rng, az);
    if (nca) orc_boxcar2d(rng, arng, nrow, ncol - 1, kperp / 2, kpar / 2);
    if (nra) orc_boxcar2d(az, aaz, nrow - 1, ncol, kpar / 2, kperp / 2);
    /* row arcs (r,c)->(r+1,c) use azimuth diffs */
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < nrow - 1; ++r)
        for (int c = 0; c < ncol; ++c) {
            size_t a = (size_t)r * ncol + c;
            short w = weights ? weights[a] : 1;
            arc_cost((double)corr[(size_t)r * ncol + c], (double)corr[(size_t)(r + 1) * ncol + c],
                     az[a], aaz[a], w, mode, k, p->defomax, out + a * es);
        }
    /* col arcs (r,c)->(r,c+1) use range diffs */
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol - 1; ++c) {
            size_t a = (size_t)r * (ncol - 1) + c;
            short w = weights ? weights[nra + a] : 1;
            arc_cost((double)corr[(size_t)r * ncol + c], (double)corr[(size_t)r * ncol + c + 1],
                     rng[a], arng[a], w, mode, k, p->defomax, out + (nra + a) * es);
        }
    free(rng); free(az); free(arng); free(aaz);
    return es * 2;
}

/* ── A8: residues.  No cuPHU code exists; defined as the rounded sum of the
 * A2 wrapped differences (cycles) around the elementary loop
 * (r,c)->(r,c+1)->(r+1,c+1)->(r+1,c)->(r,c).  Output (nrow-1)x(ncol-1). */
void orc_residues(const float *phase, int nrow, int ncol, signed char *out)
{
    for (int r = 0; r < nrow - 1; ++r)
        for (int c = 0; c < ncol - 1; ++c) {
            const float *p0 = phase + (size_t)r * ncol + c;
            const float *p1 = p0 + ncol;
            float rng0 = wrap_cycles((p0[1] - p0[0]) / TWOPI_F);
            float rng1 = wrap_cycles((p1[1] - p1[0]) / TWOPI_F);
            float az0 = wrap_cycles((p0[0] - p1[0]) / TWOPI_F);
            float az1 = wrap_cycles((p0[1] - p1[1]) / TWOPI_F);
            float s = ((rng0 - az1) - rng1) + az0;
            out[(size_t)r * (ncol - 1) + c] = (signed char)rintf(s);
        }
}

/* ── canonical deterministic reduction, mirrored by the GPU solver ─────────
 * A tile is cut into work items of by rows x (tx*vx) columns; thread
 * (ty,tx) of an item accumulates its vx pixels with fma in column order;
 * warps reduce with a shuffle-down tree; warp 0 reduces the warp sums; the
 * tile total reduces item partials with a strided per-thread sum followed by
 * the same block tree. */
static double tree32(double *v)
{
    for (int off = 16; off >= 1; off >>= 1)
        for (int i = 0; i < off; ++i) v[i] = v[i] + v[i + off];
    return v[0];
}

static double block_tree(const double *th, int nthreads)
{
    double ws[32];
    int nw = nthreads / 32;
    for (int w = 0; w < nw; ++w) {
        double v[32];
        memcpy(v, th + 32 * w, sizeof(v));
        ws[w] = tree32(v);
    }
    double v[32];
    for (int i = 0; i < 32; ++i) v[i] = i < nw ? ws[i] : 0.0;
    return tree32(v);
}

typedef struct {
    int nrow, ncol, tx, vx, by, bx, nbx, nby, nitems, nthreads;
} dotgeom;

static dotgeom make_geom(int nrow, int ncol, int tx, int vx, int by)
{
    dotgeom g;
    g.nrow = nrow; g.ncol = ncol; g.tx = tx; g.vx = vx; g.by = by;
    g.bx = tx * vx;
    g.nbx = (ncol + g.bx - 1) / g.bx;
    g.nby = (nrow + by - 1) / by;
    g.nitems = g.nbx * g.nby;
    g.nthreads = tx * by;
    return g;
}

static double item_partial(const dotgeom *g, int item, const double *a, const double *b)
{
    double th[1024];
    int iby = item / g->nbx, ibx = item % g->nbx;
    for (int ty = 0; ty < g->by; ++ty)
        for (int tx = 0; tx < g->tx; ++tx) {
            double acc = 0.0;
            int row = iby * g->by + ty;
            for (int j = 0; j < g->vx; ++j) {
                int col = ibx * g->bx + tx * g->vx + j;
                if (row < g->nrow && col < g->ncol) {
                    size_t i = (size_t)row * g->ncol + col;
                    acc = fma(a[i], b[i], acc);
                }
            }
            th[ty * g->tx + tx] = acc;
        }
    return block_tree(th, g->nthreads);
}

static double tile_total(const dotgeom *g, const double *part)
{
    double th[1024];
    for (int j = 0; j < g->nthreads; ++j) {
        double acc = 0.0;
        for (int i = j; i < g->nitems; i += g->nthreads) acc = acc + part[i];
        th[j] = acc;
    }
    return block_tree(th, g->nthreads);
}

static double dot_geom(const dotgeom *g, const double *a, const double *b, double *part)
{
    #pragma omp parallel for schedule(static)
    for (int it = 0; it < g->nitems; ++it) part[it] = item_partial(g, it, a, b);
    return tile_total(g, part);
}

double orc_dot_canonical(const double *a, const double *b, int nrow, int ncol,
                         int tx, int vx, int by)
{
    dotgeom g = make_geom(nrow, ncol, tx, vx, by);
    double *part = (double *)malloc((size_t)g.nitems * sizeof(double));
    double s = dot_geom(&g, a, b, part);
    free(part);
    return s;
}

/* ── A9-A14: Laplace WLS Jacobi-PCG + IRLS, FP64 (cuphu_laplace.cu:65-549) ─ */
static inline float lap_wrap_pi(float x)
{
    return fmaf(-TWOPI_F, rintf(x * INV_TWOPI_F), x);
}

/* y = A x: eps*x + sum over arcs (down, up, right, left) w*(x_a - x_nb) */
static void lap_matvec(const float *wd, const float *wr, const double *x, double *y,
                       int nrow, int ncol)
{
    const double eps = (double)LAP_EPS_F;
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol; ++c) {
            size_t i = (size_t)r * ncol + c;
            double xa = x[i];
            double v = eps * xa;
            if (r < nrow - 1) v = fma((double)wd[i], xa - x[i + ncol], v);
            if (r > 0)        v = fma((double)wd[i - ncol], xa - x[i - ncol], v);
            if (c < ncol - 1) v = fma((double)wr[(size_t)r * (ncol - 1) + c], xa - x[i + 1], v);
            if (c > 0)        v = fma((double)wr[(size_t)r * (ncol - 1) + c - 1], xa - x[i - 1], v);
            y[i] = v;
        }
}

int orc_laplace_f64(const short *costs, int cost_stride, const float *phase,
                    int nrow, int ncol, const orc_lap_opts *o,
                    double *x_out, int *k_out, float *unw_out, int *iters_out)
{
    size_t npix = (size_t)nrow * ncol;
    size_t nra = (size_t)(nrow - 1) * ncol, nca = (size_t)nrow * (ncol - 1);
    size_t narcs = nra + nca;
    float *w0 = (float *)malloc((narcs + 1) * sizeof(float));
    float *w = (float *)malloc((narcs + 1) * sizeof(float));
    double *x = x_out;
    double *rv = (double *)malloc(npix * sizeof(double));
    double *z = (double *)malloc(npix * sizeof(double));
    double *pv = (double *)malloc(npix * sizeof(double));
    double *q = (double *)malloc(npix * sizeof(double));
    double *b = (double *)malloc(npix * sizeof(double));
    double *diag = (double *)malloc(npix * sizeof(double));
    dotgeom g = make_geom(nrow, ncol, o->item_tx, o->item_vx, o->item_by);
    double *part = (double *)malloc((size_t)g.nitems * sizeof(double));
    const double eps = (double)LAP_EPS_F;

    /* A9: w0 = 1/sigsq, 0 when masked or no-preference (cuphu_laplace.cu:65-69) */
    for (size_t a = 0; a < narcs; ++a) {
        short s = costs[a * cost_stride + 1];
        w0[a] = (s <= 0 || s >= LARGESIGSQ) ? 0.0f : 1.0f / (float)s;
        w[a] = w0[a];
    }
    const float *w0d = w0, *w0r = w0 + nra;
    float *wd = w, *wr = w + nra;

    for (int outer = 0; outer <= o->n_irls; ++outer) {
        /* A10: b and diag (cuphu_laplace.cu:88-148), double accumulation */
        #pragma omp parallel for schedule(static)
        for (int r = 0; r < nrow; ++r)
            for (int c = 0; c < ncol; ++c) {
                size_t i = (size_t)r * ncol + c;
                float pa = phase[i];
                double bv = 0.0, ws = 0.0;
                if (r < nrow - 1) {
                    float wv = wd[i];
                    if (wv > 0.0f) {
                        float gph = lap_wrap_pi(phase[i + ncol] - pa);
                        bv = fma(-(double)wv, (double)gph, bv);
                        ws += wv;
                    }
                }
                if (r > 0) {
                    float wv = wd[i - ncol];
                    if (wv > 0.0f) {
                        float gph = lap_wrap_pi(pa - phase[i - ncol]);
                        bv = fma((double)wv, (double)gph, bv);
                        ws += wv;
                    }
                }
                if (c < ncol - 1) {
                    float wv = wr[(size_t)r * (ncol - 1) + c];
                    if (wv > 0.0f) {
                        float gph = lap_wrap_pi(phase[i + 1] - pa);
                        bv = fma(-(double)wv, (double)gph, bv);
                        ws += wv;
                    }
                }
                if (c > 0) {
                    float wv = wr[(size_t)r * (ncol - 1) + c - 1];
                    if (wv > 0.0f) {
                        float gph = lap_wrap_pi(pa - phase[i - 1]);
                        bv = fma((double)wv, (double)gph, bv);
                        ws += wv;
                    }
                }
                b[i] = bv;
                diag[i] = ws + eps;
            }
        if (outer == 0) memset(x, 0, npix * sizeof(double));
        /* r = b - A x, z = r/diag, p = z */
        lap_matvec(wd, wr, x, q, nrow, ncol);
        for (size_t i = 0; i < npix; ++i) {
            rv[i] = b[i] - q[i];
            z[i] = rv[i] / diag[i];
            pv[i] = z[i];
        }
        double rz = dot_geom(&g, rv, z, part);
        double rz0 = rz;
        int iter = 0;
        if (rz0 > 0.0) {
            double thr = (double)o->tol * (double)o->tol * rz0;
            for (; iter < o->max_iter; ++iter) {
                lap_matvec(wd, wr, pv, q, nrow, ncol);
                double pq = dot_geom(&g, pv, q, part);
                if (pq <= 0.0) break;
                double alpha = rz / pq;
                #pragma omp parallel for schedule(static)
                for (size_t i = 0; i < npix; ++i) {
                    x[i] = fma(alpha, pv[i], x[i]);
                    rv[i] = fma(-alpha, q[i], rv[i]);
                    z[i] = rv[i] / diag[i];
                }
                double rzn = dot_geom(&g, rv, z, part);
                if (rzn < thr) { iter++; break; }
                double beta = rzn / rz;
                rz = rzn;
                #pragma omp parallel for schedule(static)
                for (size_t i = 0; i < npix; ++i) pv[i] = fma(beta, pv[i], z[i]);
            }
        }
        if (iters_out) iters_out[outer] = iter;
        /* A13: IRLS reweight (cuphu_laplace.cu:214-247, schedule :515-522) */
        if (outer < o->n_irls) {
            float delta = fmaxf(o->delta_min, o->delta_max * powf(0.5f, (float)outer));
            double dd = (double)delta * (double)delta;
            #pragma omp parallel for schedule(static)
            for (long a = 0; a < (long)narcs; ++a) {
                float w0v = (size_t)a < nra ? w0d[a] : w0r[a - nra];
                float *dst = (size_t)a < nra ? &wd[a] : &wr[a - nra];
                if (w0v <= 0.0f) { *dst = 0.0f; continue; }
                size_t tail, head;
                if ((size_t)a < nra) {
                    int r = (int)(a / ncol), c = (int)(a % ncol);
                    tail = (size_t)r * ncol + c; head = tail + ncol;
                } else {
                    long j = a - (long)nra;
                    int r = (int)(j / (ncol - 1)), c = (int)(j % (ncol - 1));
                    tail = (size_t)r * ncol + c; head = tail + 1;
                }
                float gph = lap_wrap_pi(phase[head] - phase[tail]);
                double e = (x[head] - x[tail]) - (double)gph;
                *dst = (float)((double)w0v / sqrt(fma(e, e, dd)));
            }
        }
    }
    /* A14: anchor at (0,0) and congruence (cuphu_laplace.cu:527-549) */
    double off = (double)phase[0] - x[0];
    for (size_t i = 0; i < npix; ++i) {
        double d = (x[i] + off) - (double)phase[i];
        double kk = rint(d / (2.0 * M_PI));
        if (k_out) k_out[i] = (int)kk;
        if (unw_out) unw_out[i] = fmaf(TWOPI_F, (float)kk, phase[i]);
    }
    free(w0); free(w); free(rv); free(z); free(pv); free(q); free(b); free(diag); free(part);
    return 0;
}

/* ── A16: connected components (cuphu_conncomp.cu:67-93, 178-286, 290-428) ─
 * Sequential union-find; roots are minimum pixel indices, so the result is
 * the reference's canonical labelling. */
static unsigned uf_find(unsigned *par, unsigned i)
{
    while (par[i] != i) { par[i] = par[par[i]]; i = par[i]; }
    return i;
}

static void uf_union(unsigned *par, unsigned a, unsigned b)
{
    unsigned ra = uf_find(par, a), rb = uf_find(par, b);
    if (ra == rb) return;
    if (ra < rb) par[rb] = ra; else par[ra] = rb;
}

int orc_conncomp(const float *unw, const float *corr, const unsigned char *mask,
                 int nrow, int ncol, const short *poscost, const short *negcost,
                 double minfrac, long maxncomps, long conncompthresh,
                 unsigned *labels)
{
    size_t npix = (size_t)nrow * ncol;
    size_t nra = (size_t)(nrow - 1) * ncol;
    unsigned *par = (unsigned *)malloc(npix * sizeof(unsigned));
    unsigned char *valid = (unsigned char *)malloc(npix);
    const float pthresh = 3.14159274101257324f;   /* (float)CUDART_PI_F */
    for (size_t i = 0; i < npix; ++i) {
        par[i] = (unsigned)i;
        int bad = corr[i] < 0.05f;
        if (mask) bad = bad || mask[i] == 0;
        valid[i] = !bad;
    }
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol; ++c) {
            size_t i = (size_t)r * ncol + c;
            if (!valid[i]) continue;
            if (c + 1 < ncol && valid[i + 1] && fabsf(unw[i] - unw[i + 1]) < pthresh) {
                int ok = 1;
                if (poscost) {
                    size_t a = nra + (size_t)r * (ncol - 1) + c;
                    short mc = poscost[a] < negcost[a] ? poscost[a] : negcost[a];
                    ok = (long)mc >= conncompthresh;
                }
                if (ok) uf_union(par, (unsigned)i, (unsigned)(i + 1));
            }
            if (r + 1 < nrow && valid[i + ncol] && fabsf(unw[i] - unw[i + ncol]) < pthresh) {
                int ok = 1;
                if (poscost) {
                    size_t a = (size_t)r * ncol + c;
                    short mc = poscost[a] < negcost[a] ? poscost[a] : negcost[a];
                    ok = (long)mc >= conncompthresh;
                }
                if (ok) uf_union(par, (unsigned)i, (unsigned)(i + ncol));
            }
        }
    unsigned *cnt = (unsigned *)calloc(npix, sizeof(unsigned));
    for (size_t i = 0; i < npix; ++i)
        if (valid[i]) cnt[uf_find(par, (unsigned)i)]++;
    int min_size = (int)(minfrac * (double)npix);
    if (min_size < 1) min_size = 1;
    unsigned *map = (unsigned *)calloc(npix, sizeof(unsigned));
    unsigned next = 1;
    for (size_t i = 0; i < npix && (long)next - 1 < maxncomps; ++i)
        if (cnt[i] >= (unsigned)min_size) map[i] = next++;
    for (size_t i = 0; i < npix; ++i)
        labels[i] = valid[i] ? map[uf_find(par, (unsigned)i)] : 0u;
    free(par); free(valid); free(cnt); free(map);
    return (int)(next - 1);
}

/* ── A15: flow integration (cuphu_phase.cu:27-106), sequential float sums ─ */
static inline float wrap_angle(float x)
{
    return fmaf(-TWOPI_F, rintf(x / TWOPI_F), x);
}

void orc_integrate_phase(const float *phase, const short *hflows, const short *vflows,
                         int nrow, int ncol, float *unw)
{
    float *rowoff = (float *)malloc((size_t)nrow * sizeof(float));
    float cs = 0.0f;
    rowoff[0] = 0.0f;
    for (int r = 1; r < nrow; ++r) {
        float d = phase[(size_t)r * ncol] - phase[(size_t)(r - 1) * ncol];
        cs += fmaf(-TWOPI_F, (float)hflows[(size_t)(r - 1) * ncol], wrap_angle(d));
        rowoff[r] = cs;
    }
    float ref = phase[0];
    for (int r = 0; r < nrow; ++r) {
        float c2 = 0.0f;
        unw[(size_t)r * ncol] = (ref + rowoff[r]) + 0.0f;
        for (int c = 1; c < ncol; ++c) {
            float d = phase[(size_t)r * ncol + c] - phase[(size_t)r * ncol + c - 1];
            c2 += fmaf(TWOPI_F, (float)vflows[(size_t)r * (ncol - 1) + c - 1], wrap_angle(d));
            unw[(size_t)r * ncol + c] = (ref + rowoff[r]) + c2;
        }
    }
    free(rowoff);
}

/* ── A18: incremental costs (cuphu_incrcost.cu:25-98, 157-191) ──────────── */
static inline long ceil_div(long a, long b) { return a > 0 ? (a + b - 1) / b : a / b; }
static inline long floor_div(long a, long b) { return a >= 0 ? a / b : (a - b + 1) / b; }

int orc_incrcost(const short *costs, const short *flows, long narcs, long nsc,
                 int nflow, short *pos, short *neg)
{
    int mnp = 32000, mnn = 32000;
    for (long i = 0; i < narcs; ++i) {
        short off = costs[2 * i], sg = costs[2 * i + 1];
        if (sg == 32000) { pos[i] = 0; neg[i] = 0; }
        else {
            long flow = flows[i], o = off, s = sg, nf = nflow;
            long i1 = labs(flow * nsc + o);
            long ip = labs((flow + nf) * nsc + o);
            long in = labs((flow - nf) * nsc + o);
            long c1 = (i1 * i1) / s;
            long pr = (ip * ip) / s - c1;
            long nr = (in * in) / s - c1;
            long nfsq = nf * nf;
            long pc = pr > 0 ? ceil_div(pr, nfsq) : floor_div(pr, nfsq);
            long nc = nr > 0 ? ceil_div(nr, nfsq) : floor_div(nr, nfsq);
            pc = pc < -32000 ? -32000 : (pc > 32000 ? 32000 : pc);
            nc = nc < -32000 ? -32000 : (nc > 32000 ? 32000 : nc);
            pos[i] = (short)pc; neg[i] = (short)nc;
        }
        if (pos[i] < mnp) mnp = pos[i];
        if (neg[i] < mnn) mnn = neg[i];
    }
    return (mnp >= 0 && mnn >= 0) ? 1 : 0;
}

/* ── A19: tile geometry, stitching and merge (cuphu_solver.cpp:1753-2031) ─ */
void orc_tile_bounds(int n, int nt, int ovl, int t, int *first, int *len)
{
    int f = (int)((long)t * (n - ovl) / nt);
    int last = (t == nt - 1) ? n : (int)((long)(t + 1) * (n - ovl) / nt) + ovl;
    *first = f;
    *len = last - f;
}

typedef struct { float v, w; } vw_pair;

static int cmp_pair(const void *a, const void *b)
{
    float x = ((const vw_pair *)a)->v, y = ((const vw_pair *)b)->v;
    return (x > y) - (x < y);
}

static double weighted_median(vw_pair *d, size_t n)
{
    if (n == 0) return 0.0;
    qsort(d, n, sizeof(vw_pair), cmp_pair);
    double total = 0.0;
    for (size_t i = 0; i < n; ++i) total += d[i].w;
    double half = total / 2.0, acc = 0.0;
    for (size_t i = 0; i < n; ++i) {
        acc += d[i].w;
        if (acc >= half) return (double)d[i].v;
    }
    return (double)d[n - 1].v;
}

typedef struct {
    int r0, c0, nr, nc;
    float *phase, *corr, *unw;
    unsigned char *mask, *conf;
    unsigned *cc;
} orc_tile;

static void tile_solve(orc_tile *t, int mode, const orc_cost_params *p, int kperp, int kpar,
                       const orc_lap_opts *o, double minfrac, long maxncomps, long cthr)
{
    size_t npix = (size_t)t->nr * t->nc;
    size_t narcs = (size_t)(t->nr - 1) * t->nc + (size_t)t->nr * (t->nc - 1);
    int es = mode ? 4 : 2;
    short *w = NULL;
    if (t->mask) {
        w = (short *)malloc((narcs + 1) * sizeof(short));
        orc_arc_weights_from_mask(t->mask, t->nr, t->nc, w);
    }
    short *costs = (short *)malloc((narcs + 1) * es * sizeof(short));
    orc_build_costs(t->phase, t->corr, w, t->nr, t->nc, mode, p, kperp, kpar, costs);
    double *x = (double *)malloc(npix * sizeof(double));
    orc_laplace_f64(costs, es, t->phase, t->nr, t->nc, o, x, NULL, t->unw, NULL);
    orc_conncomp(t->unw, t->corr, t->mask, t->nr, t->nc, NULL, NULL, minfrac, maxncomps,
                 cthr, t->cc);
    free(w); free(costs); free(x);
}

int orc_unwrap_tiled(const float *phase, const float *corr, const unsigned char *mask,
                     const unsigned char *conf_mask, int nrow, int ncol, int mode,
                     const orc_cost_params *p, int kperp, int kpar,
                     const orc_lap_opts *o, int ntr, int ntc, int rovl, int covl,
                     double minfrac, long maxncomps, long cthr,
                     float *unw, unsigned *cc, double *tile_k_out)
{
    int nt = ntr * ntc;
    orc_tile *T = (orc_tile *)calloc(nt, sizeof(orc_tile));
    const unsigned char *cm = conf_mask ? conf_mask : mask;
    for (int tr = 0; tr < ntr; ++tr)
        for (int tc = 0; tc < ntc; ++tc) {
            orc_tile *t = &T[tr * ntc + tc];
            if (ntr == 1 && ntc == 1) { t->r0 = 0; t->c0 = 0; t->nr = nrow; t->nc = ncol; }
            else {
                orc_tile_bounds(nrow, ntr, rovl, tr, &t->r0, &t->nr);
                orc_tile_bounds(ncol, ntc, covl, tc, &t->c0, &t->nc);
            }
            size_t np = (size_t)t->nr * t->nc;
            t->phase = (float *)malloc(np * sizeof(float));
            t->corr = (float *)malloc(np * sizeof(float));
            t->unw = (float *)malloc(np * sizeof(float));
            t->cc = (unsigned *)malloc(np * sizeof(unsigned));
            t->mask = mask ? (unsigned char *)malloc(np) : NULL;
            t->conf = cm ? (unsigned char *)malloc(np) : NULL;
            for (int r = 0; r < t->nr; ++r)
                for (int c = 0; c < t->nc; ++c) {
                    size_t ti = (size_t)r * t->nc + c;
                    size_t gi = (size_t)(t->r0 + r) * ncol + t->c0 + c;
                    t->phase[ti] = phase[gi];
                    t->corr[ti] = corr[gi];
                    if (mask) t->mask[ti] = mask[gi];
                    if (cm) t->conf[ti] = cm[gi];
                }
        }
    for (int i = 0; i < nt; ++i)
        tile_solve(&T[i], mode, p, kperp, kpar, o, minfrac, maxncomps, cthr);

    double *tk = (double *)calloc(nt, sizeof(double));
    if (nt > 1 && (rovl > 0 || covl > 0)) {
        int *visited = (int *)calloc(nt, sizeof(int));
        int *queue = (int *)malloc(nt * sizeof(int));
        int qh = 0, qt = 0;
        queue[qt++] = 0; visited[0] = 1;
        while (qh < qt) {
            int idx = queue[qh++];
            int br = idx / ntc, bc = idx % ntc;
            for (int dir = 0; dir < 2; ++dir) {
                int nb;
                if (dir == 0) { if (bc + 1 >= ntc) continue; nb = br * ntc + bc + 1; }
                else          { if (br + 1 >= ntr) continue; nb = (br + 1) * ntc + bc; }
                if (visited[nb]) continue;
                const orc_tile *A = &T[idx], *B = &T[nb];
                double k = 0.0;
                int ov = dir == 0 ? covl : rovl;
                int okay = dir == 0 ? (ov > 0 && ov <= A->nc && ov <= B->nc)
                                    : (ov > 0 && ov <= A->nr && ov <= B->nr);
                if (okay) {
                    size_t cap = dir == 0 ? (size_t)imin(A->nr, B->nr) * ov
                                          : (size_t)imin(A->nc, B->nc) * ov;
                    vw_pair *dw = (vw_pair *)malloc((cap + 1) * sizeof(vw_pair));
                    size_t n = 0;
                    int n1 = dir == 0 ? imin(A->nr, B->nr) : ov;
                    int n2 = dir == 0 ? ov : imin(A->nc, B->nc);
                    for (int i = 0; i < n1; ++i)
                        for (int j = 0; j < n2; ++j) {
                            size_t ap, bp;
                            if (dir == 0) {
                                ap = (size_t)i * A->nc + (A->nc - ov + j);
                                bp = (size_t)i * B->nc + j;
                            } else {
                                ap = (size_t)(A->nr - ov + i) * A->nc + j;
                                bp = (size_t)i * B->nc + j;
                            }
                            if (A->corr[ap] < 0.05f || B->corr[bp] < 0.05f) continue;
                            if (A->conf && !A->conf[ap]) continue;
                            if (B->conf && !B->conf[bp]) continue;
                            dw[n].v = A->unw[ap] - B->unw[bp];
                            dw[n].w = A->corr[ap] < B->corr[bp] ? A->corr[ap] : B->corr[bp];
                            n++;
                        }
                    k = weighted_median(dw, n) / (2.0 * M_PI);
                    free(dw);
                }
                tk[nb] = tk[idx] + k;
                visited[nb] = 1;
                queue[qt++] = nb;
            }
        }
        free(visited); free(queue);
    }
    unsigned comp_offset = 0;
    for (int tr = 0; tr < ntr; ++tr)
        for (int tc = 0; tc < ntc; ++tc) {
            orc_tile *t = &T[tr * ntc + tc];
            size_t np = (size_t)t->nr * t->nc;
            unsigned lmax = 0;
            for (size_t i = 0; i < np; ++i) if (t->cc[i] > lmax) lmax = t->cc[i];
            float padd = (float)(tk[tr * ntc + tc] * (2.0 * M_PI));
            int pr0 = tr == 0 ? 0 : rovl / 2, pc0 = tc == 0 ? 0 : covl / 2;
            int pr1 = tr == ntr - 1 ? t->nr : t->nr - rovl / 2;
            int pc1 = tc == ntc - 1 ? t->nc : t->nc - covl / 2;
            if (ntr == 1 && ntc == 1) { pr0 = pc0 = 0; pr1 = t->nr; pc1 = t->nc; }
            for (int r = pr0; r < pr1; ++r)
                for (int c = pc0; c < pc1; ++c) {
                    size_t ti = (size_t)r * t->nc + c;
                    size_t gi = (size_t)(t->r0 + r) * ncol + t->c0 + c;
                    unw[gi] = t->unw[ti] + padd;
                    cc[gi] = t->cc[ti] == 0 ? 0u : t->cc[ti] + comp_offset;
                }
            comp_offset += lmax;
        }
    if (tile_k_out) memcpy(tile_k_out, tk, nt * sizeof(double));
    for (int i = 0; i < nt; ++i) {
        free(T[i].phase); free(T[i].corr); free(T[i].unw); free(T[i].cc);
        free(T[i].mask); free(T[i].conf);
    }
    free(T); free(tk);
    return 0;
}
