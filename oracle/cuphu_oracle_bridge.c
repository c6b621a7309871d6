/*
 * cuphu_oracle_bridge.c -- CPU restatement of the reference's phase bridging
 * (TEST INFRASTRUCTURE ONLY): apply_phase_bridging,
 * cuphu_solver.cpp:996-1352, with the pixel-scale stages of
 * cuphu_bridge_gpu.cu restated serially:
 *
 *  1. regions: 8-connected components of the pixels whose topology value is
 *     nonzero (masked pixels count as zero), labelled 1..N in raster order
 *     of their first pixel (cuphu_bridge_gpu.cu:29-140, 600-672);
 *  2. regions under min_num_pixel dropped, labels compacted in order
 *     (cuphu_solver.cpp:1024-1036);
 *  3. erosion survival with a square, then a circular structuring element of
 *     radius erosion_size, out-of-image counting as background; a region
 *     with no surviving pixel is dropped (cuphu_bridge_gpu.cu:150-260);
 *  4. the reference region: the largest, first in label order on ties;
 *  5. optional ramp fit over the reference region, removed before and
 *     restored after (cuphu_solver.cpp:1047-1160);
 *  6. boundary pixels: a 3x3 window (out-of-image = the centre) holding more
 *     than one label, centre labelled (cuphu_bridge_gpu.cu:262-300);
 *  7. per region the boundary pixels in raster order, every
 *     max(1, count / cap)-th up to cap (cap <= 4096) with local indices;
 *     per region pair the minimum over point pairs of the key
 *     (floor(64 * sqrtf(dx^2 + dy^2)), local p, local q)
 *     (cuphu_bridge_gpu.cu:330-520; the reference's ring search is sized to
 *     reach every cell, so its minimum is the minimum over all pairs);
 *  8. Prim's tree from the reference region (first minimum, strict updates)
 *     and a breadth-first walk of it (cuphu_solver.cpp:1170-1235);
 *  9. per bridge the medians (element size/2 of the window values in raster
 *     order, sorted) of both regions in windows of the given radius around
 *     the bridge end points, and the whole-cycle correction
 *     (cuphu_solver.cpp:1237-1330).
 * The conncomp output is overwritten with the region labels.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "cuphu_oracle.h"

static unsigned uf_root(unsigned *par, unsigned i)
{
    while (par[i] != i) {
        par[i] = par[par[i]];
        i = par[i];
    }
    return i;
}

static void uf_join(unsigned *par, unsigned a, unsigned b)
{
    a = uf_root(par, a);
    b = uf_root(par, b);
    if (a < b) par[b] = a;
    else if (b < a) par[a] = b;
}

static int label8(const float *topo, int nrow, int ncol, uint32_t *lab)
{
    const size_t n = (size_t)nrow * ncol;
    unsigned *par = (unsigned *)malloc(n * sizeof(unsigned));
    for (size_t i = 0; i < n; ++i) par[i] = (unsigned)i;
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol; ++c) {
            size_t i = (size_t)r * ncol + c;
            if (topo[i] == 0.0f) continue;
            for (int dr = -1; dr <= 1; ++dr)
                for (int dc = -1; dc <= 1; ++dc) {
                    int rr = r + dr, cc = c + dc;
                    if ((dr == 0 && dc == 0) || rr < 0 || rr >= nrow || cc < 0 || cc >= ncol)
                        continue;
                    size_t j = (size_t)rr * ncol + cc;
                    if (topo[j] != 0.0f) uf_join(par, (unsigned)i, (unsigned)j);
                }
        }
    uint32_t *rank = (uint32_t *)calloc(n, sizeof(uint32_t));
    int nl = 0;
    for (size_t i = 0; i < n; ++i)
        if (topo[i] != 0.0f && uf_root(par, (unsigned)i) == i) rank[i] = (uint32_t)++nl;
    for (size_t i = 0; i < n; ++i) lab[i] = topo[i] != 0.0f ? rank[uf_root(par, (unsigned)i)] : 0u;
    free(rank);
    free(par);
    return nl;
}

/* keep the labels with keep[l] != 0, compacted in label order */
static int remap_keep(uint32_t *lab, size_t n, int nl, const unsigned char *keep)
{
    uint32_t *m = (uint32_t *)calloc((size_t)nl + 1, sizeof(uint32_t));
    int next = 0;
    for (int l = 1; l <= nl; ++l)
        if (keep[l]) m[l] = (uint32_t)++next;
    for (size_t i = 0; i < n; ++i) lab[i] = m[lab[i]];
    free(m);
    return next;
}

static int erode_prune(uint32_t *lab, int nrow, int ncol, int nl, int e, int circular)
{
    if (e <= 0 || nl == 0) return nl;
    unsigned char *keep = (unsigned char *)calloc((size_t)nl + 1, 1);
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol; ++c) {
            uint32_t l = lab[(size_t)r * ncol + c];
            if (!l || keep[l]) continue;
            int ok = 1;
            for (int dr = -e; dr <= e && ok; ++dr)
                for (int dc = -e; dc <= e && ok; ++dc) {
                    if (circular && dr * dr + dc * dc > e * e) continue;
                    int rr = r + dr, cc = c + dc;
                    if (rr < 0 || rr >= nrow || cc < 0 || cc >= ncol ||
                        lab[(size_t)rr * ncol + cc] == 0u)
                        ok = 0;
                }
            if (ok) keep[l] = 1;
        }
    int out = remap_keep(lab, (size_t)nrow * ncol, nl, keep);
    free(keep);
    return out;
}

static int ramp_terms(int type, double r, double c, double g[6])
{
    switch (type) {
    case 1: g[0] = r; g[1] = c; g[2] = 1; return 3;
    case 2: g[0] = r * r; g[1] = c * c; g[2] = r * c; g[3] = r; g[4] = c; g[5] = 1; return 6;
    case 3: g[0] = c; g[1] = 1; return 2;
    case 4: g[0] = r; g[1] = 1; return 2;
    case 5: g[0] = c * c; g[1] = c; g[2] = 1; return 3;
    case 6: g[0] = r * r; g[1] = r; g[2] = 1; return 3;
    default: return 0;
    }
}

/* Gaussian elimination with partial pivoting on the normal equations */
static int solve_normal(double A[6][6], double b[6], int n, double x[6])
{
    for (int p = 0; p < n; ++p) {
        int piv = p;
        for (int r = p + 1; r < n; ++r)
            if (fabs(A[r][p]) > fabs(A[piv][p])) piv = r;
        if (fabs(A[piv][p]) < 1e-12) return 0;
        if (piv != p) {
            for (int c = 0; c < 6; ++c) { double t = A[piv][c]; A[piv][c] = A[p][c]; A[p][c] = t; }
            double t = b[piv]; b[piv] = b[p]; b[p] = t;
        }
        for (int r = p + 1; r < n; ++r) {
            double f = A[r][p] / A[p][p];
            for (int c = p; c < n; ++c) A[r][c] -= f * A[p][c];
            b[r] -= f * b[p];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        double s = b[r];
        for (int c = r + 1; c < n; ++c) s -= A[r][c] * x[c];
        x[r] = s / A[r][r];
    }
    return 1;
}

static void ramp_apply(float *unw, int nrow, int ncol, int type, int nt, const double *coef,
                       double sign, const unsigned char *nz)
{
    for (int r = 0; r < nrow; ++r)
        for (int c = 0; c < ncol; ++c) {
            size_t i = (size_t)r * ncol + c;
            if (!nz[i]) continue;
            double g[6], ramp = 0.0;
            ramp_terms(type, (double)r, (double)c, g);
            for (int a = 0; a < nt; ++a) ramp += coef[a] * g[a];
            unw[i] += (float)(sign * ramp);
        }
}

static int cmp_f(const void *a, const void *b)
{
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

static int window_median(const float *unw, const uint32_t *lab, int nrow, int ncol, int cy, int cx,
                         int radius, uint32_t id, float *buf, double *out)
{
    int r0 = cy - radius < 0 ? 0 : cy - radius, r1 = cy + radius + 1 > nrow ? nrow : cy + radius + 1;
    int c0 = cx - radius < 0 ? 0 : cx - radius, c1 = cx + radius + 1 > ncol ? ncol : cx + radius + 1;
    size_t m = 0;
    for (int r = r0; r < r1; ++r)
        for (int c = c0; c < c1; ++c) {
            size_t i = (size_t)r * ncol + c;
            if (lab[i] == id) buf[m++] = unw[i];
        }
    if (!m) return 0;
    qsort(buf, m, sizeof(float), cmp_f);
    *out = buf[m / 2];
    return 1;
}

int orc_bridge(float *unw, uint32_t *conncomp, int nrow, int ncol, const unsigned char *mask,
               int radius, int min_num_pixel, int erosion_size, int max_boundary_samples,
               int ramp_type, int ramp_max_num_sample)
{
    const size_t n = (size_t)nrow * ncol;
    float *topo = (float *)malloc(n * sizeof(float));
    for (size_t i = 0; i < n; ++i) topo[i] = (mask && !mask[i]) ? 0.0f : unw[i];
    uint32_t *lab = (uint32_t *)malloc(n * sizeof(uint32_t));
    int nl = label8(topo, nrow, ncol, lab);
    free(topo);
    int ret = 0;
    if (nl <= 1) goto done;
    {
        int *cnt = (int *)calloc((size_t)nl + 1, sizeof(int));
        for (size_t i = 0; i < n; ++i) cnt[lab[i]]++;
        unsigned char *keep = (unsigned char *)calloc((size_t)nl + 1, 1);
        for (int l = 1; l <= nl; ++l) keep[l] = cnt[l] >= min_num_pixel;
        nl = remap_keep(lab, n, nl, keep);
        free(keep);
        free(cnt);
    }
    if (nl <= 1) goto done;
    nl = erode_prune(lab, nrow, ncol, nl, erosion_size, 0);
    if (nl <= 1) goto done;
    nl = erode_prune(lab, nrow, ncol, nl, erosion_size, 1);
    if (nl <= 1) goto done;
    {
        const int n1 = nl + 1;
        int *cnt = (int *)calloc((size_t)n1, sizeof(int));
        for (size_t i = 0; i < n; ++i) cnt[lab[i]]++;
        int ref = 1;
        for (int l = 2; l <= nl; ++l)
            if (cnt[l] > cnt[ref]) ref = l;
        free(cnt);
        /* ramp over the reference region */
        int nt = 0, ramp_ok = 0;
        double coef[6] = {0, 0, 0, 0, 0, 0};
        unsigned char *nz = NULL;
        if (ramp_type != 0) {
            double dummy[6];
            nt = ramp_terms(ramp_type, 0, 0, dummy);
            size_t count = 0;
            for (size_t i = 0; i < n; ++i) count += lab[i] == (uint32_t)ref && unw[i] != 0.0f;
            if (count) {
                int step = 1;
                if (ramp_max_num_sample > 0 && (long)count > ramp_max_num_sample)
                    step = (int)ceil(sqrt((double)count / ramp_max_num_sample));
                int half = step / 2;
                double A[6][6] = {{0}}, b[6] = {0};
                for (int r = 0; r < nrow; ++r) {
                    if (step > 1 && r % step != half) continue;
                    for (int c = 0; c < ncol; ++c) {
                        if (step > 1 && c % step != half) continue;
                        size_t i = (size_t)r * ncol + c;
                        if (lab[i] != (uint32_t)ref || unw[i] == 0.0f) continue;
                        double g[6];
                        ramp_terms(ramp_type, (double)r, (double)c, g);
                        for (int a = 0; a < nt; ++a) {
                            b[a] += g[a] * (double)unw[i];
                            for (int bb = 0; bb < nt; ++bb) A[a][bb] += g[a] * g[bb];
                        }
                    }
                }
                ramp_ok = solve_normal(A, b, nt, coef);
            }
            if (ramp_ok) {
                nz = (unsigned char *)malloc(n);
                for (size_t i = 0; i < n; ++i) nz[i] = unw[i] != 0.0f;
                ramp_apply(unw, nrow, ncol, ramp_type, nt, coef, -1.0, nz);
            }
        }
        /* boundary points per region, subsampled */
        int cap = max_boundary_samples > 4096 ? 4096 : max_boundary_samples;
        int *bcnt = (int *)calloc((size_t)n1, sizeof(int));
        unsigned char *bnd = (unsigned char *)calloc(n, 1);
        for (int r = 0; r < nrow; ++r)
            for (int c = 0; c < ncol; ++c) {
                size_t i = (size_t)r * ncol + c;
                uint32_t ce = lab[i], mx = ce, mn = ce;
                for (int dr = -1; dr <= 1; ++dr)
                    for (int dc = -1; dc <= 1; ++dc) {
                        int rr = r + dr, cc = c + dc;
                        uint32_t v = (rr < 0 || rr >= nrow || cc < 0 || cc >= ncol)
                                         ? ce : lab[(size_t)rr * ncol + cc];
                        if (v > mx) mx = v;
                        if (v < mn) mn = v;
                    }
                bnd[i] = mx != mn && ce > 0;
                if (bnd[i]) bcnt[ce]++;
            }
        int **py = (int **)calloc((size_t)n1, sizeof(int *)), **px = (int **)calloc((size_t)n1, sizeof(int *));
        int *np = (int *)calloc((size_t)n1, sizeof(int)), *seen = (int *)calloc((size_t)n1, sizeof(int));
        for (int l = 1; l <= nl; ++l) {
            int k = bcnt[l] < cap ? bcnt[l] : cap;
            py[l] = (int *)malloc((size_t)(k + 1) * sizeof(int));
            px[l] = (int *)malloc((size_t)(k + 1) * sizeof(int));
        }
        for (int r = 0; r < nrow; ++r)
            for (int c = 0; c < ncol; ++c) {
                size_t i = (size_t)r * ncol + c;
                if (!bnd[i]) continue;
                int l = (int)lab[i];
                int stride = bcnt[l] / cap > 1 ? bcnt[l] / cap : 1;
                int k = seen[l]++;
                if (k % stride == 0 && np[l] < cap) {
                    py[l][np[l]] = r;
                    px[l][np[l]] = c;
                    np[l]++;
                }
            }
        free(seen);
        free(bnd);
        free(bcnt);
        uint64_t *key = (uint64_t *)malloc((size_t)n1 * n1 * sizeof(uint64_t));
        for (size_t i = 0; i < (size_t)n1 * n1; ++i) key[i] = ~0ull;
        for (int a = 1; a <= nl; ++a)
            for (int b = 1; b <= nl; ++b) {
                if (a == b) continue;
                uint64_t best = ~0ull;
                for (int p = 0; p < np[a]; ++p)
                    for (int q = 0; q < np[b]; ++q) {
                        float dx = (float)(px[b][q] - px[a][p]), dy = (float)(py[b][q] - py[a][p]);
                        float d = sqrtf(dx * dx + dy * dy);
                        uint64_t k = ((uint64_t)(d * 64.0f) << 24) | ((uint64_t)p << 12) | (uint64_t)q;
                        if (k < best) best = k;
                    }
                key[(size_t)a * n1 + b] = best;
            }
        /* Prim from the reference region, then a breadth-first walk */
        float *bd = (float *)malloc((size_t)n1 * sizeof(float));
        int *bp = (int *)malloc((size_t)n1 * sizeof(int));
        unsigned char *in = (unsigned char *)calloc((size_t)n1, 1);
        int *ep = (int *)malloc((size_t)2 * nl * sizeof(int)), ne = 0;
#define DIST(i, j) (key[(size_t)(i) * n1 + (j)] == ~0ull ? INFINITY \
                    : (float)(key[(size_t)(i) * n1 + (j)] >> 24) / 64.0f)
        in[ref] = 1;
        for (int j = 1; j <= nl; ++j) {
            bd[j] = j == ref ? INFINITY : DIST(ref, j);
            bp[j] = ref;
        }
        for (int it = 1; it < nl; ++it) {
            int u = -1;
            float ud = INFINITY;
            for (int j = 1; j <= nl; ++j)
                if (!in[j] && bd[j] < ud) { ud = bd[j]; u = j; }
            if (u < 0) break;
            in[u] = 1;
            ep[2 * ne] = bp[u];
            ep[2 * ne + 1] = u;
            ne++;
            for (int j = 1; j <= nl; ++j)
                if (!in[j] && DIST(u, j) < bd[j]) { bd[j] = DIST(u, j); bp[j] = u; }
        }
#undef DIST
        /* adjacency in edge order, then the walk */
        int *deg = (int *)calloc((size_t)n1, sizeof(int));
        for (int e = 0; e < ne; ++e) { deg[ep[2 * e]]++; deg[ep[2 * e + 1]]++; }
        int *off = (int *)calloc((size_t)n1 + 1, sizeof(int));
        for (int l = 1; l <= nl; ++l) off[l + 1] = off[l] + deg[l];
        int *adj = (int *)malloc((size_t)(2 * ne + 1) * sizeof(int));
        int *fill = (int *)calloc((size_t)n1, sizeof(int));
        for (int e = 0; e < ne; ++e) {
            int a = ep[2 * e], b = ep[2 * e + 1];
            adj[off[a] + fill[a]++] = b;
            adj[off[b] + fill[b]++] = a;
        }
        double *corr = (double *)calloc((size_t)n1, sizeof(double));
        int *queue = (int *)malloc((size_t)n1 * sizeof(int)), qh = 0, qt = 0;
        unsigned char *vis = (unsigned char *)calloc((size_t)n1, 1);
        int rad = radius < (nrow < ncol ? nrow : ncol) / 2 ? radius : (nrow < ncol ? nrow : ncol) / 2;
        float *buf = (float *)malloc((size_t)(2 * rad + 1) * (2 * rad + 1) * sizeof(float) + 4);
        queue[qt++] = ref;
        vis[ref] = 1;
        while (qh < qt) {
            int u = queue[qh++];
            for (int k = off[u]; k < off[u + 1]; ++k) {
                int v = adj[k];
                if (vis[v]) continue;
                vis[v] = 1;
                queue[qt++] = v;
                uint64_t kk = key[(size_t)u * n1 + v];
                int p = (int)((kk >> 12) & 4095u), q = (int)(kk & 4095u);
                double m0, m1;
                int ok0 = window_median(unw, lab, nrow, ncol, py[u][p], px[u][p], rad, (uint32_t)u,
                                        buf, &m0);
                int ok1 = window_median(unw, lab, nrow, ncol, py[v][q], px[v][q], rad, (uint32_t)v,
                                        buf, &m1);
                if (!ok0 || !ok1) continue;
                double diff = m1 - (m0 + corr[u]);
                double jump = floor((fabs(diff) + M_PI) / (2.0 * M_PI));
                if (diff > 0) jump *= -1.0;
                corr[v] = jump * (2.0 * M_PI);
            }
        }
        for (size_t i = 0; i < n; ++i) {
            uint32_t l = lab[i];
            conncomp[i] = l;
            if (l) unw[i] += (float)corr[l];
        }
        if (ramp_ok) ramp_apply(unw, nrow, ncol, ramp_type, nt, coef, 1.0, nz);
        ret = nl;
        free(buf); free(vis); free(queue); free(corr); free(fill); free(adj); free(off);
        free(deg); free(ep); free(in); free(bp); free(bd); free(key);
        for (int l = 1; l <= nl; ++l) { free(py[l]); free(px[l]); }
        free(py); free(px); free(np);
        free(nz);
    }
done:
    free(lab);
    return ret;
}
