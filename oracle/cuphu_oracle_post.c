/*
 * cuphu_oracle_post.c -- CPU restatement of the reference's optional
 * post-passes on a stitched scene (TEST INFRASTRUCTURE ONLY).
 *
 *   orc_fix_cycle_spikes     fix_cycle_spikes (cuphu_solver.cpp:1385-1441)
 *   orc_neighbor_feedback    apply_laplace_neighbor_feedback
 *                            (cuphu_solver.cpp:1469-1656)
 *
 * Plain IEEE arithmetic in the reference's types and order (double for the
 * medians, differences, ramps and fades, float for the pixels), compiled
 * with -ffp-contract=off like the reference's host build (no FMA
 * contraction on the default x86-64 target).  Medians are the element at
 * index size/2 of the sorted values, which is what std::nth_element places
 * there.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cuphu_oracle.h"

static int cmp_f(const void *a, const void *b)
{
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

static int cmp_d(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* one direction of the spike scan: lines are rows (by_row) or columns */
static void spikes_dir(float *unw, const unsigned char *mask, int nrow, int ncol, int by_row)
{
    const double two_pi = 2.0 * M_PI, tol = 0.5;
    const int nl = by_row ? nrow : ncol, len = by_row ? ncol : nrow;
    double *med = (double *)malloc((size_t)nl * sizeof(double));
    unsigned char *have = (unsigned char *)calloc((size_t)nl, 1);
    float *vals = (float *)malloc((size_t)len * sizeof(float));
    for (int i = 0; i < nl; ++i) {
        int m = 0;
        for (int j = 0; j < len; ++j) {
            size_t gi = by_row ? (size_t)i * ncol + j : (size_t)j * ncol + i;
            if (!mask || mask[gi]) vals[m++] = unw[gi];
        }
        med[i] = NAN;
        if (m > 20) {
            qsort(vals, (size_t)m, sizeof(float), cmp_f);
            med[i] = vals[m / 2];
            have[i] = 1;
        }
    }
    for (int i = 1; i + 1 < nl; ++i) {
        if (!have[i] || !have[i - 1] || !have[i + 1]) continue;
        double up = med[i] - med[i - 1], dn = med[i] - med[i + 1];
        double ku = round(up / two_pi), kd = round(dn / two_pi);
        if (ku == 0.0 || ku != kd) continue;
        if (fabs(up - ku * two_pi) > tol || fabs(dn - kd * two_pi) > tol) continue;
        float shift = (float)(ku * two_pi);
        for (int j = 0; j < len; ++j) {
            size_t gi = by_row ? (size_t)i * ncol + j : (size_t)j * ncol + i;
            if (!mask || mask[gi]) unw[gi] -= shift;
        }
        med[i] -= shift;
    }
    free(vals);
    free(have);
    free(med);
}

void orc_fix_cycle_spikes(float *unw, const unsigned char *mask, int nrow, int ncol)
{
    spikes_dir(unw, mask, nrow, ncol, 1);
    spikes_dir(unw, mask, nrow, ncol, 0);
}

/* moving median over the measured entries of a window of w around each
 * measured entry; unmeasured entries become 0 */
static void moving_median(double *x, const unsigned char *have, int n, int w)
{
    double *out = (double *)calloc((size_t)n, sizeof(double));
    double *seg = (double *)malloc((size_t)w * sizeof(double));
    const int half = w / 2;
    for (int i = 0; i < n; ++i) {
        if (!have[i]) continue;
        int lo = i - half < 0 ? 0 : i - half, hi = i + half + 1 > n ? n : i + half + 1, m = 0;
        for (int j = lo; j < hi; ++j)
            if (have[j]) seg[m++] = x[j];
        qsort(seg, (size_t)m, sizeof(double), cmp_d);
        out[i] = seg[m / 2];
    }
    memcpy(x, out, (size_t)n * sizeof(double));
    free(seg);
    free(out);
}

/* gaps between measurements: linear between neighbours at most 2 mf
 * apart, else a fade to zero over mf entries from each side; mf entries of
 * fade before the first and after the last measurement */
static void fill_gaps(double *x, unsigned char *have, int n, int mf)
{
    int first = -1, last = -1;
    for (int i = 0; i < n; ++i)
        if (have[i]) {
            if (first < 0) first = i;
            last = i;
        }
    if (first < 0) return;
    double *out = (double *)calloc((size_t)n, sizeof(double));
    unsigned char *oh = (unsigned char *)calloc((size_t)n, 1);
#define FADE(src, i)                                                        \
    do {                                                                    \
        double w_ = 1.0 - (double)abs((i) - (src)) / (double)mf;           \
        out[i] = x[src] * w_;                                               \
        oh[i] = 1;                                                          \
    } while (0)
    for (int i = first - mf < 0 ? 0 : first - mf; i < first; ++i) FADE(first, i);
    for (int i = last + 1; i < n && i < last + 1 + mf; ++i) FADE(last, i);
    int a = first;
    for (int b = first + 1; b <= last; ++b) {
        if (!have[b]) continue;
        int gap = b - a;
        if (gap <= 2 * mf) {
            for (int i = a + 1; i < b; ++i) {
                double t = (double)(i - a) / (double)gap;
                out[i] = x[a] + t * (x[b] - x[a]);
                oh[i] = 1;
            }
        } else {
            for (int i = a + 1; i <= a + mf; ++i) FADE(a, i);
            for (int i = b - mf; i < b; ++i) FADE(b, i);
        }
        a = b;
    }
#undef FADE
    for (int i = 0; i < n; ++i)
        if (have[i]) {
            out[i] = x[i];
            oh[i] = 1;
        }
    memcpy(x, out, (size_t)n * sizeof(double));
    memcpy(have, oh, (size_t)n);
    free(oh);
    free(out);
}

/* one internal boundary: across columns (vertical seam at column b, the
 * correction varies per row) or across rows (horizontal seam at row b) */
static void feedback_seam(float *unw, const unsigned char *mask, int nrow, int ncol, int b,
                          int across_cols, int feather)
{
    const int smooth = 21, max_fill = 2 * 21;
    const int n = across_cols ? nrow : ncol;
    const int lim = across_cols ? ncol : nrow;
    if (b - 1 < 0 || b + 1 >= lim) return;
    double *diff = (double *)calloc((size_t)n, sizeof(double));
    unsigned char *have = (unsigned char *)calloc((size_t)n, 1);
    for (int i = 0; i < n; ++i) {
        size_t p0 = across_cols ? (size_t)i * ncol + (b - 1) : (size_t)(b - 1) * ncol + i;
        size_t p1 = across_cols ? (size_t)i * ncol + b : (size_t)b * ncol + i;
        if ((mask && !mask[p0]) || (mask && !mask[p1])) continue;
        diff[i] = (double)unw[p0] - (double)unw[p1];
        have[i] = 1;
    }
    moving_median(diff, have, n, smooth);
    fill_gaps(diff, have, n, max_fill);
    const int end = b + feather < lim ? b + feather : lim;
    for (int i = 0; i < n; ++i) {
        if (!have[i]) continue;
        for (int k = b; k < end; ++k) {
            size_t gi = across_cols ? (size_t)i * ncol + k : (size_t)k * ncol + i;
            if (mask && !mask[gi]) continue;
            float w = 1.0f - (float)(k - b) / (float)feather;
            unw[gi] += (float)(diff[i] * w);
        }
    }
    free(have);
    free(diff);
}

void orc_neighbor_feedback(float *unw, const unsigned char *mask, int nrow, int ncol, int ntr,
                           int ntc, int rovl, int covl, int feather)
{
    if (feather <= 0) return;
    for (int tc = 1; tc < ntc; ++tc) {
        int b = (int)((long)tc * (ncol - covl) / ntc) + covl / 2;
        feedback_seam(unw, mask, nrow, ncol, b, 1, feather);
    }
    for (int tr = 1; tr < ntr; ++tr) {
        int b = (int)((long)tr * (nrow - rovl) / ntr) + rovl / 2;
        feedback_seam(unw, mask, nrow, ncol, b, 0, feather);
    }
}
