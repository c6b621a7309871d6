/*
 * postpass.cu -- the reference's optional post-passes on a stitched scene,
 * as device kernels.
 *
 *  fix_cycle_spikes (cuphu_solver.cpp:1385-1441): per row, then per column,
 *    the median of the valid pixels (more than 20 of them); a line whose
 *    median differs from both neighbours' by the same nonzero whole number
 *    of cycles (within 0.5 rad) is shifted back by it.
 *      k_row_median / k_col_median   exact medians by a 4-pass radix select
 *                                    (the element std::nth_element puts at
 *                                    index size/2);
 *      k_spike_scan                  the sequential decision over lines
 *                                    (each decision updates the line's
 *                                    median, which the next line reads);
 *      k_spike_apply                 the shifts.
 *  Laplace neighbor feedback (cuphu_solver.cpp:1469-1656): per internal
 *    tile seam (column seams first, then row seams, in order), the
 *    difference of the two pixels that straddle the seam, a 21-entry moving
 *    median, gaps filled linearly (at most 84 entries) or faded to zero over
 *    42 entries, then a correction feathered into the tile interior.
 *      k_nf_sample, k_nf_median, k_nf_neighbors, k_nf_fill, k_nf_apply.
 *
 * Arithmetic: the reference's types and order, IEEE round-to-nearest per
 * operation written out with intrinsics so nvcc contracts nothing (the
 * reference's host build has no FMA contraction).
 */
#include "kernels.cuh"

#include <algorithm>

namespace cuphu {

namespace {

constexpr double kTwoPiPost = 6.283185307179586;   /* 2.0 * M_PI */
constexpr int kSmoothWin = 21;
constexpr int kMaxFill = 2 * kSmoothWin;

__device__ __forceinline__ bool pvalid(const unsigned char *mask, size_t gi)
{
    return !mask || mask[gi] != 0;
}

/* float -> key whose unsigned order is the float order (NaN aside) */
__device__ __forceinline__ uint32_t okey(float f)
{
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float okey_inv(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

/* rank-k element of one row (k = count / 2), 4 passes of 8 bits */
__global__ void __launch_bounds__(256) k_row_median(const float *__restrict__ unw,
                                                    const unsigned char *__restrict__ mask,
                                                    int nrow, int ncol, double *med,
                                                    unsigned char *have)
{
    __shared__ unsigned hist[256];
    __shared__ unsigned s_cnt, s_prefix, s_pmask, s_k;
    for (int r = blockIdx.x; r < nrow; r += gridDim.x) {
        const float *row = unw + (size_t)r * ncol;
        const unsigned char *mrow = mask ? mask + (size_t)r * ncol : nullptr;
        if (threadIdx.x == 0) { s_cnt = 0u; s_prefix = 0u; s_pmask = 0u; }
        __syncthreads();
        unsigned loc = 0u;
        for (int c = threadIdx.x; c < ncol; c += blockDim.x) loc += (!mrow || mrow[c]) ? 1u : 0u;
        atomicAdd(&s_cnt, loc);
        __syncthreads();
        const unsigned m = s_cnt;
        if (m <= 20u) {
            if (threadIdx.x == 0) { have[r] = 0; med[r] = 0.0; }
            __syncthreads();
            continue;
        }
        if (threadIdx.x == 0) s_k = m / 2u;
        for (int shift = 24; shift >= 0; shift -= 8) {
            for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0u;
            __syncthreads();
            const unsigned pre = s_prefix, pm = s_pmask;
            for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
                if (mrow && !mrow[c]) continue;
                uint32_t k = okey(row[c]);
                if ((k & pm) == pre) atomicAdd(&hist[(k >> shift) & 255u], 1u);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned k = s_k, acc = 0u;
                int b = 0;
                for (; b < 255; ++b) {
                    if (acc + hist[b] > k) break;
                    acc += hist[b];
                }
                s_k = k - acc;
                s_prefix = pre | ((unsigned)b << shift);
                s_pmask = pm | (255u << shift);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            med[r] = (double)okey_inv(s_prefix);
            have[r] = 1;
        }
        __syncthreads();
    }
}

/* the same per column, 32 columns per block (coalesced row reads) */
__global__ void __launch_bounds__(256) k_col_median(const float *__restrict__ unw,
                                                    const unsigned char *__restrict__ mask,
                                                    int nrow, int ncol, double *med,
                                                    unsigned char *have)
{
    __shared__ unsigned hist[32][257];
    __shared__ unsigned s_cnt[32], s_prefix[32], s_pmask[32], s_k[32];
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    for (int c0 = blockIdx.x * 32; c0 < ncol; c0 += gridDim.x * 32) {
        const int c = c0 + lx;
        if (threadIdx.x < 32) { s_cnt[lx] = 0u; s_prefix[lx] = 0u; s_pmask[lx] = 0u; }
        __syncthreads();
        unsigned loc = 0u;
        if (c < ncol)
            for (int r = ly; r < nrow; r += 8) loc += pvalid(mask, (size_t)r * ncol + c) ? 1u : 0u;
        atomicAdd(&s_cnt[lx], loc);
        __syncthreads();
        if (threadIdx.x < 32) s_k[lx] = s_cnt[lx] / 2u;
        for (int shift = 24; shift >= 0; shift -= 8) {
            for (int b = ly; b < 256; b += 8) hist[lx][b] = 0u;
            __syncthreads();
            const unsigned pre = s_prefix[lx], pm = s_pmask[lx];
            if (c < ncol && s_cnt[lx] > 20u)
                for (int r = ly; r < nrow; r += 8) {
                    size_t gi = (size_t)r * ncol + c;
                    if (!pvalid(mask, gi)) continue;
                    uint32_t k = okey(unw[gi]);
                    if ((k & pm) == pre) atomicAdd(&hist[lx][(k >> shift) & 255u], 1u);
                }
            __syncthreads();
            if (threadIdx.x < 32) {
                unsigned k = s_k[lx], acc = 0u;
                int b = 0;
                for (; b < 255; ++b) {
                    if (acc + hist[lx][b] > k) break;
                    acc += hist[lx][b];
                }
                s_k[lx] = k - acc;
                s_prefix[lx] = pre | ((unsigned)b << shift);
                s_pmask[lx] = pm | (255u << shift);
            }
            __syncthreads();
        }
        if (threadIdx.x < 32 && c < ncol) {
            const bool h = s_cnt[lx] > 20u;
            have[c] = h ? 1 : 0;
            med[c] = h ? (double)okey_inv(s_prefix[lx]) : 0.0;
        }
        __syncthreads();
    }
}

/* the sequential decision over lines; shift[i] = whole-cycle correction */
__global__ void k_spike_scan(double *med, const unsigned char *have, int nl, float *shift)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int i = 0; i < nl; ++i) shift[i] = 0.0f;
    for (int i = 1; i + 1 < nl; ++i) {
        if (!have[i] || !have[i - 1] || !have[i + 1]) continue;
        const double up = __dsub_rn(med[i], med[i - 1]);
        const double dn = __dsub_rn(med[i], med[i + 1]);
        const double ku = round(__ddiv_rn(up, kTwoPiPost));
        const double kd = round(__ddiv_rn(dn, kTwoPiPost));
        if (ku == 0.0 || ku != kd) continue;
        if (fabs(__dsub_rn(up, __dmul_rn(ku, kTwoPiPost))) > 0.5) continue;
        if (fabs(__dsub_rn(dn, __dmul_rn(kd, kTwoPiPost))) > 0.5) continue;
        const float corr = __double2float_rn(__dmul_rn(ku, kTwoPiPost));
        shift[i] = corr;
        med[i] = __dsub_rn(med[i], (double)corr);
    }
}

__global__ void __launch_bounds__(256) k_spike_apply(float *unw, const unsigned char *mask,
                                                     int nrow, int ncol, int by_row,
                                                     const float *shift)
{
    const long long n = (long long)nrow * ncol;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int line = by_row ? (int)(i / ncol) : (int)(i % ncol);
        const float s = shift[line];
        if (s != 0.0f && pvalid(mask, (size_t)i)) unw[i] = __fsub_rn(unw[i], s);
    }
}

/* ── neighbor feedback, one seam ──────────────────────────────────────────
 * across_cols: a vertical seam at column b (pixels (i, b-1) and (i, b),
 * correction per row i); otherwise a horizontal seam at row b. */
__device__ __forceinline__ size_t seam_px(int i, int k, int ncol, bool across_cols)
{
    return across_cols ? (size_t)i * ncol + k : (size_t)k * ncol + i;
}

__global__ void __launch_bounds__(256) k_nf_sample(const float *__restrict__ unw,
                                                   const unsigned char *__restrict__ mask,
                                                   int ncol, int n, int b, int across_cols,
                                                   double *diff, unsigned char *have)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t p0 = seam_px(i, b - 1, ncol, across_cols), p1 = seam_px(i, b, ncol, across_cols);
    const bool ok = pvalid(mask, p0) && pvalid(mask, p1);
    diff[i] = ok ? __dsub_rn((double)unw[p0], (double)unw[p1]) : 0.0;
    have[i] = ok ? 1 : 0;
}

/* moving median: the element at index size/2 of the sorted measured values
 * within +-10 entries; unmeasured entries become 0 */
__global__ void __launch_bounds__(256) k_nf_median(const double *__restrict__ x,
                                                   const unsigned char *__restrict__ have, int n,
                                                   double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!have[i]) {
        out[i] = 0.0;
        return;
    }
    double seg[kSmoothWin];
    int m = 0;
    const int lo = max(0, i - kSmoothWin / 2), hi = min(n, i + kSmoothWin / 2 + 1);
    for (int j = lo; j < hi; ++j) {
        if (!have[j]) continue;
        double v = x[j];
        int p = m++;
        while (p > 0 && seg[p - 1] > v) {
            seg[p] = seg[p - 1];
            --p;
        }
        seg[p] = v;
    }
    out[i] = seg[m / 2];
}

/* nearest measured entry at or before (prev) and at or after (next) each
 * entry; -1 / n when there is none.  One block: each thread scans a chunk,
 * the chunk ends are combined by a block-wide scan. */
__global__ void __launch_bounds__(1024) k_nf_neighbors(const unsigned char *__restrict__ have,
                                                       int n, int *prev, int *next)
{
    __shared__ int s_last[1024], s_first[1024];
    const int t = threadIdx.x, nt = blockDim.x;
    const int chunk = (n + nt - 1) / nt;
    const int a = min(n, t * chunk), b = min(n, a + chunk);
    int last = -1, first = n;
    for (int i = a; i < b; ++i)
        if (have[i]) {
            if (first == n) first = i;
            last = i;
        }
    s_last[t] = last;
    s_first[t] = first;
    __syncthreads();
    /* inclusive max-scan of last (forward) and min-scan of first (backward) */
    for (int off = 1; off < nt; off <<= 1) {
        int l = t >= off ? s_last[t - off] : -1;
        int f = t + off < nt ? s_first[t + off] : n;
        __syncthreads();
        s_last[t] = max(s_last[t], l);
        s_first[t] = min(s_first[t], f);
        __syncthreads();
    }
    int run = t > 0 ? s_last[t - 1] : -1;
    for (int i = a; i < b; ++i) {
        if (have[i]) run = i;
        prev[i] = run;
    }
    run = t + 1 < nt ? s_first[t + 1] : n;
    for (int i = b - 1; i >= a; --i) {
        if (have[i]) run = i;
        next[i] = run;
    }
}

__device__ __forceinline__ double fade_from(const double *x, int src, int i)
{
    const double w = __dsub_rn(1.0, __ddiv_rn((double)abs(i - src), (double)kMaxFill));
    return __dmul_rn(x[src], w);
}

/* gap filling: linear between measurements at most 2 * kMaxFill apart,
 * otherwise a fade to zero over kMaxFill entries from each measured side */
__global__ void __launch_bounds__(256) k_nf_fill(const double *__restrict__ x,
                                                 const unsigned char *__restrict__ have,
                                                 const int *__restrict__ prev,
                                                 const int *__restrict__ next, int n, double *out,
                                                 unsigned char *out_have)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = 0.0;
    bool h = false;
    if (have[i]) {
        v = x[i];
        h = true;
    } else {
        const int a = prev[i], b = next[i];
        if (a >= 0 && b < n) {
            const int gap = b - a;
            if (gap <= 2 * kMaxFill) {
                const double t = __ddiv_rn((double)(i - a), (double)gap);
                v = __dadd_rn(x[a], __dmul_rn(t, __dsub_rn(x[b], x[a])));
                h = true;
            } else if (i - a <= kMaxFill) {
                v = fade_from(x, a, i);
                h = true;
            } else if (b - i <= kMaxFill) {
                v = fade_from(x, b, i);
                h = true;
            }
        } else if (b < n) {
            if (b - i <= kMaxFill) { v = fade_from(x, b, i); h = true; }
        } else if (a >= 0) {
            if (i - a <= kMaxFill) { v = fade_from(x, a, i); h = true; }
        }
    }
    out[i] = v;
    out_have[i] = h ? 1 : 0;
}

/* the feathered correction: entry i of the seam, offset k - b into the
 * tile, weight 1 - (k - b) / feather (float), added as float(corr * w) */
__global__ void __launch_bounds__(256) k_nf_apply(float *unw, const unsigned char *mask, int ncol,
                                                  int n, int b, int end, int across_cols,
                                                  int feather, const double *corr,
                                                  const unsigned char *have)
{
    const int width = end - b;
    const long long tot = (long long)n * width;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = across_cols ? (int)(e / width) : (int)(e % n);
        const int k = b + (across_cols ? (int)(e % width) : (int)(e / n));
        if (!have[i]) continue;
        const size_t gi = seam_px(i, k, ncol, across_cols);
        if (!pvalid(mask, gi)) continue;
        const float w = __fsub_rn(1.0f, __fdiv_rn((float)(k - b), (float)feather));
        unw[gi] = __fadd_rn(unw[gi], __double2float_rn(__dmul_rn(corr[i], (double)w)));
    }
}

inline int blocks_for(long long n, int per = 256)
{
    return (int)std::max<long long>(1, std::min<long long>((n + per - 1) / per, 148LL * 32));
}

}  // namespace

size_t postpass_scratch_bytes(int nrow, int ncol)
{
    const size_t n = (size_t)std::max(nrow, ncol) + 16;
    /* 3 double vectors, 2 int vectors, 2 byte vectors, 1 float vector */
    return n * (3 * 8 + 2 * 4 + 2 + 4) + 256;
}

int launch_fix_cycle_spikes(float *unw, const unsigned char *mask, int nrow, int ncol,
                            void *scratch, cudaStream_t s)
{
    if (nrow < 1 || ncol < 1) return 0;
    const size_t n = (size_t)std::max(nrow, ncol) + 16;
    char *p = static_cast<char *>(scratch);
    double *med = reinterpret_cast<double *>(p);
    float *shift = reinterpret_cast<float *>(p + 3 * 8 * n);
    unsigned char *have = reinterpret_cast<unsigned char *>(p + 3 * 8 * n + 2 * 4 * n + 4 * n);
    k_row_median<<<std::min(nrow, 148 * 8), 256, 0, s>>>(unw, mask, nrow, ncol, med, have);
    k_spike_scan<<<1, 1, 0, s>>>(med, have, nrow, shift);
    k_spike_apply<<<blocks_for((long long)nrow * ncol), 256, 0, s>>>(unw, mask, nrow, ncol, 1,
                                                                     shift);
    k_col_median<<<std::min((ncol + 31) / 32, 148 * 4), 256, 0, s>>>(unw, mask, nrow, ncol, med,
                                                                     have);
    k_spike_scan<<<1, 1, 0, s>>>(med, have, ncol, shift);
    k_spike_apply<<<blocks_for((long long)nrow * ncol), 256, 0, s>>>(unw, mask, nrow, ncol, 0,
                                                                     shift);
    return cuda_fail(cudaGetLastError(), "fix_cycle_spikes kernels");
}

int launch_neighbor_feedback(float *unw, const unsigned char *mask, int nrow, int ncol, int ntr,
                             int ntc, int rovl, int covl, int feather, void *scratch,
                             cudaStream_t s)
{
    if (feather <= 0) return 0;
    const size_t n = (size_t)std::max(nrow, ncol) + 16;
    char *p = static_cast<char *>(scratch);
    double *diff = reinterpret_cast<double *>(p);
    double *smooth = diff + n;
    double *filled = smooth + n;
    int *prev = reinterpret_cast<int *>(p + 3 * 8 * n);
    int *next = prev + n;
    unsigned char *have = reinterpret_cast<unsigned char *>(p + 3 * 8 * n + 2 * 4 * n + 4 * n);
    unsigned char *have2 = have + n;
    auto seam = [&](int b, int across_cols) {
        const int len = across_cols ? nrow : ncol;
        const int lim = across_cols ? ncol : nrow;
        if (b - 1 < 0 || b + 1 >= lim) return;
        const int g = (len + 255) / 256;
        k_nf_sample<<<g, 256, 0, s>>>(unw, mask, ncol, len, b, across_cols, diff, have);
        k_nf_median<<<g, 256, 0, s>>>(diff, have, len, smooth);
        k_nf_neighbors<<<1, 1024, 0, s>>>(have, len, prev, next);
        k_nf_fill<<<g, 256, 0, s>>>(smooth, have, prev, next, len, filled, have2);
        const int end = std::min(lim, b + feather);
        k_nf_apply<<<blocks_for((long long)len * (end - b)), 256, 0, s>>>(
            unw, mask, ncol, len, b, end, across_cols, feather, filled, have2);
    };
    for (int tc = 1; tc < ntc; ++tc) seam((int)((long)tc * (ncol - covl) / ntc) + covl / 2, 1);
    for (int tr = 1; tr < ntr; ++tr) seam((int)((long)tr * (nrow - rovl) / ntr) + rovl / 2, 0);
    return cuda_fail(cudaGetLastError(), "neighbor feedback kernels");
}

}  // namespace cuphu
