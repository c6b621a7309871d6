/*
 * bridge.cu -- phase bridging on the device: the reference's
 * apply_phase_bridging (cuphu_solver.cpp:996-1352, with the pixel-scale
 * stages of cuphu_bridge_gpu.cu), which reconciles whole-cycle offsets
 * between regions of a stitched scene that a mask or zero-valued pixels
 * split apart.
 *
 * Pixel-scale work runs as kernels: union-find labelling of the 8-connected
 * nonzero pixels (labels in raster order of each region's first pixel, as
 * the reference's min-label propagation ends), size pruning, the erosion
 * survival tests, boundary extraction, compaction of the boundary pixels in
 * raster order, the all-pairs nearest-boundary search (the reference's packed
 * key: quantised distance, then the two points' indices), the window
 * medians of every bridge end and the final correction.  Region-scale steps
 * -- the reference region, the ramp fit, Prim's tree and its walk, the
 * cycle arithmetic per bridge -- are small and sequential, and run on the
 * host over copied-back region tables, as in the reference.
 *
 * Exactness: integer and selection stages are exact; the distances are
 * sqrtf(dx*dx + dy*dy) rounded per operation (exact inputs while |dx|, |dy|
 * < 4096); the ramp fit is the reference's sequential double accumulation
 * on the host; the ramp and the corrections are applied per pixel in the
 * reference's operation order.
 */
#include "kernels.cuh"

#include <algorithm>
#include <cmath>
#include <queue>
#include <vector>

namespace cuphu {
namespace {

constexpr uint32_t kNone = 0xffffffffu;
constexpr int kIdxBits = 12;                 /* 4096 boundary samples per region */

__global__ void k_br_init(const float *__restrict__ unw, const unsigned char *__restrict__ mask,
                          long long n, uint32_t *par)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const bool v = unw[i] != 0.0f && (!mask || mask[i] != 0);
        par[i] = v ? (uint32_t)i : kNone;
    }
}

__device__ __forceinline__ uint32_t uf_find(const uint32_t *par, uint32_t p)
{
    uint32_t q = __ldcg(par + p);
    while (q != p) {
        p = q;
        q = __ldcg(par + p);
    }
    return p;
}

/* hook the larger root under the smaller one */
__device__ __forceinline__ void uf_union(uint32_t *par, uint32_t a, uint32_t b)
{
    for (int guard = 0; guard < (1 << 20); ++guard) {
        a = uf_find(par, a);
        b = uf_find(par, b);
        if (a == b) return;
        if (a > b) {
            uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicCAS(par + b, b, a);
        if (old == b) return;
        b = old;
    }
}

/* unions with the 4 neighbours after the pixel in raster order that an
 * 8-neighbourhood touches: right, down-left, down, down-right */
__global__ void k_br_union(uint32_t *par, int nrow, int ncol)
{
    const long long n = (long long)nrow * ncol;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (__ldcg(par + i) == kNone) continue;
        const int r = (int)(i / ncol), c = (int)(i % ncol);
        const int dr[4] = {0, 1, 1, 1}, dc[4] = {1, -1, 0, 1};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int rr = r + dr[k], cc = c + dc[k];
            if (rr >= nrow || cc < 0 || cc >= ncol) continue;
            const long long j = (long long)rr * ncol + cc;
            if (__ldcg(par + j) != kNone) uf_union(par, (uint32_t)i, (uint32_t)j);
        }
    }
}

__global__ void k_br_flatten(uint32_t *par, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (par[i] != kNone) par[i] = uf_find(par, (uint32_t)i);
}

/* ── raster-order ranks of flagged elements: per-chunk counts, a scan of
 *    the chunk counts, then per-chunk local ranks ───────────────────────── */
constexpr int kScanChunk = 4096;

template <typename Pred>
__global__ void __launch_bounds__(256) k_chunk_count(long long n, Pred pred, unsigned *sums)
{
    __shared__ unsigned s;
    if (threadIdx.x == 0) s = 0u;
    __syncthreads();
    const long long a = (long long)blockIdx.x * kScanChunk;
    const long long b = min(n, a + kScanChunk);
    unsigned loc = 0u;
    for (long long i = a + threadIdx.x; i < b; i += blockDim.x) loc += pred(i) ? 1u : 0u;
    atomicAdd(&s, loc);
    __syncthreads();
    if (threadIdx.x == 0) sums[blockIdx.x] = s;
}

/* exclusive scan of m values in place (one block); total in sums[m] */
__global__ void __launch_bounds__(1024) k_scan_sums(unsigned *sums, int m)
{
    __shared__ unsigned part[1024];
    const int t = threadIdx.x, nt = blockDim.x;
    const int per = (m + nt - 1) / nt;
    const int a = min(m, t * per), b = min(m, a + per);
    unsigned loc = 0u;
    for (int i = a; i < b; ++i) loc += sums[i];
    part[t] = loc;
    __syncthreads();
    for (int off = 1; off < nt; off <<= 1) {
        unsigned v = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    unsigned run = t > 0 ? part[t - 1] : 0u;
    for (int i = a; i < b; ++i) {
        unsigned v = sums[i];
        sums[i] = run;
        run += v;
    }
    if (t == nt - 1) sums[m] = part[nt - 1];
}

/* rank of every flagged element within the chunk order; out(i, rank) */
template <typename Pred, typename Out>
__global__ void __launch_bounds__(256) k_chunk_rank(long long n, Pred pred, const unsigned *sums,
                                                    Out out)
{
    __shared__ unsigned warp_tot[8];
    __shared__ unsigned base;
    const long long a = (long long)blockIdx.x * kScanChunk;
    const long long b = min(n, a + kScanChunk);
    if (threadIdx.x == 0) base = sums[blockIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (long long s0 = a; s0 < b; s0 += blockDim.x) {
        const long long i = s0 + threadIdx.x;
        const bool f = i < b && pred(i);
        const unsigned m = __ballot_sync(0xffffffffu, f);
        const unsigned before = __popc(m & ((1u << lane) - 1u));
        if (lane == 0) warp_tot[w] = __popc(m);
        __syncthreads();
        unsigned wb = 0u;
        for (int k = 0; k < w; ++k) wb += warp_tot[k];
        if (f) out(i, base + wb + before);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned tot = 0u;
            for (int k = 0; k < 8; ++k) tot += warp_tot[k];
            base += tot;
        }
        __syncthreads();
    }
}

struct IsRoot {
    const uint32_t *par;
    __device__ bool operator()(long long i) const { return par[i] == (uint32_t)i; }
};
struct PutRootRank {
    uint32_t *rank;
    __device__ void operator()(long long i, unsigned r) const { rank[i] = r + 1u; }
};

/* label of each pixel: the rank of its root (roots ordered by index) */
__global__ void k_br_label(const uint32_t *par, const uint32_t *rootrank, long long n,
                           uint32_t *lab)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t p = par[i];
        lab[i] = p == kNone ? 0u : rootrank[p];
    }
}

__global__ void k_br_count(const uint32_t *lab, long long n, unsigned *cnt)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (lab[i]) atomicAdd(cnt + lab[i], 1u);
}

/* erosion survival (a structuring element of radius e, square or circular;
 * out-of-image counts as background): marks the labels with a survivor */
__global__ void k_br_erode(const uint32_t *lab, int nrow, int ncol, int e, int circular,
                           unsigned char *survive)
{
    const long long n = (long long)nrow * ncol;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t l = lab[i];
        if (!l) continue;
        const int r = (int)(i / ncol), c = (int)(i % ncol);
        bool ok = r - e >= 0 && r + e < nrow && c - e >= 0 && c + e < ncol;
        for (int dr = -e; dr <= e && ok; ++dr)
            for (int dc = -e; dc <= e && ok; ++dc) {
                if (circular && dr * dr + dc * dc > e * e) continue;
                if (lab[(long long)(r + dr) * ncol + (c + dc)] == 0u) ok = false;
            }
        if (ok) survive[l] = 1;
    }
}

__global__ void k_br_remap(uint32_t *lab, long long n, const uint32_t *remap)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        lab[i] = remap[lab[i]];
}

/* boundary: a 3x3 window (out-of-image = the centre) holding more than one
 * label value, centre labelled */
struct IsBoundary {
    const uint32_t *lab;
    int nrow, ncol;
    __device__ bool operator()(long long i) const
    {
        const uint32_t ce = lab[i];
        if (!ce) return false;
        const int r = (int)(i / ncol), c = (int)(i % ncol);
        uint32_t mx = ce, mn = ce;
        for (int dr = -1; dr <= 1; ++dr)
            for (int dc = -1; dc <= 1; ++dc) {
                const int rr = r + dr, cc = c + dc;
                const uint32_t v = (rr < 0 || rr >= nrow || cc < 0 || cc >= ncol)
                                       ? ce : lab[(long long)rr * ncol + cc];
                mx = max(mx, v);
                mn = min(mn, v);
            }
        return mx != mn;
    }
};
struct PutIndex {
    uint32_t *idx;
    __device__ void operator()(long long i, unsigned r) const { idx[r] = (uint32_t)i; }
};

/* the nearest boundary pair of every ordered region pair: one thread per
 * sampled point p (region a), one minimum per other region, one atomicMin
 * of the packed key (64 d quantised, local index of p, local index of q) */
__global__ void __launch_bounds__(256) k_br_nn(const int *py, const int *px, const int *plab,
                                               const int *ploc, int np, const int *seg, int nl,
                                               unsigned long long *key)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const int a = plab[p], yp = py[p], xp = px[p];
    const unsigned long long lp = (unsigned long long)ploc[p];
    for (int b = 1; b <= nl; ++b) {
        if (b == a) continue;
        unsigned long long best = ~0ull;
        for (int q = seg[b]; q < seg[b + 1]; ++q) {
            const float dx = (float)(px[q] - xp), dy = (float)(py[q] - yp);
            const float d = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
            const unsigned long long k = ((unsigned long long)__fmul_rn(d, 64.0f) << (2 * kIdxBits)) |
                                         (lp << kIdxBits) | (unsigned long long)ploc[q];
            best = k < best ? k : best;
        }
        if (best != ~0ull) atomicMin(key + (size_t)a * (nl + 1) + b, best);
    }
}

/* the median (element m/2 of the sorted values) of the pixels labelled id
 * in a window; one block per request, 4-pass radix select */
__device__ __forceinline__ uint32_t okey_b(float f)
{
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float okey_b_inv(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void __launch_bounds__(256) k_br_median(const float *unw, const uint32_t *lab, int ncol,
                                                   const int4 *req, const uint32_t *rid,
                                                   double *med, int *ok)
{
    __shared__ unsigned hist[256];
    __shared__ unsigned s_cnt, s_pre, s_pm, s_k;
    const int4 w = req[blockIdx.x];          /* r0, r1, c0, c1 */
    const uint32_t id = rid[blockIdx.x];
    const int wc = w.w - w.z;
    const long long tot = (long long)(w.y - w.x) * wc;
    if (threadIdx.x == 0) { s_cnt = 0u; s_pre = 0u; s_pm = 0u; }
    __syncthreads();
    unsigned loc = 0u;
    for (long long e = threadIdx.x; e < tot; e += blockDim.x) {
        const long long i = (long long)(w.x + e / wc) * ncol + (w.z + e % wc);
        loc += lab[i] == id ? 1u : 0u;
    }
    atomicAdd(&s_cnt, loc);
    __syncthreads();
    if (s_cnt == 0u) {
        if (threadIdx.x == 0) { ok[blockIdx.x] = 0; med[blockIdx.x] = 0.0; }
        return;
    }
    if (threadIdx.x == 0) s_k = s_cnt / 2u;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int bn = threadIdx.x; bn < 256; bn += blockDim.x) hist[bn] = 0u;
        __syncthreads();
        const unsigned pre = s_pre, pm = s_pm;
        for (long long e = threadIdx.x; e < tot; e += blockDim.x) {
            const long long i = (long long)(w.x + e / wc) * ncol + (w.z + e % wc);
            if (lab[i] != id) continue;
            const uint32_t k = okey_b(unw[i]);
            if ((k & pm) == pre) atomicAdd(&hist[(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned k = s_k, acc = 0u;
            int bn = 0;
            for (; bn < 255; ++bn) {
                if (acc + hist[bn] > k) break;
                acc += hist[bn];
            }
            s_k = k - acc;
            s_pre = pre | ((unsigned)bn << shift);
            s_pm = pm | (255u << shift);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ok[blockIdx.x] = 1;
        med[blockIdx.x] = (double)okey_b_inv(s_pre);
    }
}

__global__ void k_br_gather(const uint32_t *lab, const uint32_t *idx, unsigned nb, uint32_t *out)
{
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x)
        out[k] = lab[idx[k]];
}

__global__ void k_br_apply(float *unw, uint32_t *cc, const uint32_t *lab, long long n,
                           const double *corr)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t l = lab[i];
        cc[i] = l;
        if (l) unw[i] = __fadd_rn(unw[i], __double2float_rn(corr[l]));
    }
}

/* ramp terms at (r, c) (cuphu_solver.cpp:1056-1073) */
__host__ __device__ inline int ramp_terms(int type, double r, double c, double g[6])
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

struct Ramp {
    int type, nt;
    double coef[6];
};

/* unw += float(sign * ramp) where the original value was nonzero */
__global__ void k_br_ramp(float *unw, const unsigned char *nz, int nrow, int ncol, Ramp R,
                          double sign)
{
    const long long n = (long long)nrow * ncol;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (!nz[i]) continue;
        double g[6], ramp = 0.0;
        ramp_terms(R.type, (double)(i / ncol), (double)(i % ncol), g);
        for (int a = 0; a < R.nt; ++a) ramp = __dadd_rn(ramp, __dmul_rn(R.coef[a], g[a]));
        unw[i] = __fadd_rn(unw[i], __double2float_rn(sign * ramp));
    }
}

__global__ void k_br_nonzero(const float *unw, long long n, unsigned char *nz)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        nz[i] = unw[i] != 0.0f;
}

inline int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 32)); }

/* normal equations in the reference's sequential order (host) */
bool fit_ramp_host(const std::vector<float> &unw, const std::vector<uint32_t> &lab, int nrow,
                   int ncol, uint32_t ref, int type, int max_sample, Ramp &R)
{
    double dummy[6];
    R.type = type;
    R.nt = ramp_terms(type, 0, 0, dummy);
    size_t count = 0;
    for (size_t i = 0; i < unw.size(); ++i) count += lab[i] == ref && unw[i] != 0.0f;
    if (!count) return false;
    int step = 1;
    if (max_sample > 0 && (long)count > max_sample)
        step = (int)std::ceil(std::sqrt((double)count / max_sample));
    const int half = step / 2;
    double A[6][6] = {{0}}, b[6] = {0};
    for (int r = 0; r < nrow; ++r) {
        if (step > 1 && r % step != half) continue;
        for (int c = 0; c < ncol; ++c) {
            if (step > 1 && c % step != half) continue;
            size_t i = (size_t)r * ncol + c;
            if (lab[i] != ref || unw[i] == 0.0f) continue;
            double g[6];
            ramp_terms(type, (double)r, (double)c, g);
            for (int a = 0; a < R.nt; ++a) {
                b[a] += g[a] * (double)unw[i];
                for (int bb = 0; bb < R.nt; ++bb) A[a][bb] += g[a] * g[bb];
            }
        }
    }
    const int n = R.nt;
    for (int p = 0; p < n; ++p) {
        int piv = p;
        for (int r = p + 1; r < n; ++r)
            if (std::fabs(A[r][p]) > std::fabs(A[piv][p])) piv = r;
        if (std::fabs(A[piv][p]) < 1e-12) return false;
        if (piv != p) {
            std::swap(A[piv], A[p]);
            std::swap(b[piv], b[p]);
        }
        for (int r = p + 1; r < n; ++r) {
            double f = A[r][p] / A[p][p];
            for (int c = p; c < n; ++c) A[r][c] -= f * A[p][c];
            b[r] -= f * b[p];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        double s = b[r];
        for (int c = r + 1; c < n; ++c) s -= A[r][c] * R.coef[c];
        R.coef[r] = s / A[r][r];
    }
    return true;
}

}  // namespace

/* Scratch from the caller's stream (stream-ordered allocations, freed on
 * return); copies of region-scale tables synchronise the stream. */
int run_bridge(float *unw, uint32_t *cc, const unsigned char *mask, int nrow, int ncol,
               const CuPhuBridgeParams &bp, cudaStream_t s)
{
    const long long n = (long long)nrow * ncol;
    if (n < 2) return 0;
    std::vector<void *> owned;
    auto take = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMallocAsync(&p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        owned.push_back(p);
        return p;
    };
    struct Free {
        std::vector<void *> &v;
        cudaStream_t s;
        ~Free() { for (void *p : v) cudaFreeAsync(p, s); }
    } guard{owned, s};
    const int nchunk = (int)((n + kScanChunk - 1) / kScanChunk);
    uint32_t *par = (uint32_t *)take(n * 4), *lab = (uint32_t *)take(n * 4);
    uint32_t *rank = (uint32_t *)take(n * 4);
    unsigned *sums = (unsigned *)take((size_t)(nchunk + 1) * 4);
    if (!par || !lab || !rank || !sums) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
    const int g = grid_for(n);

    /* 1. regions of the nonzero, unmasked pixels */
    k_br_init<<<g, 256, 0, s>>>(unw, mask, n, par);
    k_br_union<<<g, 256, 0, s>>>(par, nrow, ncol);
    k_br_flatten<<<g, 256, 0, s>>>(par, n);
    k_chunk_count<<<nchunk, 256, 0, s>>>(n, IsRoot{par}, sums);
    k_scan_sums<<<1, 1024, 0, s>>>(sums, nchunk);
    k_chunk_rank<<<nchunk, 256, 0, s>>>(n, IsRoot{par}, sums, PutRootRank{rank});
    k_br_label<<<g, 256, 0, s>>>(par, rank, n, lab);
    unsigned nl = 0;
    CUPHU_TRY_CUDA(cudaMemcpyAsync(&nl, sums + nchunk, 4, cudaMemcpyDeviceToHost, s));
    CUPHU_TRY_CUDA(cudaStreamSynchronize(s));
    if (nl <= 1) return 0;

    /* 2-3. size pruning, then the two erosion survival tests; every stage
     * compacts the surviving labels in order */
    std::vector<unsigned> cnt;
    auto counts = [&](unsigned nlab) -> int {
        unsigned *d = (unsigned *)take((size_t)(nlab + 1) * 4);
        if (!d) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
        CUPHU_TRY_CUDA(cudaMemsetAsync(d, 0, (size_t)(nlab + 1) * 4, s));
        k_br_count<<<g, 256, 0, s>>>(lab, n, d);
        cnt.assign(nlab + 1, 0u);
        CUPHU_TRY_CUDA(cudaMemcpyAsync(cnt.data(), d, (size_t)(nlab + 1) * 4,
                                       cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaStreamSynchronize(s));
        return 0;
    };
    auto keep_only = [&](unsigned nlab, const std::vector<unsigned char> &keep,
                         unsigned &out) -> int {
        std::vector<uint32_t> remap(nlab + 1, 0u);
        unsigned next = 0;
        for (unsigned l = 1; l <= nlab; ++l)
            if (keep[l]) remap[l] = ++next;
        uint32_t *d = (uint32_t *)take((size_t)(nlab + 1) * 4);
        if (!d) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d, remap.data(), (size_t)(nlab + 1) * 4,
                                       cudaMemcpyHostToDevice, s));
        k_br_remap<<<g, 256, 0, s>>>(lab, n, d);
        CUPHU_TRY_CUDA(cudaStreamSynchronize(s));   /* the host table outlives the copy */
        out = next;
        return 0;
    };
    int rc = counts(nl);
    if (rc) return rc;
    {
        std::vector<unsigned char> keep(nl + 1, 0);
        for (unsigned l = 1; l <= nl; ++l) keep[l] = (long)cnt[l] >= (long)bp.min_num_pixel;
        if ((rc = keep_only(nl, keep, nl))) return rc;
    }
    if (nl <= 1) return 0;
    for (int circular = 0; circular < 2 && bp.erosion_size > 0; ++circular) {
        unsigned char *d = (unsigned char *)take(nl + 1);
        if (!d) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
        CUPHU_TRY_CUDA(cudaMemsetAsync(d, 0, nl + 1, s));
        k_br_erode<<<g, 256, 0, s>>>(lab, nrow, ncol, bp.erosion_size, circular, d);
        std::vector<unsigned char> keep(nl + 1, 0);
        CUPHU_TRY_CUDA(cudaMemcpyAsync(keep.data(), d, nl + 1, cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaStreamSynchronize(s));
        if ((rc = keep_only(nl, keep, nl))) return rc;
        if (nl <= 1) return 0;
    }

    /* 4. the reference region: the largest, first in label order */
    if ((rc = counts(nl))) return rc;
    uint32_t ref = 1;
    for (unsigned l = 2; l <= nl; ++l)
        if (cnt[l] > cnt[ref]) ref = l;

    /* 5. optional ramp over the reference region (host fit, as the
     * reference), removed before and restored after */
    Ramp R = {};
    bool ramp_ok = false;
    unsigned char *nz = nullptr;
    if (bp.ramp_type != CUPHU_RAMP_NONE) {
        std::vector<float> hu(n);
        std::vector<uint32_t> hl(n);
        CUPHU_TRY_CUDA(cudaMemcpyAsync(hu.data(), unw, n * 4, cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(hl.data(), lab, n * 4, cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaStreamSynchronize(s));
        ramp_ok = fit_ramp_host(hu, hl, nrow, ncol, ref, (int)bp.ramp_type,
                                bp.ramp_max_num_sample, R);
        if (ramp_ok) {
            nz = (unsigned char *)take(n);
            if (!nz) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
            k_br_nonzero<<<g, 256, 0, s>>>(unw, n, nz);
            k_br_ramp<<<g, 256, 0, s>>>(unw, nz, nrow, ncol, R, -1.0);
        }
    }

    /* 6-7. boundary pixels in raster order, sampled per region */
    IsBoundary isb{lab, nrow, ncol};
    k_chunk_count<<<nchunk, 256, 0, s>>>(n, isb, sums);
    k_scan_sums<<<1, 1024, 0, s>>>(sums, nchunk);
    unsigned nb = 0;
    CUPHU_TRY_CUDA(cudaMemcpyAsync(&nb, sums + nchunk, 4, cudaMemcpyDeviceToHost, s));
    CUPHU_TRY_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> bidx(nb), blab(nb);
    if (nb) {
        uint32_t *d_bidx = (uint32_t *)take((size_t)nb * 8);
        if (!d_bidx) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
        k_chunk_rank<<<nchunk, 256, 0, s>>>(n, isb, sums, PutIndex{d_bidx});
        k_br_gather<<<grid_for(nb), 256, 0, s>>>(lab, d_bidx, nb, d_bidx + nb);
        CUPHU_TRY_CUDA(cudaMemcpyAsync(bidx.data(), d_bidx, (size_t)nb * 4, cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(blab.data(), d_bidx + nb, (size_t)nb * 4,
                                       cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaStreamSynchronize(s));
    }
    const int cap = std::min(bp.max_boundary_samples, 1 << kIdxBits);
    if (cap < 1) return fail(CUPHU_ERR_INVALID, "bridge max_boundary_samples must be >= 1");
    std::vector<unsigned> bcnt(nl + 1, 0u);
    for (unsigned k = 0; k < nb; ++k) bcnt[blab[k]]++;
    std::vector<int> seg(nl + 2, 0);
    for (unsigned l = 1; l <= nl; ++l) seg[l + 1] = seg[l] + (int)std::min<unsigned>(bcnt[l], cap);
    const int np = seg[nl + 1];
    std::vector<int> hpy(np), hpx(np), hlab(np), hloc(np), fillc(nl + 1, 0), seen(nl + 1, 0);
    for (unsigned k = 0; k < nb; ++k) {
        const uint32_t l = blab[k];
        const int stride = std::max(1, (int)(bcnt[l] / (unsigned)cap));
        const int j = seen[l]++;
        if (j % stride || fillc[l] >= cap) continue;
        const int at = seg[l] + fillc[l];
        hpy[at] = (int)(bidx[k] / ncol);
        hpx[at] = (int)(bidx[k] % ncol);
        hlab[at] = (int)l;
        hloc[at] = fillc[l]++;
    }
    /* the points a region actually got (fewer than the cap when the stride
     * skips past the end) */
    {
        int at = 0;
        std::vector<int> seg2(nl + 2, 0);
        for (unsigned l = 1; l <= nl; ++l) {
            for (int k = 0; k < fillc[l]; ++k) {
                hpy[at + k] = hpy[seg[l] + k];
                hpx[at + k] = hpx[seg[l] + k];
                hlab[at + k] = hlab[seg[l] + k];
                hloc[at + k] = hloc[seg[l] + k];
            }
            seg2[l] = at;
            at += fillc[l];
            seg2[l + 1] = at;
        }
        seg.swap(seg2);
    }
    const int npts = seg[nl + 1];
    const size_t n1 = (size_t)nl + 1;
    std::vector<unsigned long long> key(n1 * n1, ~0ull);
    if (npts) {
        int *d_pts = (int *)take((size_t)npts * 16 + (n1 + 1) * 4);
        unsigned long long *d_key = (unsigned long long *)take(n1 * n1 * 8);
        if (!d_pts || !d_key) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_pts, hpy.data(), (size_t)npts * 4, cudaMemcpyHostToDevice, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_pts + npts, hpx.data(), (size_t)npts * 4, cudaMemcpyHostToDevice, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_pts + 2 * npts, hlab.data(), (size_t)npts * 4, cudaMemcpyHostToDevice, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_pts + 3 * npts, hloc.data(), (size_t)npts * 4, cudaMemcpyHostToDevice, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_pts + 4 * npts, seg.data(), (n1 + 1) * 4, cudaMemcpyHostToDevice, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_key, key.data(), n1 * n1 * 8, cudaMemcpyHostToDevice, s));
        k_br_nn<<<(npts + 255) / 256, 256, 0, s>>>(d_pts, d_pts + npts, d_pts + 2 * npts,
                                                   d_pts + 3 * npts, npts, d_pts + 4 * npts,
                                                   (int)nl, d_key);
        CUPHU_TRY_CUDA(cudaMemcpyAsync(key.data(), d_key, n1 * n1 * 8, cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaStreamSynchronize(s));
    }

    /* 8. Prim's tree from the reference region (first minimum, strict
     * improvement), then a breadth-first walk in edge order */
    auto dist = [&](size_t i, size_t j) -> float {
        const unsigned long long k = key[i * n1 + j];
        return k == ~0ull ? INFINITY : (float)(k >> (2 * kIdxBits)) / 64.0f;
    };
    std::vector<char> in(n1, 0);
    std::vector<float> bd(n1, INFINITY);
    std::vector<int> bpar(n1, -1);
    in[ref] = 1;
    for (size_t j = 1; j <= nl; ++j)
        if (j != ref) { bd[j] = dist(ref, j); bpar[j] = (int)ref; }
    std::vector<std::pair<int, int>> edges;
    for (unsigned it = 1; it < nl; ++it) {
        int u = -1;
        float ud = INFINITY;
        for (size_t j = 1; j <= nl; ++j)
            if (!in[j] && bd[j] < ud) { ud = bd[j]; u = (int)j; }
        if (u < 0) break;
        in[u] = 1;
        edges.push_back({bpar[u], u});
        for (size_t j = 1; j <= nl; ++j) {
            if (in[j]) continue;
            const float d = dist(u, j);
            if (d < bd[j]) { bd[j] = d; bpar[j] = u; }
        }
    }
    std::vector<std::vector<int>> adj(n1);
    for (auto &e : edges) { adj[e.first].push_back(e.second); adj[e.second].push_back(e.first); }
    struct Bridge { int u, v; int4 w0, w1; };
    std::vector<Bridge> br;
    const int rad = std::min(bp.radius, std::min(nrow, ncol) / 2);
    auto window = [&](int cy, int cx) {
        return make_int4(std::max(0, cy - rad), std::min(nrow, cy + rad + 1), std::max(0, cx - rad),
                         std::min(ncol, cx + rad + 1));
    };
    {
        std::vector<char> vis(n1, 0);
        std::queue<int> q;
        q.push((int)ref);
        vis[ref] = 1;
        while (!q.empty()) {
            const int u = q.front();
            q.pop();
            for (int v : adj[u]) {
                if (vis[v]) continue;
                vis[v] = 1;
                const unsigned long long k = key[(size_t)u * n1 + v];
                const int lp = (int)((k >> kIdxBits) & ((1u << kIdxBits) - 1)),
                          lq = (int)(k & ((1u << kIdxBits) - 1));
                const int pa = seg[u] + lp, pb = seg[v] + lq;
                br.push_back({u, v, window(hpy[pa], hpx[pa]), window(hpy[pb], hpx[pb])});
                q.push(v);
            }
        }
    }

    /* 9. window medians of both ends of every bridge (device), then the
     * whole-cycle corrections in walk order (host) */
    std::vector<double> corr(n1, 0.0);
    if (!br.empty()) {
        const int nreq = 2 * (int)br.size();
        std::vector<int4> hw(nreq);
        std::vector<uint32_t> hid(nreq);
        for (size_t b = 0; b < br.size(); ++b) {
            hw[2 * b] = br[b].w0;
            hid[2 * b] = (uint32_t)br[b].u;
            hw[2 * b + 1] = br[b].w1;
            hid[2 * b + 1] = (uint32_t)br[b].v;
        }
        char *d = (char *)take((size_t)nreq * (16 + 4 + 8 + 4));
        if (!d) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
        int4 *d_w = (int4 *)d;
        double *d_med = (double *)(d + (size_t)nreq * 16);
        uint32_t *d_id = (uint32_t *)(d + (size_t)nreq * 24);
        int *d_ok = (int *)(d + (size_t)nreq * 28);
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_w, hw.data(), (size_t)nreq * 16, cudaMemcpyHostToDevice, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_id, hid.data(), (size_t)nreq * 4, cudaMemcpyHostToDevice, s));
        k_br_median<<<nreq, 256, 0, s>>>(unw, lab, ncol, d_w, d_id, d_med, d_ok);
        std::vector<double> med(nreq);
        std::vector<int> okv(nreq);
        CUPHU_TRY_CUDA(cudaMemcpyAsync(med.data(), d_med, (size_t)nreq * 8, cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(okv.data(), d_ok, (size_t)nreq * 4, cudaMemcpyDeviceToHost, s));
        CUPHU_TRY_CUDA(cudaStreamSynchronize(s));
        for (size_t b = 0; b < br.size(); ++b) {
            if (!okv[2 * b] || !okv[2 * b + 1]) continue;
            const double m0 = med[2 * b], m1 = med[2 * b + 1];
            const double diff = m1 - (m0 + corr[br[b].u]);
            double jump = std::floor((std::fabs(diff) + M_PI) / (2.0 * M_PI));
            if (diff > 0) jump *= -1.0;
            corr[br[b].v] = jump * (2.0 * M_PI);
        }
    }
    double *d_corr = (double *)take(n1 * 8);
    if (!d_corr) return fail(CUPHU_ERR_ALLOC, "bridging scratch allocation failed");
    CUPHU_TRY_CUDA(cudaMemcpyAsync(d_corr, corr.data(), n1 * 8, cudaMemcpyHostToDevice, s));
    k_br_apply<<<g, 256, 0, s>>>(unw, cc, lab, n, d_corr);
    if (ramp_ok) k_br_ramp<<<g, 256, 0, s>>>(unw, nz, nrow, ncol, R, 1.0);
    CUPHU_TRY_CUDA(cudaStreamSynchronize(s));   /* the host tables outlive the copies */
    return cuda_fail(cudaGetLastError(), "bridging kernels");
}

}  // namespace cuphu
