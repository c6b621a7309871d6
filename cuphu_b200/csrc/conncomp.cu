/*
 * conncomp.cu -- connected-component labelling of the unwrapped phase (A16).
 *
 * Semantics of cuphu_conncomp_gpu (cuphu_conncomp.cu:83-93, 96-114, 178-286,
 * 290-428): a pixel is valid when corr >= 0.05 and mask != 0; two 4-neighbours
 * are joined when both are valid, |unw_a - unw_b| < pi (float) and, when MCF
 * incremental costs are given, min(poscost, negcost) >= conncompthresh.
 * Components of at least max(1, (int)(minconncompfrac * npix)) pixels get
 * labels 1..maxncomps in increasing order of their smallest pixel index;
 * everything else is 0.
 *
 * B200 design: lock-free union-find with atomicMin linking (roots are always
 * component minima, so the canonical order comes for free), pointer-halving
 * finds, then the label map is built on the device by a per-row ballot scan
 * (the reference downloads all npix counts, builds the map on the host and
 * uploads it again, cuphu_conncomp.cu:401-424).  Every kernel takes a list of
 * tiles so all tiles of all scenes label in one launch per step.
 */
#include "kernels.cuh"

namespace cuphu {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t uf_find(uint32_t *P, uint32_t x)
{
    while (true) {
        uint32_t p = __ldcg(P + x);
        if (p == x) return x;
        uint32_t gp = __ldcg(P + p);
        if (gp != p) P[x] = gp;   /* path halving: gp is an ancestor of x */
        x = gp;
    }
}

__device__ __forceinline__ void uf_unite(uint32_t *P, uint32_t a, uint32_t b)
{
    while (true) {
        a = uf_find(P, a);
        b = uf_find(P, b);
        if (a == b) return;
        if (a < b) { uint32_t t = a; a = b; b = t; }
        uint32_t old = atomicMin(P + a, b);
        if (old == a) return;
        a = old;
    }
}

struct PixIter {
    int r, c0;
};

__device__ __forceinline__ PixIter pix_of(const TileDesc &T, int li)
{
    PixIter q;
    int iby = li / T.nbx, ibx = li % T.nbx;
    q.r = iby * kItemBy + threadIdx.x / kItemTx;
    q.c0 = ibx * kItemBx + (threadIdx.x % kItemTx) * kItemVx;
    return q;
}

__global__ void __launch_bounds__(kItemThreads) k_cc_init(const TileDesc *__restrict__ tiles,
                                                          const int *__restrict__ item_tile,
                                                          int nitems, SolverPlanes P, CcArgs a)
{
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const TileDesc &T = tiles[item_tile[item]];
        PixIter q = pix_of(T, item - T.item0);
        if (q.r >= T.nr) continue;
        for (int j = 0; j < kItemVx; ++j) {
            int c = q.c0 + j;
            if (c >= T.nc) continue;
            size_t gi = (size_t)q.r * T.ph_pitch + c;
            bool bad = sane(T.corr[gi]) < a.corr_thresh;
            if (T.mask) bad = bad || T.mask[gi] == 0;
            uint32_t li = (uint32_t)((size_t)q.r * T.pitch + c);
            P.cc[T.pix + li] = bad ? kInvalid : li;
            P.aux[T.pix + li] = 0u;
        }
    }
}

__global__ void __launch_bounds__(kItemThreads) k_cc_union(const TileDesc *__restrict__ tiles,
                                                           const int *__restrict__ item_tile,
                                                           int nitems, SolverPlanes P, CcArgs a)
{
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const TileDesc &T = tiles[item_tile[item]];
        PixIter q = pix_of(T, item - T.item0);
        if (q.r >= T.nr) continue;
        uint32_t *par = P.cc + T.pix;
        const float *u = P.unw + T.pix;
        for (int j = 0; j < kItemVx; ++j) {
            int c = q.c0 + j;
            if (c >= T.nc) continue;
            uint32_t i = (uint32_t)((size_t)q.r * T.pitch + c);
            if (__ldcg(par + i) == kInvalid) continue;
            float ua = u[i];
            if (c + 1 < T.nc && __ldcg(par + i + 1) != kInvalid && fabsf(ua - u[i + 1]) < kPiF) {
                bool ok = true;
                if (a.poscost) {
                    size_t arc = (size_t)(T.nr - 1) * T.nc + (size_t)q.r * (T.nc - 1) + c;
                    short mc = min(a.poscost[arc], a.negcost[arc]);
                    ok = (long)mc >= a.conncompthresh;
                }
                if (ok) uf_unite(par, i, i + 1);
            }
            if (q.r + 1 < T.nr && __ldcg(par + i + T.pitch) != kInvalid &&
                fabsf(ua - u[i + T.pitch]) < kPiF) {
                bool ok = true;
                if (a.poscost) {
                    size_t arc = (size_t)q.r * T.nc + c;
                    short mc = min(a.poscost[arc], a.negcost[arc]);
                    ok = (long)mc >= a.conncompthresh;
                }
                if (ok) uf_unite(par, i, i + T.pitch);
            }
        }
    }
}

__global__ void __launch_bounds__(kItemThreads) k_cc_flatten(const TileDesc *__restrict__ tiles,
                                                             const int *__restrict__ item_tile,
                                                             int nitems, SolverPlanes P)
{
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const TileDesc &T = tiles[item_tile[item]];
        PixIter q = pix_of(T, item - T.item0);
        if (q.r >= T.nr) continue;
        uint32_t *par = P.cc + T.pix;
        for (int j = 0; j < kItemVx; ++j) {
            int c = q.c0 + j;
            if (c >= T.nc) continue;
            uint32_t i = (uint32_t)((size_t)q.r * T.pitch + c);
            if (__ldcg(par + i) == kInvalid) continue;
            uint32_t root = uf_find(par, i);
            atomicAdd(P.aux + T.pix + root, 1u);
        }
    }
}

/* store the root of every valid pixel (after all finds of the previous
 * kernel completed, so the forest is final) */
__global__ void __launch_bounds__(kItemThreads) k_cc_compress(const TileDesc *__restrict__ tiles,
                                                              const int *__restrict__ item_tile,
                                                              int nitems, SolverPlanes P)
{
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const TileDesc &T = tiles[item_tile[item]];
        PixIter q = pix_of(T, item - T.item0);
        if (q.r >= T.nr) continue;
        uint32_t *par = P.cc + T.pix;
        for (int j = 0; j < kItemVx; ++j) {
            int c = q.c0 + j;
            if (c >= T.nc) continue;
            uint32_t i = (uint32_t)((size_t)q.r * T.pitch + c);
            uint32_t p = __ldcg(par + i);
            if (p == kInvalid || p == i) continue;
            par[i] = uf_find(par, p);
        }
    }
}

__device__ __forceinline__ int tile_min_size(const TileDesc &T, double minfrac)
{
    int m = (int)(minfrac * (double)((long long)T.nr * T.nc));
    return m < 1 ? 1 : m;
}

/* one warp per tile row: number of labelled roots in the row */
__global__ void k_cc_rowcount(const TileDesc *__restrict__ tiles, const int *__restrict__ row_tile,
                              int total_rows, SolverPlanes P, CcArgs a, int *rowcnt)
{
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= total_rows) return;
    const TileDesc &T = tiles[row_tile[warp]];
    int r = warp - T.row0;
    int ms = tile_min_size(T, a.minfrac);
    const uint32_t *par = P.cc + T.pix;
    const uint32_t *cnt = P.aux + T.pix;
    int n = 0;
    for (int c0 = 0; c0 < T.nc; c0 += 32) {
        int c = c0 + lane;
        bool qv = false;
        if (c < T.nc) {
            uint32_t i = (uint32_t)((size_t)r * T.pitch + c);
            qv = __ldcg(par + i) == i && __ldcg(cnt + i) >= (uint32_t)ms;
        }
        n += __popc(__ballot_sync(0xffffffffu, qv));
    }
    if (lane == 0) rowcnt[warp] = n;
}

/* one block per tile: exclusive scan of its row counts; labels in the tile */
__global__ void __launch_bounds__(1024) k_cc_rowscan(const TileDesc *__restrict__ tiles,
                                                     int ntiles, int *rowcnt, CcArgs a,
                                                     int *ntile_labels)
{
    __shared__ int swarp[32];
    __shared__ int s_carry;
    int t = blockIdx.x;
    if (t >= ntiles) return;
    const TileDesc &T = tiles[t];
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < T.nr; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < T.nr ? rowcnt[T.row0 + i] : 0;
        int x = v;
        for (int off = 1; off < 32; off <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31) swarp[w] = x;
        __syncthreads();
        if (w == 0) {
            int s = lane < (int)(blockDim.x >> 5) ? swarp[lane] : 0;
            for (int off = 1; off < 32; off <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, s, off);
                if (lane >= off) s += y;
            }
            swarp[lane] = s;
        }
        __syncthreads();
        int incl = x + (w > 0 ? swarp[w - 1] : 0);
        int carry = s_carry;
        if (i < T.nr) rowcnt[T.row0 + i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = carry + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) ntile_labels[t] = min(s_carry, a.maxncomps);
}

/* one warp per tile row: labels of the row's roots (rank < maxncomps) */
__global__ void k_cc_rowlabel(const TileDesc *__restrict__ tiles, const int *__restrict__ row_tile,
                              int total_rows, SolverPlanes P, CcArgs a, const int *rowoff)
{
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= total_rows) return;
    const TileDesc &T = tiles[row_tile[warp]];
    int r = warp - T.row0;
    int ms = tile_min_size(T, a.minfrac);
    const uint32_t *par = P.cc + T.pix;
    uint32_t *aux = P.aux + T.pix;
    int run = rowoff[warp];
    for (int c0 = 0; c0 < T.nc; c0 += 32) {
        int c = c0 + lane;
        bool root = false, qv = false;
        uint32_t i = 0;
        if (c < T.nc) {
            i = (uint32_t)((size_t)r * T.pitch + c);
            root = __ldcg(par + i) == i;
            qv = root && __ldcg(aux + i) >= (uint32_t)ms;
        }
        unsigned b = __ballot_sync(0xffffffffu, qv);
        if (root) {
            int rank = run + __popc(b & ((1u << lane) - 1u));
            aux[i] = (qv && rank < a.maxncomps) ? (uint32_t)(rank + 1) : 0u;
        }
        run += __popc(b);
    }
}

__global__ void __launch_bounds__(kItemThreads) k_cc_final(const TileDesc *__restrict__ tiles,
                                                           const int *__restrict__ item_tile,
                                                           int nitems, SolverPlanes P)
{
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const TileDesc &T = tiles[item_tile[item]];
        PixIter q = pix_of(T, item - T.item0);
        if (q.r >= T.nr) continue;
        uint32_t *par = P.cc + T.pix;
        const uint32_t *aux = P.aux + T.pix;
        for (int j = 0; j < kItemVx; ++j) {
            int c = q.c0 + j;
            if (c >= T.nc) continue;
            uint32_t i = (uint32_t)((size_t)q.r * T.pitch + c);
            uint32_t p = par[i];
            par[i] = p == kInvalid ? 0u : __ldcg(aux + p);
        }
    }
}

int launch_conncomp(const TileDesc *tiles, int ntiles, int total_rows, const int *item_tile,
                    int nitems, const SolverPlanes &P, const CcArgs &a, int *rowcnt,
                    int *ntile_labels, cudaStream_t s)
{
    /* rowcnt: [total_rows] scratch followed by [total_rows] row->tile map */
    const int *row_tile = rowcnt + total_rows;
    int g = std::min(nitems, 148 * 16);
    int gw = (total_rows * 32 + 255) / 256;
    k_cc_init<<<g, kItemThreads, 0, s>>>(tiles, item_tile, nitems, P, a);
    k_cc_union<<<g, kItemThreads, 0, s>>>(tiles, item_tile, nitems, P, a);
    k_cc_flatten<<<g, kItemThreads, 0, s>>>(tiles, item_tile, nitems, P);
    k_cc_compress<<<g, kItemThreads, 0, s>>>(tiles, item_tile, nitems, P);
    k_cc_rowcount<<<gw, 256, 0, s>>>(tiles, row_tile, total_rows, P, a, rowcnt);
    k_cc_rowscan<<<ntiles, 1024, 0, s>>>(tiles, ntiles, rowcnt, a, ntile_labels);
    k_cc_rowlabel<<<gw, 256, 0, s>>>(tiles, row_tile, total_rows, P, a, rowcnt);
    k_cc_final<<<g, kItemThreads, 0, s>>>(tiles, item_tile, nitems, P);
    return cuda_fail(cudaGetLastError(), "conncomp kernels");
}

}  // namespace cuphu
