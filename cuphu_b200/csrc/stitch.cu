/*
 * stitch.cu -- tile registration and merge (A19), all on the device.
 *
 * Reference (cuphu_solver.cpp:1846-2031): for every adjacent tile pair the
 * coherence-weighted median of (unw_A - unw_B) over the shared overlap
 * (pixels with corr >= 0.05 in both and valid in the confidence mask),
 * divided by 2*pi (left fractional for Laplace); a BFS from tile (0,0),
 * right neighbour before bottom neighbour, accumulates tile offsets; the
 * merge writes each tile's interior (overlap halves trimmed, later tiles
 * win on odd overlaps) plus its offset, and shifts conncomp labels by the
 * running maximum label of the preceding tiles.  The Python reference-pixel
 * shift (_unwrap.py:605-617) is applied in the same merge pass.
 *
 * B200 design: one CTA per tile pair finds the weighted median by a 4-pass
 * radix select over the order-preserving 32-bit key of the float
 * differences, with weights accumulated as exact 2^-28 fixed point (every
 * coherence weight >= 0.05 is an exact multiple of 2^-28, so the sums equal
 * the reference's double accumulation exactly); no sort, no host copy.
 */
#include "kernels.cuh"

namespace cuphu {

__device__ __forceinline__ uint32_t fkey(float v)
{
    uint32_t u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float fkey_inv(uint32_t k)
{
    uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    return __uint_as_float(u);
}

struct PairSample {
    bool ok;
    uint32_t key;
    unsigned long long w;
};

__device__ __forceinline__ PairSample pair_sample(const PairDesc &pd, const TileDesc &A,
                                                  const TileDesc &B, const SolverPlanes &P,
                                                  int i, int j)
{
    PairSample s;
    s.ok = false;
    int ar, ac, br, bc;
    if (pd.dir == 0) { ar = i; ac = A.nc - pd.ov + j; br = i; bc = j; }
    else             { ar = A.nr - pd.ov + i; ac = j; br = i; bc = j; }
    size_t ga = (size_t)ar * A.ph_pitch + ac, gb = (size_t)br * B.ph_pitch + bc;
    float ca = sane(A.corr[ga]), cb = sane(B.corr[gb]);
    if (ca < 0.05f || cb < 0.05f) return s;
    if (A.conf && !A.conf[ga]) return s;
    if (B.conf && !B.conf[gb]) return s;
    float ua = P.unw[A.pix + (size_t)ar * A.pitch + ac];
    float ub = P.unw[B.pix + (size_t)br * B.pitch + bc];
    s.ok = true;
    s.key = fkey(ua - ub);
    float w = ca < cb ? ca : cb;
    s.w = (unsigned long long)((double)w * 268435456.0);
    return s;
}

__global__ void __launch_bounds__(256) k_pair_median(const PairDesc *__restrict__ pairs,
                                                     const TileDesc *__restrict__ tiles,
                                                     SolverPlanes P, double *pair_k)
{
    __shared__ unsigned long long hist[256];
    __shared__ unsigned long long s_total, s_below;
    __shared__ uint32_t s_prefix, s_mask;
    const PairDesc pd = pairs[blockIdx.x];
    const TileDesc &A = tiles[pd.a];
    const TileDesc &B = tiles[pd.b];
    bool valid = pd.ov > 0 && (pd.dir == 0 ? (pd.ov <= A.nc && pd.ov <= B.nc)
                                          : (pd.ov <= A.nr && pd.ov <= B.nr));
    if (!valid) {
        if (threadIdx.x == 0) pair_k[blockIdx.x] = 0.0;
        return;
    }
    int n1 = pd.dir == 0 ? min(A.nr, B.nr) : pd.ov;
    int n2 = pd.dir == 0 ? pd.ov : min(A.nc, B.nc);
    long long ns = (long long)n1 * n2;
    if (threadIdx.x == 0) { s_total = 0ull; s_below = 0ull; s_prefix = 0u; s_mask = 0u; }
    __syncthreads();
    unsigned long long loc = 0ull;
    for (long long k = threadIdx.x; k < ns; k += blockDim.x) {
        PairSample s = pair_sample(pd, A, B, P, (int)(k / n2), (int)(k % n2));
        if (s.ok) loc += s.w;
    }
    atomicAdd(&s_total, loc);
    __syncthreads();
    unsigned long long total = s_total;
    if (total == 0ull) {
        if (threadIdx.x == 0) pair_k[blockIdx.x] = 0.0;
        return;
    }
    for (int shift = 24; shift >= 0; shift -= 8) {
        hist[threadIdx.x] = 0ull;
        __syncthreads();
        uint32_t prefix = s_prefix, mask = s_mask;
        for (long long k = threadIdx.x; k < ns; k += blockDim.x) {
            PairSample s = pair_sample(pd, A, B, P, (int)(k / n2), (int)(k % n2));
            if (s.ok && (s.key & mask) == prefix)
                atomicAdd(&hist[(s.key >> shift) & 255u], s.w);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long below = s_below;
            int sel = 255;
            for (int b = 0; b < 256; ++b) {
                if (2ull * (below + hist[b]) >= total) { sel = b; break; }
                below += hist[b];
            }
            s_below = below;
            s_prefix = prefix | ((uint32_t)sel << shift);
            s_mask = mask | (255u << shift);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) pair_k[blockIdx.x] = (double)fkey_inv(s_prefix) / kTwoPiD;
}

/* one thread per scene: BFS tile offsets, label offsets, reference shift */
__global__ void k_stitch_finalize(const ScenePlan *__restrict__ scenes, int nscenes,
                                  const TileDesc *__restrict__ tiles, SolverPlanes P,
                                  const int *__restrict__ ntile_labels,
                                  const double *__restrict__ pair_k, double *tile_k,
                                  unsigned *comp_off, SceneOut *sout, int *queue)
{
    int sidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= nscenes) return;
    const ScenePlan &S = scenes[sidx];
    int nt = S.ntr * S.ntc;
    double *tk = tile_k + S.tile0;
    for (int i = 0; i < nt; ++i) tk[i] = 0.0;
    if (nt > 1 && (S.rovl > 0 || S.covl > 0)) {
        int *q = queue + S.tile0;          /* BFS queue of local tile indices */
        int qh = 0, qt = 0;
        unsigned *seen = comp_off + S.tile0; /* visited marks; comp_off is filled below */
        for (int i = 0; i < nt; ++i) seen[i] = 0u;
        q[qt++] = 0;
        seen[0] = 1u;
        const int nh = S.ntr * (S.ntc - 1);
        while (qh < qt) {
            int idx = q[qh++];
            int br = idx / S.ntc, bc = idx % S.ntc;
            if (bc + 1 < S.ntc) {
                int nb = br * S.ntc + bc + 1;
                if (!seen[nb]) {
                    tk[nb] = tk[idx] + pair_k[S.pair0 + br * (S.ntc - 1) + bc];
                    seen[nb] = 1u;
                    q[qt++] = nb;
                }
            }
            if (br + 1 < S.ntr) {
                int nb = (br + 1) * S.ntc + bc;
                if (!seen[nb]) {
                    tk[nb] = tk[idx] + pair_k[S.pair0 + nh + br * S.ntc + bc];
                    seen[nb] = 1u;
                    q[qt++] = nb;
                }
            }
        }
    }
    unsigned run = 0u;
    for (int i = 0; i < nt; ++i) {
        comp_off[S.tile0 + i] = run;
        run += (unsigned)ntile_labels[S.tile0 + i];
    }
    SceneOut o;
    o.shift = 0.0f;
    o.do_shift = 0;
    if (S.ref_row >= 0 && S.ref_col >= 0 && S.ref_row < S.nrow && S.ref_col < S.ncol) {
        int tr = S.rowmap[S.ref_row], tc = S.colmap[S.ref_col];
        int t = S.tile0 + tr * S.ntc + tc;
        const TileDesc &T = tiles[t];
        float u = P.unw[T.pix + (size_t)(S.ref_row - T.r0) * T.pitch + (S.ref_col - T.c0)];
        if (!S.single) u = u + (float)(tk[tr * S.ntc + tc] * kTwoPiD);
        double ref = (double)S.ph[(size_t)S.ref_row * S.ncol + S.ref_col];
        double n = rint(((double)u - ref) / kTwoPiD);
        if (n != 0.0) {
            o.shift = (float)(n * kTwoPiD);
            o.do_shift = 1;
        }
    }
    sout[sidx] = o;
}

__global__ void __launch_bounds__(256) k_merge(const ScenePlan *__restrict__ scenes, int sidx,
                                               const TileDesc *__restrict__ tiles,
                                               SolverPlanes P, const double *__restrict__ tile_k,
                                               const unsigned *__restrict__ comp_off,
                                               const SceneOut *__restrict__ sout)
{
    const ScenePlan &S = scenes[sidx];
    const SceneOut o = sout[sidx];
    long long n = (long long)S.nrow * S.ncol;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int R = (int)(i / S.ncol), Cc = (int)(i % S.ncol);
        int tr = S.rowmap[R], tc = S.colmap[Cc];
        int t = S.tile0 + tr * S.ntc + tc;
        const TileDesc &T = tiles[t];
        size_t pi = T.pix + (size_t)(R - T.r0) * T.pitch + (Cc - T.c0);
        float u = P.unw[pi];
        if (!S.single) u = u + (float)(tile_k[t] * kTwoPiD);
        if (o.do_shift) u = u - o.shift;
        S.unw_out[i] = u;
        if (S.cc_out) {
            uint32_t c = P.cc[pi];
            S.cc_out[i] = c == 0u ? 0u : c + comp_off[t];
        }
    }
}

/* the reference-pixel shift of a merged scene whose post-passes ran after
 * the merge: n = rint((unw[ref] - phi[ref]) / 2pi), then unw -= float(n 2pi)
 * (the merge kernel's rule, on the post-processed value) */
__global__ void k_ref_shift_n(const float *unw, const float *ph, int ncol, int ref_row,
                              int ref_col, SceneOut *o)
{
    size_t i = (size_t)ref_row * ncol + ref_col;
    double n = rint(((double)unw[i] - (double)ph[i]) / kTwoPiD);
    o->shift = (float)(n * kTwoPiD);
    o->do_shift = n != 0.0 ? 1 : 0;
}

__global__ void __launch_bounds__(256) k_ref_shift_apply(float *unw, long long n,
                                                         const SceneOut *o)
{
    if (!o->do_shift) return;
    const float sh = o->shift;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        unw[i] = unw[i] - sh;
}

int launch_ref_shift(float *unw, const float *ph, int nrow, int ncol, int ref_row, int ref_col,
                     SceneOut *tmp, cudaStream_t s)
{
    if (ref_row < 0 || ref_col < 0 || ref_row >= nrow || ref_col >= ncol) return 0;
    k_ref_shift_n<<<1, 1, 0, s>>>(unw, ph, ncol, ref_row, ref_col, tmp);
    long long n = (long long)nrow * ncol;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_ref_shift_apply<<<blocks, 256, 0, s>>>(unw, n, tmp);
    return cuda_fail(cudaGetLastError(), "reference-pixel shift");
}

int launch_stitch(const ScenePlan *scenes, int nscenes, const TileDesc *tiles,
                  const PairDesc *pairs, int npairs, const SolverPlanes &P,
                  const int *ntile_labels, double *pair_k, double *tile_k,
                  unsigned *comp_off, SceneOut *sout, cudaStream_t s)
{
    if (npairs > 0) k_pair_median<<<npairs, 256, 0, s>>>(pairs, tiles, P, pair_k);
    /* the BFS queue reuses pair_k's tail: [npairs] medians, then [ntiles] queue */
    int *queue = reinterpret_cast<int *>(pair_k + npairs);
    k_stitch_finalize<<<(nscenes + 63) / 64, 64, 0, s>>>(scenes, nscenes, tiles, P, ntile_labels,
                                                        pair_k, tile_k, comp_off, sout, queue);
    return cuda_fail(cudaGetLastError(), "stitch kernels");
}

int launch_merge(const ScenePlan *scenes, const ScenePlan *h_scenes, int nscenes,
                 const TileDesc *tiles, const SolverPlanes &P, const double *tile_k,
                 const unsigned *comp_off, const SceneOut *sout, cudaStream_t s)
{
    for (int i = 0; i < nscenes; ++i) {
        long long n = (long long)h_scenes[i].nrow * h_scenes[i].ncol;
        int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
        k_merge<<<blocks, 256, 0, s>>>(scenes, i, tiles, P, tile_k, comp_off, sout);
    }
    return cuda_fail(cudaGetLastError(), "k_merge");
}

}  // namespace cuphu
