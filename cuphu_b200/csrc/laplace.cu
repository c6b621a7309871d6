/*
 * laplace.cu -- persistent, tile-batched Jacobi-PCG + IRLS Laplace solver.
 *
 * Restates cuphu_laplace_unwrap_gpu (cuphu_laplace.cu:352-552): per tile,
 * w0 = 1/sigsq, then N_IRLS+1 weighted-least-squares solves of
 * (D^T W D + eps I) u = D^T W wrap(D phi) by Jacobi-preconditioned CG, the
 * first from u = 0 and the rest warm-started, with IRLS reweighting
 * w = w0 / sqrt(e^2 + delta^2) between solves; then the (0,0) anchor and the
 * congruence projection.
 *
 * B200 design:
 *  - ONE cooperative launch runs every pass of every tile of every scene.
 *    Phases are separated by a grid barrier (atomic arrive + generation flag,
 *    bounded spin with an error status); per-tile dot products reduce
 *    deterministically (fixed tree per work item, last-arriving block of a
 *    tile reduces the item partials in fixed order) in FP64, so there are no
 *    host round trips and no float atomics (the reference does two blocking
 *    D2H syncs per iteration and accumulates dots with float atomicAdd).
 *  - FP64 mode keeps every vector in double and is bit-identical to the CPU
 *    FP64 oracle (same operation order, explicit fma, same reduction tree):
 *    two passes and two grid barriers per iteration.  The stencil pass
 *    rebuilds p = z + beta p_old for its item and halo in shared memory
 *    (p is double-buffered so neighbours never race) and computes q = A p;
 *    the update pass moves x, r and z.
 *  - Mixed mode runs ONE pass and ONE grid barrier per iteration (a
 *    single-synchronisation form of the same Jacobi-PCG).  The solution is an
 *    FP64 base x plus an FP32 increment dx; r, p, q are FP32 and each is
 *    double-buffered.  Each pass applies the previous iteration's update
 *    (dx += alpha p_old, r = r - alpha q), forms z = M^-1 r (M^-1 the
 *    hardware reciprocal of an FP32 Jacobi diagonal summed from the staged
 *    arc weights), folds p = z + beta p_old, own pixels and halo alike, and
 *    computes q = A p; it reduces r.z, p.q, z.q and q.M^-1 q with FP64
 *    accuracy in one tree.  alpha and the stop test use the true r.z of the
 *    pass; beta uses the one-step recurrence
 *    r.z' = r.z - 2 alpha z.q + alpha^2 q.M^-1 q anchored at that true value.
 *    Every `replace_every` iterations the increment is folded into x and the
 *    recursive residual is replaced by the true residual b - A x (FP64).
 */
#include "kernels.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda/atomic>
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

namespace cuphu {

constexpr int kHaloH = kItemBy + 2;

/* ── vector access helpers (L2-coherent loads of in-kernel-written data) ── */
__device__ __forceinline__ void ld4(const float *p, float v[4])
{
    float4 t = __ldcg(reinterpret_cast<const float4 *>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ld4(const double *p, double v[4])
{
    double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
    double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void st4(float *p, const float v[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double *p, const double v[4])
{
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
template <typename T> __device__ __forceinline__ T ldc(const T *p) { return __ldcg(p); }

/* ── canonical block reduction: shuffle-down tree per warp, then warp 0
 *    reduces the warp sums (result in thread 0) ─────────────────────────── */
__device__ __forceinline__ double block_sum(double v, double *sw)
{
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sw[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sw[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    }
    return v;
}

/* Tile total of the item partials of one phase, in fixed order: thread j
 * sums items j, j+256, ... then the block tree.  Every block computes it the
 * same way, so all blocks touching a tile agree bit for bit. */
__device__ __forceinline__ double tile_reduce(const TileDesc &T, const double *part, double *sw,
                                              double *s_bcast)
{
    double a = 0.0;
    for (int i = threadIdx.x; i < T.nitems; i += blockDim.x) a = a + __ldcg(part + T.item0 + i);
    double tot = block_sum(a, sw);
    if (threadIdx.x == 0) *s_bcast = tot;
    __syncthreads();
    tot = *s_bcast;
    __syncthreads();
    return tot;
}

/* Partials of items [a, b) of tile T, eight items per pair of block
 * barriers: each warp reduces its thread values of an item by block_sum's
 * first tree and parks the warp sum; after the barrier warp k forms item
 * k's partial by block_sum's second tree.  The partials are block_sum's of
 * each item (the canonical tree the FP64 oracle reproduces), but warps run
 * ahead through the eight items instead of meeting at two barriers per
 * item.  f(li) returns the thread's value of item li. */
constexpr int kItemGroup = 8;
template <typename F>
__device__ __forceinline__ void item_partials(const TileDesc &T, int a, int b, double *part,
                                              double (*sgrp)[8], F &&f)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int g0 = a; g0 < b; g0 += kItemGroup) {
        const int n = min(kItemGroup, b - g0);
        for (int k = 0; k < n; ++k) {
            double v = f(g0 + k);
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) sgrp[k][w] = v;
        }
        __syncthreads();
        if (w < n) {
            double v = lane < (int)(blockDim.x >> 5) ? sgrp[w][lane] : 0.0;
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) part[T.item0 + g0 + w] = v;
        }
        __syncthreads();
    }
}

/* block tree without the leading barrier, for item loops: consecutive items
 * pass alternating halves of the scratch (sw, sw + 8), so a warp that runs
 * ahead into the next item never overwrites warp sums that warp 0 has not
 * read; returns after the barrier that follows the warp sums, so every thread
 * has finished the caller's work on the item */
__device__ __forceinline__ double block_sum_item(double v, double *sw)
{
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sw[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sw[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    }
    return v;
}

/* A block has written the partials of its items [a, b) of tile t for this
 * phase (thread 0 writes every partial of a block).  The block whose items
 * complete the tile's count computes the canonical tile total once and
 * publishes it in tot[t]; the other blocks move on.  The total is the same
 * whichever block computes it, because tile_reduce fixes the order.  Readers
 * pick it up after the next grid barrier. */
__device__ void seg_done(const TileDesc &T, int t, int nseg, const double *part, double *tot,
                         unsigned *cnt, double *sw, double *s_bcast, int *s_flag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned prev = atomicAdd(&cnt[t], (unsigned)nseg);
        int last = prev + (unsigned)nseg == (unsigned)T.nitems;
        if (last) __threadfence();
        *s_flag = last;
    }
    __syncthreads();
    if (*s_flag) {
        double v = tile_reduce(T, part, sw, s_bcast);
        if (threadIdx.x == 0) {
            tot[t] = v;
            cnt[t] = 0u;
        }
    }
}

/* seg_done for the kNComp-component partials of the mixed pass: component c
 * of item i at part[c * nitems + i], of tile t at tot[c * ntiles + t] */
/* warp sums of four values by a reduce-scatter tree: after the xor-16 and
 * xor-8 steps each lane holds one component (lanes 8c..8c+7 component c),
 * then three plain levels; every lane of group c returns the warp's sum of
 * component c (the same value in all eight lanes) */
__device__ __forceinline__ double warp_scatter4(const double a[kNComp])
{
    static_assert(kNComp == 4, "four components");
    const int lane = threadIdx.x & 31;
    const bool hi16 = lane & 16, hi8 = lane & 8;
    const double r0 = __shfl_xor_sync(0xffffffffu, hi16 ? a[0] : a[2], 16);
    const double r1 = __shfl_xor_sync(0xffffffffu, hi16 ? a[1] : a[3], 16);
    const double k0 = (hi16 ? a[2] : a[0]) + r0;
    const double k1 = (hi16 ? a[3] : a[1]) + r1;
    const double r2 = __shfl_xor_sync(0xffffffffu, hi8 ? k0 : k1, 8);
    double v = (hi8 ? k1 : k0) + r2;
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v;
}

__device__ void seg_done4(const TileDesc &T, int t, int nseg, const double *part, int nitems,
                          double *tot, int ntiles, unsigned *cnt, double *sw, double *s_bcast,
                          int *s_flag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned prev = atomicAdd(&cnt[t], (unsigned)nseg);
        int last = prev + (unsigned)nseg == (unsigned)T.nitems;
        if (last) __threadfence();
        *s_flag = last;
    }
    __syncthreads();
    if (*s_flag) {
        /* the four tile totals in one sweep, in a fixed order: thread j
         * sums items j, j+256, ... per component, then the warp trees
         * (warp_scatter4) and a three-level tree over the eight warps */
        double a[kNComp] = {0.0, 0.0, 0.0, 0.0};
        for (int i = threadIdx.x; i < T.nitems; i += blockDim.x)
#pragma unroll
            for (int c = 0; c < kNComp; ++c)
                a[c] = a[c] + __ldcg(part + (size_t)c * nitems + T.item0 + i);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const double v = warp_scatter4(a);
        if ((lane & 7) == 0) sw[(lane >> 3) * 8 + warp] = v;
        __syncthreads();
        if (warp == 0) {
            double x = sw[(lane >> 3) * 8 + (lane & 7)];
            x += __shfl_xor_sync(0xffffffffu, x, 4);
            x += __shfl_xor_sync(0xffffffffu, x, 2);
            x += __shfl_xor_sync(0xffffffffu, x, 1);
            if ((lane & 7) == 0) tot[(size_t)(lane >> 3) * ntiles + t] = x;
        }
        if (threadIdx.x == 0) cnt[t] = 0u;
        __syncthreads();
    }
}

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* Grid barrier with a bounded wait.  The last arriving block snapshots the
 * active-tile count, so every block takes the same loop decision.  A block
 * called with arrive = false waits without arriving (the failure test of
 * cuphu_test_skip_barrier_once): every wait then runs out and the error
 * status ends the kernel. */
__device__ __forceinline__ bool grid_sync(SolverCtl *ctl, long long timeout_ns,
                                          bool arrive = true)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(ctl->bar_gen);
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(ctl->bar_count);
        cuda::atomic_ref<int, cuda::thread_scope_device> act(ctl->n_active);
        __threadfence();
        unsigned g = gen.load(cuda::memory_order_acquire);
        unsigned prev = arrive ? cnt.fetch_add(1u, cuda::memory_order_acq_rel) : 0u;
        if (arrive && prev == gridDim.x - 1u) {
            cnt.store(0u, cuda::memory_order_relaxed);
            *(volatile int *)&ctl->snap = act.load(cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
        } else {
            unsigned long long t0 = globaltimer();
            long long spins = 0;
            while (gen.load(cuda::memory_order_acquire) == g) {
                if (*(volatile int *)&ctl->err) break;
                if (((++spins) & 63) == 0 && (long long)(globaltimer() - t0) > timeout_ns) {
                    atomicExch(&ctl->err, 1);
                    break;
                }
                if (spins > (1LL << 34)) { atomicExch(&ctl->err, 1); break; }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)&ctl->err == 0;
}

struct ItemXY {
    int r, c0, ty, tx;
};

__device__ __forceinline__ ItemXY item_xy(const TileDesc &T, int li)
{
    ItemXY q;
    int iby = li / T.nbx, ibx = li % T.nbx;
    q.ty = threadIdx.x / kItemTx;
    q.tx = threadIdx.x % kItemTx;
    q.r = iby * kItemBy + q.ty;
    q.c0 = ibx * kItemBx + q.tx * kItemVx;
    return q;
}

/* ── mixed-precision preconditioner and dots ─────────────────────────────
 * diag32: the Jacobi diagonal as an FP32 sum of the positive in-tile arc
 * weights (down, up, right, left) plus eps; rcp_pre: its reciprocal by the
 * hardware approximation (rcp.approx, within 1 ulp).  M^-1 = rcp_pre(diag32)
 * is the preconditioner of the mixed solve: every place that forms
 * z = M^-1 r (the INIT/true-residual phase, an item's own pixels, its halo
 * ring) evaluates these two functions on the same weights, so all blocks
 * agree on M bit for bit and no division is needed. */
__device__ __forceinline__ float diag32(int r, int c, int nr, int nc, float wdn, float wup,
                                        float wrt, float wlf)
{
    float ws = 0.0f;
    if (r < nr - 1 && wdn > 0.0f) ws = __fadd_rn(ws, wdn);
    if (r > 0 && wup > 0.0f) ws = __fadd_rn(ws, wup);
    if (c < nc - 1 && wrt > 0.0f) ws = __fadd_rn(ws, wrt);
    if (c > 0 && wlf > 0.0f) ws = __fadd_rn(ws, wlf);
    return __fadd_rn(ws, kLapEpsF);
}

__device__ __forceinline__ float rcp_pre(float d)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
    return y;
}

/* sum_j a[j] b[j] over a thread's four pixels with FP64 accuracy and no
 * per-element conversion: each FP32 product is split exactly into
 * p + e (e = fma(a, b, -p)), the p are summed with Knuth's TwoSum (the
 * rounding error of each addition recovered exactly), and the small terms
 * in FP32; hi + lo is then converted once.  For products in FP32's normal
 * range the error is ~2^-44 of the sum of the magnitudes, far below what
 * the FP64 tree reduction over a tile rounds away. */
__device__ __forceinline__ double dot4_df(const float a[4], const float b[4])
{
    float hi = __fmul_rn(a[0], b[0]);
    float lo = __fmaf_rn(a[0], b[0], -hi);
#pragma unroll
    for (int j = 1; j < 4; ++j) {
        const float p = __fmul_rn(a[j], b[j]);
        const float e = __fmaf_rn(a[j], b[j], -p);
        const float s = __fadd_rn(hi, p);
        const float bp = __fsub_rn(s, hi);
        const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(p, bp));
        hi = s;
        lo = __fadd_rn(lo, __fadd_rn(e, err));
    }
    return (double)hi + (double)lo;
}

/* paired FP32 arithmetic (two lanes per instruction, IEEE round-to-nearest
 * per lane, the same results as the scalar operations) */
__device__ __forceinline__ float2 pf2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b)   /* a - b, one rounding */
{
    return __ffma2_rn(b, pf2(-1.0f, -1.0f), a);
}

/* two dot4_df sums at once, lane 0 for (a0, b0) and lane 1 for (a1, b1):
 * the same operations, so each result equals dot4_df's */
__device__ __forceinline__ void dot4_df2(const float a0[4], const float b0[4], const float a1[4],
                                         const float b1[4], double &r0, double &r1)
{
    float2 a = pf2(a0[0], a1[0]), b = pf2(b0[0], b1[0]);
    float2 hi = __fmul2_rn(a, b);
    float2 lo = __ffma2_rn(a, b, pf2(-hi.x, -hi.y));
#pragma unroll
    for (int j = 1; j < 4; ++j) {
        a = pf2(a0[j], a1[j]);
        b = pf2(b0[j], b1[j]);
        const float2 p = __fmul2_rn(a, b);
        const float2 e = __ffma2_rn(a, b, pf2(-p.x, -p.y));
        const float2 sm = __fadd2_rn(hi, p);
        const float2 bp = psub(sm, hi);
        const float2 err = __fadd2_rn(psub(hi, psub(sm, bp)), psub(p, bp));
        hi = sm;
        lo = __fadd2_rn(lo, __fadd2_rn(e, err));
    }
    r0 = (double)hi.x + (double)lo.x;
    r1 = (double)hi.y + (double)lo.y;
}

/* ── INIT / true residual: b, diag (A10) and r = b - A x, rz partial ────────
 * zero_x: first pass (x = 0, r = b).  write_diag: assemble pass (else the
 * stored diag is reused: residual replacement).  FP64 mode: z = r / diag
 * goes to zout.  Mixed mode: the FP32 residual r goes to zout (its
 * double-buffered residual plane), the preconditioner is M^-1 =
 * rcp_pre(diag32) recomputed from the weights, and the partial r.z comes
 * from dot4_df.  With P.bvec (mixed mode) the assemble pass stores the
 * right-hand side b and the replacements of the same IRLS pass read it back
 * instead of rebuilding it from the wrapped phase (the same doubles either
 * way).  The thread's row and the rows above and below of x and of the arc
 * weights arrive as 16-byte vectors; only the phase (scene layout) is read
 * element by element.  The arithmetic and its order are the oracle's. */
template <typename V, bool WLS>
__device__ double phase_init(const TileDesc &T, int li, const SolverPlanes &P, bool zero_x,
                             bool write_diag, V *zout)
{
    ItemXY q = item_xy(T, li);
    if (q.r >= T.nr || q.c0 >= T.nc) return 0.0;
    double *x = P.x + T.pix;
    V *rr = (V *)P.r + T.pix;
    V *dg = (V *)P.diag + T.pix;
    const float *wd = P.wd + T.pix, *wr = P.wr + T.pix;
    const float *ph = T.ph;
    /* WLS mode: per-arc targets or an explicit right-hand side */
    const float *gdp = (WLS && P.gd) ? P.gd + T.pix : nullptr;
    const float *grp = (WLS && P.gr) ? P.gr + T.pix : nullptr;
    const float *rhsp = (WLS && P.rhs) ? P.rhs + T.pix : nullptr;
    const double eps = (double)kLapEpsF;
    const int r = q.r, nr = T.nr, nc = T.nc, pitch = T.pitch, pp = T.ph_pitch;
    const size_t prow = (size_t)r * pitch;
    const bool has_dn = r < nr - 1, has_up = r > 0;
    const bool has_l = q.c0 > 0, has_r = q.c0 + kItemVx < nc;
    /* the down arcs of this row and of the row above (the up arcs), the
     * right arcs of this row and the one left of the thread's columns; the
     * last row of wd and the last column of wr are zero, so the vectors
     * stay inside the tile's rows */
    float wdn[4], wup[4] = {0.f, 0.f, 0.f, 0.f}, wrt[4];
    ld4(wd + prow + q.c0, wdn);
    if (has_up) ld4(wd + prow - pitch + q.c0, wup);
    ld4(wr + prow + q.c0, wrt);
    const float wlf = has_l ? ldc(wr + prow + q.c0 - 1) : 0.0f;
    double xv[4], xdn[4] = {0.0, 0.0, 0.0, 0.0}, xup[4] = {0.0, 0.0, 0.0, 0.0};
    double xl = 0.0, xr = 0.0;
    if (!zero_x) {
        ld4(x + prow + q.c0, xv);
        if (has_dn) ld4(x + prow + pitch + q.c0, xdn);
        if (has_up) ld4(x + prow - pitch + q.c0, xup);
        if (has_l) xl = ldc(x + prow + q.c0 - 1);
        if (has_r) xr = ldc(x + prow + q.c0 + kItemVx);
    }
    V rv[4], dv[4], zv[4];
    float zf[4];   /* mixed: z = M^-1 r of the thread's pixels */
    if (!write_diag && sizeof(V) == 8) ld4(dg + prow + q.c0, dv);
    double *bvp = P.bvec ? P.bvec + T.pix + prow + q.c0 : nullptr;
    const bool b_stored = bvp && !write_diag;
    double bst[4];
    if (b_stored) ld4((const double *)bvp, bst);
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        int c = q.c0 + j;
        if (c >= nc) {
            rv[j] = (V)0;
            zv[j] = (V)0;
            zf[j] = 0.0f;
            if (write_diag) dv[j] = (V)0;
            if (zero_x) xv[j] = 0.0;
            bst[j] = 0.0;
            continue;
        }
        const float w_dn = wdn[j], w_up = wup[j], w_rt = wrt[j];
        const float w_lf = j == 0 ? wlf : wrt[j - 1];
        double bv = 0.0, ws = 0.0;
        float ws32 = 0.0f;   /* mixed: diag32's sum, in its order */
        if (b_stored) {
            bv = bst[j];
            if (has_dn && w_dn > 0.0f) ws32 = __fadd_rn(ws32, w_dn);
            if (has_up && w_up > 0.0f) ws32 = __fadd_rn(ws32, w_up);
            if (c < nc - 1 && w_rt > 0.0f) ws32 = __fadd_rn(ws32, w_rt);
            if (c > 0 && w_lf > 0.0f) ws32 = __fadd_rn(ws32, w_lf);
        } else {
            const size_t gi = (size_t)r * pp + c, pi = prow + c;
            float pa = gdp ? 0.0f : __ldg(ph + gi);
            if (has_dn && w_dn > 0.0f) {
                float g = gdp ? ldc(gdp + pi) : lap_wrap_pi(__ldg(ph + gi + pp) - pa);
                bv = __fma_rn(-(double)w_dn, (double)g, bv);
                ws += w_dn;
                ws32 = __fadd_rn(ws32, w_dn);
            }
            if (has_up && w_up > 0.0f) {
                float g = gdp ? ldc(gdp + pi - pitch) : lap_wrap_pi(pa - __ldg(ph + gi - pp));
                bv = __fma_rn((double)w_up, (double)g, bv);
                ws += w_up;
                ws32 = __fadd_rn(ws32, w_up);
            }
            if (c < nc - 1 && w_rt > 0.0f) {
                float g = grp ? ldc(grp + pi) : lap_wrap_pi(__ldg(ph + gi + 1) - pa);
                bv = __fma_rn(-(double)w_rt, (double)g, bv);
                ws += w_rt;
                ws32 = __fadd_rn(ws32, w_rt);
            }
            if (c > 0 && w_lf > 0.0f) {
                float g = grp ? ldc(grp + pi - 1) : lap_wrap_pi(pa - __ldg(ph + gi - 1));
                bv = __fma_rn((double)w_lf, (double)g, bv);
                ws += w_lf;
                ws32 = __fadd_rn(ws32, w_lf);
            }
            if (rhsp) bv = (double)ldc(rhsp + pi);
            bst[j] = bv;
        }
        double d = write_diag ? ws + eps : (double)dv[j];
        double y;
        if (zero_x) {
            y = 0.0;
            xv[j] = 0.0;
        } else {
            const double xa = xv[j];
            const double x_l = j == 0 ? xl : xv[j - 1];
            const double x_r = j == kItemVx - 1 ? xr : xv[j + 1];
            y = eps * xa;
            if (has_dn)     y = __fma_rn((double)w_dn, xa - xdn[j], y);
            if (has_up)     y = __fma_rn((double)w_up, xa - xup[j], y);
            if (c < nc - 1) y = __fma_rn((double)w_rt, xa - x_r, y);
            if (c > 0)      y = __fma_rn((double)w_lf, xa - x_l, y);
        }
        V rs = (V)(bv - y);
        if constexpr (sizeof(V) == 8) {
            V ds = (V)d;
            double z = (double)rs / (double)ds;
            acc = __fma_rn((double)rs, z, acc);
            rv[j] = rs;
            zv[j] = (V)z;
            if (write_diag) dv[j] = ds;
        } else {
            const float d32 = __fadd_rn(ws32, kLapEpsF);
            rv[j] = rs;
            zf[j] = __fmul_rn((float)rs, rcp_pre(d32));
            zv[j] = rs;
            if (write_diag) dv[j] = (V)d32;
        }
    }
    if constexpr (sizeof(V) == 4) acc = dot4_df((const float *)rv, zf);
    if (sizeof(V) == 8) st4(rr + prow + q.c0, rv);
    st4(zout + T.pix + prow + q.c0, zv);
    if (write_diag) st4(dg + prow + q.c0, dv);
    if (bvp && write_diag) st4(bvp, bst);
    if (zero_x) {
        st4(x + prow + q.c0, xv);
        if (P.dx) {
            const float zero[4] = {0.f, 0.f, 0.f, 0.f};
            st4(P.dx + T.pix + prow + q.c0, zero);
        }
    }
    return acc;
}

/* ── TMA-staged stencil and update passes ─────────────────────────────────
 * Every plane of a job is one 2-D array (all tiles stacked row-wise with a
 * common pitch), described by a TMA tensor map.  A block walks its work items
 * through an NS-stage shared-memory ring: one thread issues the item's 2-D
 * tensor copies (cp.async.bulk.tensor, no multicast) into a free stage and
 * arms the stage's mbarrier with the box bytes; all threads compute on the
 * oldest stage.  Boxes start at column c0b - 4 (16-byte aligned) and may
 * reach outside the array; the TMA unit fills those elements with zeros and
 * the kernels never read values outside the tile. */
constexpr int kSegW = kItemBx + 8;        /* stencil box width: 4 columns each side */
constexpr int kWrW = kItemBx + 4;         /* right-arc box incl. the left neighbour */

struct SolveMaps {
    /* FP64 two-pass form */
    CUtensorMap zA, p0A, p1A, wdA, wrA;        /* stencil pass boxes (zA: z buffer 0) */
    CUtensorMap xB, p0B, p1B, qB, rB, dB;      /* update pass boxes                   */
    /* mixed single-synchronisation pass (zA, p0A, p1A shared; xB = dx) */
    CUtensorMap zS1, qS0, qS1;                 /* z buffer 1, q buffers 0 and 1 (halo boxes) */
    CUtensorMap wdS, wrS;                      /* arc weights for the halo's diag as well    */
};

__host__ __device__ constexpr size_t al128(size_t b) { return (b + 127) & ~(size_t)127; }

/* FP64 stencil-pass stage: z and p_old with halo, down and right arc weights */
struct StageA {
    static constexpr size_t kVec = al128((size_t)(kItemBy + 2) * kSegW * sizeof(double));
    static constexpr size_t kWd = al128((size_t)(kItemBy + 1) * kItemBx * sizeof(float));
    static constexpr size_t kWr = al128((size_t)kItemBy * kWrW * sizeof(float));
    static constexpr size_t kBytes = 2 * kVec + kWd + kWr;
    static constexpr uint32_t kTx = (uint32_t)(2 * (kItemBy + 2) * kSegW * sizeof(double) +
                                               (kItemBy + 1) * kItemBx * 4 + kItemBy * kWrW * 4);
};
/* FP64 update-pass stage: x, p, q, r, diag */
struct StageB {
    static constexpr size_t kX = (size_t)kItemBy * kItemBx * sizeof(double);
    static constexpr size_t kV = (size_t)kItemBy * kItemBx * sizeof(double);
    static constexpr size_t kBytes = kX + 4 * kV;
    static constexpr uint32_t kTxFull = (uint32_t)(kX + 4 * kV);
    static constexpr uint32_t kTxX = (uint32_t)(kX + kV);
};
/* Mixed single-synchronisation stage.  z, q, p_old and the right-arc
 * weights as 18 x 72 boxes (rows r0b-1 .. r0b+16, columns c0b-4 .. c0b+67),
 * the down-arc weights as a 19 x 72 box starting one row higher (the diag of
 * a halo pixel in row r0b-1 needs the arc above it), and the item's dx. */
struct StageS {
    static constexpr int kBoxH = kItemBy + 2;
    static constexpr int kWdH = kItemBy + 3;
    static constexpr size_t kBox = al128((size_t)kBoxH * kSegW * 4);
    static constexpr size_t kWd = al128((size_t)kWdH * kSegW * 4);
    static constexpr size_t kDx = (size_t)kItemBy * kItemBx * 4;
    static constexpr size_t oZ = 0, oQ = kBox, oPO = 2 * kBox, oWR = 3 * kBox, oWD = 4 * kBox;
    static constexpr size_t oDX = 4 * kBox + kWd;
    static constexpr size_t kBytes = al128(oDX + kDx);
    static constexpr uint32_t kTxBox = (uint32_t)(kBoxH * kSegW * 4);
    static constexpr uint32_t kTxWd = (uint32_t)(kWdH * kSegW * 4);
    static constexpr uint32_t kTxDx = (uint32_t)(kItemBy * kItemBx * 4);
};
template <typename V> __host__ __device__ constexpr size_t stage_bytes()
{
    return sizeof(V) == 4 ? StageS::kBytes
                          : al128(StageA::kBytes > StageB::kBytes ? StageA::kBytes : StageB::kBytes);
}
/* p_new of an item with its halo ring, rows of kSegW elements laid out like
 * the staged boxes (column 0 <-> c0b - 4), so own columns start 16-byte
 * aligned at column 4 */
template <typename V> __host__ __device__ constexpr size_t pn_bytes()
{
    return al128((size_t)kHaloH * kSegW * sizeof(V));
}
/* NS: stages of the shared-memory ring (items in flight per block) */
template <typename V, int NS> __host__ __device__ constexpr size_t solve_smem_bytes()
{
    /* mixed mode double-buffers Pn by item parity */
    return NS * stage_bytes<V>() + (sizeof(V) == 4 ? 2 : 1) * pn_bytes<V>() + 128;
}


__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}
/* one bounded test of a phase; a thread whose phase is not complete may be
 * suspended for up to 20 us (the suspend-time hint) instead of returning at
 * once, so waiting warps do not take issue slots from computing ones */
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}
/* bounded wait for a stage; on timeout the error status is raised and the
 * next grid barrier ends the kernel */
__device__ __forceinline__ void mbar_wait(uint64_t *bar, uint32_t parity, SolverCtl *ctl,
                                          long long timeout_ns)
{
    if (mbar_try(bar, parity)) return;
    unsigned long long t0 = globaltimer();
    for (long long i = 1;; ++i) {
        if (mbar_try(bar, parity)) return;
        if ((i & 255) == 0) {
            if ((long long)(globaltimer() - t0) > timeout_ns || i > (1LL << 30)) {
                atomicExch(&ctl->err, 2);
                return;
            }
        }
    }
}
__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

/* ── FP64 two-pass form ───────────────────────────────────────────────── */
__device__ __forceinline__ void issue_a(const TileDesc &T, int li, const SolveMaps &M, int pold_sel,
                                        bool first, char *stage, uint64_t *bar)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const int y = T.row0 + r0b;
    char *Z = stage;
    char *PO = stage + StageA::kVec;
    char *WD = PO + StageA::kVec;
    char *WR = WD + StageA::kWd;
    uint32_t tx = StageA::kTx - (first ? (uint32_t)((kItemBy + 2) * kSegW * sizeof(double)) : 0u);
    mbar_expect(bar, tx);
    tma_load_2d(Z, &M.zA, c0b - 4, y - 1, bar);
    if (!first) tma_load_2d(PO, pold_sel ? &M.p1A : &M.p0A, c0b - 4, y - 1, bar);
    tma_load_2d(WD, &M.wdA, c0b, y - 1, bar);
    tma_load_2d(WR, &M.wrA, c0b - 4, y, bar);
}

/* shared-memory vector access of 4 consecutive elements (16-byte aligned) */
__device__ __forceinline__ void sld4(const float *p, float v[4])
{
    float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void sld4(const double *p, double v[4])
{
    double2 a = reinterpret_cast<const double2 *>(p)[0];
    double2 b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

/* stencil pass on a staged item (FP64, the oracle's operation order):
 * p_new = z + beta p_old (own + halo ring), q = A p_new, thread partial of
 * p.q */
__device__ double compute_a(const TileDesc &T, int li, const SolverPlanes &P, double *pnew_all,
                            bool first, double beta, const char *stage, double *Pn)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const double *Z = (const double *)stage;
    const double *PO = (const double *)(stage + StageA::kVec);
    const float *WD = (const float *)(stage + 2 * StageA::kVec);
    const float *WR = (const float *)(stage + 2 * StageA::kVec + StageA::kWd);
    const int nr = T.nr, nc = T.nc;
    const int ty = threadIdx.x / kItemTx, tx = threadIdx.x % kItemTx;
    const int r = r0b + ty, c0 = c0b + tx * kItemVx;
    const bool own = r < nr && c0 < nc;
    /* own p_new: row ty+1, columns 4 + 4 tx .. +3 */
    double pn[4] = {0.0, 0.0, 0.0, 0.0};
    const int so = (ty + 1) * kSegW + 4 + tx * kItemVx;
    if (own) {
        double zv[4], pv[4] = {0.0, 0.0, 0.0, 0.0};
        sld4(Z + so, zv);
        if (!first) sld4(PO + so, pv);
#pragma unroll
        for (int j = 0; j < kItemVx; ++j)
            if (c0 + j < nc) pn[j] = first ? zv[j] : __fma_rn(beta, pv[j], zv[j]);
    }
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) Pn[so + j] = pn[j];
    /* halo ring: rows above/below (64 each), columns left/right (16 each) */
    if (threadIdx.x < 2 * kItemBx + 2 * kItemBy) {
        int h = threadIdx.x, i, jc;
        if (h < kItemBx) { i = 0; jc = 4 + h; }
        else if (h < 2 * kItemBx) { i = kItemBy + 1; jc = 4 + h - kItemBx; }
        else if (h < 2 * kItemBx + kItemBy) { i = 1 + h - 2 * kItemBx; jc = 3; }
        else { i = 1 + h - 2 * kItemBx - kItemBy; jc = 4 + kItemBx; }
        int gr = r0b - 1 + i, gc = c0b - 4 + jc;
        double v = 0.0;
        if (gr >= 0 && gr < nr && gc >= 0 && gc < nc) {
            int sidx = i * kSegW + jc;
            v = first ? Z[sidx] : __fma_rn(beta, PO[sidx], Z[sidx]);
        }
        Pn[i * kSegW + jc] = v;
    }
    __syncthreads();
    double acc = 0.0;
    if (own) {
        double up[4], dn[4], qv[4] = {0.0, 0.0, 0.0, 0.0};
        float wdn[4], wup[4], wrt[4];
        sld4(Pn + so - kSegW, up);
        sld4(Pn + so + kSegW, dn);
        double lf = Pn[so - 1], rt = Pn[so + 4];
        sld4(WD + (ty + 1) * kItemBx + tx * kItemVx, wdn);
        sld4(WD + ty * kItemBx + tx * kItemVx, wup);
        sld4(WR + ty * kWrW + tx * kItemVx + 4, wrt);
        float wlf = WR[ty * kWrW + tx * kItemVx + 3];
#pragma unroll
        for (int j = 0; j < kItemVx; ++j) {
            int c = c0 + j;
            if (c >= nc) continue;
            double xl = j == 0 ? lf : pn[j - 1];
            double xr = j == kItemVx - 1 ? rt : pn[j + 1];
            float wl = j == 0 ? wlf : wrt[j - 1];
            double xa = pn[j];
            double y = (double)kLapEpsF * xa;
            if (r < nr - 1) y = __fma_rn((double)wdn[j], xa - dn[j], y);
            if (r > 0)      y = __fma_rn((double)wup[j], xa - up[j], y);
            if (c < nc - 1) y = __fma_rn((double)wrt[j], xa - xr, y);
            if (c > 0)      y = __fma_rn((double)wl, xa - xl, y);
            qv[j] = y;
            acc = __fma_rn(pn[j], y, acc);
        }
        size_t o = T.pix + (size_t)r * T.pitch + c0;
        st4(pnew_all + o, pn);
        st4((double *)P.q + o, qv);
    }
    return acc;
}

__device__ __forceinline__ void issue_b(const TileDesc &T, int li, const SolveMaps &M, int pnew_sel,
                                        bool update_r, char *stage, uint64_t *bar)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const int y = T.row0 + r0b;
    char *X = stage;
    char *PB = X + StageB::kX;
    char *QB = PB + StageB::kV;
    char *RB = QB + StageB::kV;
    char *DB = RB + StageB::kV;
    mbar_expect(bar, update_r ? StageB::kTxFull : StageB::kTxX);
    tma_load_2d(X, &M.xB, c0b, y, bar);
    tma_load_2d(PB, pnew_sel ? &M.p1B : &M.p0B, c0b, y, bar);
    if (update_r) {
        tma_load_2d(QB, &M.qB, c0b, y, bar);
        tma_load_2d(RB, &M.rB, c0b, y, bar);
        tma_load_2d(DB, &M.dB, c0b, y, bar);
    }
}

/* update pass (FP64): x += alpha p; r -= alpha q; z = r / diag; partial r.z */
__device__ double compute_b(const TileDesc &T, int li, const SolverPlanes &P, double alpha,
                            bool update_r, const char *stage)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const double *X = (const double *)stage;
    const double *PB = (const double *)(stage + StageB::kX);
    const double *QB = PB + kItemBy * kItemBx;
    const double *RB = QB + kItemBy * kItemBx;
    const double *DB = RB + kItemBy * kItemBx;
    const int ty = threadIdx.x / kItemTx, tx = threadIdx.x % kItemTx;
    const int r = r0b + ty, c0 = c0b + tx * kItemVx;
    if (r >= T.nr || c0 >= T.nc) return 0.0;
    const int s0 = ty * kItemBx + tx * kItemVx;
    const size_t o = T.pix + (size_t)r * T.pitch + c0;
    double acc = 0.0;
    double xv[4], pv[4], qv[4], rv[4] = {0.0, 0.0, 0.0, 0.0}, dv[4], zv[4] = {0.0, 0.0, 0.0, 0.0};
    sld4(X + s0, xv);
    sld4(PB + s0, pv);
    if (update_r) {
        sld4(QB + s0, qv);
        sld4(RB + s0, rv);
        sld4(DB + s0, dv);
    }
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        if (c0 + j >= T.nc) continue;
        xv[j] = __fma_rn(alpha, pv[j], xv[j]);
        if (update_r) {
            double rn = __fma_rn(-alpha, qv[j], rv[j]);
            rv[j] = rn;
            double z = rn / dv[j];
            zv[j] = z;
            acc = __fma_rn(rn, z, acc);
        }
    }
    st4(P.x + o, xv);
    if (update_r) {
        st4((double *)P.r + o, rv);
        st4((double *)P.z + o, zv);
    }
    return acc;
}

/* ── mixed single-synchronisation pass ─────────────────────────────────────
 * zsel: z buffer to read (the pass writes the other); ksel: p_old and q_old
 * buffer (p and q of the previous pass; the pass writes the other); first:
 * no p_old (first pass of a solve); fresh: z comes straight from a residual
 * (solve start or replacement), so there is no update to apply and no
 * q_old or dx to stage. */
__device__ __forceinline__ void issue_s(const TileDesc &T, int li, const SolveMaps &M, int zsel,
                                        int ksel, bool first, bool fresh, char *stage,
                                        uint64_t *bar)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const int y = T.row0 + r0b;
    uint32_t tx = 2 * StageS::kTxBox + StageS::kTxWd;
    if (!first) tx += StageS::kTxBox;
    if (!fresh) tx += StageS::kTxBox + StageS::kTxDx;
    mbar_expect(bar, tx);
    tma_load_2d(stage + StageS::oZ, zsel ? &M.zS1 : &M.zA, c0b - 4, y - 1, bar);
    if (!fresh) tma_load_2d(stage + StageS::oQ, ksel ? &M.qS1 : &M.qS0, c0b - 4, y - 1, bar);
    if (!first) tma_load_2d(stage + StageS::oPO, ksel ? &M.p1A : &M.p0A, c0b - 4, y - 1, bar);
    tma_load_2d(stage + StageS::oWR, &M.wrS, c0b - 4, y - 1, bar);
    tma_load_2d(stage + StageS::oWD, &M.wdS, c0b - 4, y - 2, bar);
    if (!fresh) tma_load_2d(stage + StageS::oDX, &M.xB, c0b, y, bar);
}

/* One item of the mixed pass, in two halves around the block barrier.
 * FP32 arithmetic for the vector updates and the stencil (IEEE
 * round-to-nearest per operation), FP64-accurate dots (dot4_df per thread):
 * acc[0] r.z of the updated residual (when not fresh), acc[1] p.q, acc[2]
 * z.q, acc[3] q.(M^-1 q).  The residual plane holds r; z = M^-1 r is formed
 * on the fly with M^-1 = rcp_pre(diag32) of the staged weights.
 * compute_s1: the previous iteration's update and the fold p' = z' + beta
 * p_old of the own pixels and the halo ring, into Pn; r', z' and M^-1 of
 * the own pixels stay in registers for compute_s2, which computes q = A p'
 * from Pn and the staged weights, and all four dots (two at a time). */
struct ItemS {
    const float *R, *Q, *PO, *WR, *WD, *DX;
    int r0b, c0b, ty, tx, r, c0, so, sd;
    bool own;
    bool in;   /* every pixel of the item has all four arcs inside the tile */
    size_t o;
};

__device__ __forceinline__ ItemS item_s(const TileDesc &T, int li, const char *stage)
{
    ItemS I;
    I.r0b = (li / T.nbx) * kItemBy;
    I.c0b = (li % T.nbx) * kItemBx;
    I.R = (const float *)(stage + StageS::oZ);
    I.Q = (const float *)(stage + StageS::oQ);
    I.PO = (const float *)(stage + StageS::oPO);
    I.WR = (const float *)(stage + StageS::oWR);
    I.WD = (const float *)(stage + StageS::oWD);
    I.DX = (const float *)(stage + StageS::oDX);
    I.ty = threadIdx.x / kItemTx;
    I.tx = threadIdx.x % kItemTx;
    I.r = I.r0b + I.ty;
    I.c0 = I.c0b + I.tx * kItemVx;
    I.own = I.r < T.nr && I.c0 < T.nc;
    I.in = I.r0b >= 1 && I.r0b + kItemBy <= T.nr - 1 && I.c0b >= 1 && I.c0b + kItemBx <= T.nc - 1;
    /* halo-box coordinates: row i <-> pixel row r0b - 1 + i (the down-arc
     * box starts one row higher: its row i + 1 holds row r0b - 1 + i),
     * column jc <-> c0b - 4 + jc */
    I.so = (I.ty + 1) * kSegW + 4 + I.tx * kItemVx;
    I.sd = I.so + kSegW;                 /* wd(r, c) in the down-arc box */
    I.o = T.pix + (size_t)I.r * T.pitch + I.c0;
    return I;
}

__device__ __forceinline__ void compute_s1(const TileDesc &T, const ItemS &I, float *rnew_all,
                                           float *dx_all, bool first, bool fresh, float alphaf,
                                           float betaf, float *Pn, float zn[4], float rd[4],
                                           float rv[4])
{
    const int nr = T.nr, nc = T.nc;
    float pn[4] = {0.f, 0.f, 0.f, 0.f};
    if (I.own) {
        float wdn[4], wup[4], wrt[4];
        sld4(I.WD + I.sd, wdn);
        sld4(I.WD + I.sd - kSegW, wup);
        sld4(I.WR + I.so, wrt);
        const float wlf = I.WR[I.so - 1];
        float qv[4] = {0.f, 0.f, 0.f, 0.f}, pv[4] = {0.f, 0.f, 0.f, 0.f};
        float dxv[4] = {0.f, 0.f, 0.f, 0.f};
        sld4(I.R + I.so, rv);
        if (!fresh) {
            sld4(I.Q + I.so, qv);
            sld4(I.DX + I.ty * kItemBx + I.tx * kItemVx, dxv);
        }
        if (!first) sld4(I.PO + I.so, pv);
        if (I.in) {
            /* all four arcs in the tile: diag32's sum without the tests (a
             * weight that is not positive adds +0, which diag32 skips), and
             * the updates two pixels per instruction */
#pragma unroll
            for (int j = 0; j < kItemVx; j += 2) {
                const float2 dn = pf2(fmaxf(wdn[j], 0.f), fmaxf(wdn[j + 1], 0.f));
                const float2 up = pf2(fmaxf(wup[j], 0.f), fmaxf(wup[j + 1], 0.f));
                const float2 rt = pf2(fmaxf(wrt[j], 0.f), fmaxf(wrt[j + 1], 0.f));
                const float2 lf = pf2(fmaxf(j == 0 ? wlf : wrt[j - 1], 0.f), fmaxf(wrt[j], 0.f));
                const float2 d = __fadd2_rn(__fadd2_rn(__fadd2_rn(__fadd2_rn(dn, up), rt), lf),
                                            pf2(kLapEpsF, kLapEpsF));
                const float2 m = pf2(rcp_pre(d.x), rcp_pre(d.y));
                float2 r2 = pf2(rv[j], rv[j + 1]);
                const float2 p2 = pf2(pv[j], pv[j + 1]);
                if (!fresh) {
                    r2 = __ffma2_rn(pf2(-alphaf, -alphaf), pf2(qv[j], qv[j + 1]), r2);
                    const float2 x2 = __ffma2_rn(pf2(alphaf, alphaf), p2,
                                                 pf2(dxv[j], dxv[j + 1]));
                    dxv[j] = x2.x;
                    dxv[j + 1] = x2.y;
                }
                const float2 z2 = __fmul2_rn(r2, m);
                const float2 f2v = first ? z2 : __ffma2_rn(pf2(betaf, betaf), p2, z2);
                rv[j] = r2.x; rv[j + 1] = r2.y;
                rd[j] = m.x; rd[j + 1] = m.y;
                zn[j] = z2.x; zn[j + 1] = z2.y;
                pn[j] = f2v.x; pn[j + 1] = f2v.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < kItemVx; ++j) {
                const int c = I.c0 + j;
                if (c >= nc) {
                    rv[j] = 0.f;
                    continue;
                }
                rd[j] = rcp_pre(diag32(I.r, c, nr, nc, wdn[j], wup[j], wrt[j],
                                       j == 0 ? wlf : wrt[j - 1]));
                if (!fresh) {
                    rv[j] = __fmaf_rn(-alphaf, qv[j], rv[j]);
                    dxv[j] = __fmaf_rn(alphaf, pv[j], dxv[j]);
                }
                zn[j] = __fmul_rn(rv[j], rd[j]);
                pn[j] = first ? zn[j] : __fmaf_rn(betaf, pv[j], zn[j]);
            }
        }
        if (!fresh) {
            st4(dx_all + I.o, dxv);
            st4(rnew_all + I.o, rv);
        }
    }
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) Pn[I.so + j] = pn[j];
    /* halo ring: the same update and fold, so neighbours agree bit for bit;
     * done by the last 160 threads (warps 3-7), as warps 0-3 store the
     * previous item's partials after the barrier */
    constexpr int kHalo = 2 * kItemBx + 2 * kItemBy;
    if ((int)threadIdx.x >= kItemThreads - kHalo) {
        int h = (int)threadIdx.x - (kItemThreads - kHalo), i, jc;
        if (h < kItemBx) { i = 0; jc = 4 + h; }
        else if (h < 2 * kItemBx) { i = kItemBy + 1; jc = 4 + h - kItemBx; }
        else if (h < 2 * kItemBx + kItemBy) { i = 1 + h - 2 * kItemBx; jc = 3; }
        else { i = 1 + h - 2 * kItemBx - kItemBy; jc = 4 + kItemBx; }
        const int gr = I.r0b - 1 + i, gc = I.c0b - 4 + jc;
        float v = 0.f;
        if (gr >= 0 && gr < nr && gc >= 0 && gc < nc) {
            const int sidx = i * kSegW + jc;
            const float m = rcp_pre(diag32(gr, gc, nr, nc, I.WD[sidx + kSegW], I.WD[sidx],
                                           I.WR[sidx], I.WR[sidx - 1]));
            const float rr = fresh ? I.R[sidx] : __fmaf_rn(-alphaf, I.Q[sidx], I.R[sidx]);
            const float z = __fmul_rn(rr, m);
            v = first ? z : __fmaf_rn(betaf, I.PO[sidx], z);
        }
        Pn[i * kSegW + jc] = v;
    }
}

__device__ __forceinline__ void compute_s2(const TileDesc &T, const ItemS &I, float *pnew_all,
                                           float *qnew_all, const float *Pn, const float zn[4],
                                           const float rd[4], const float rv[4], bool fresh,
                                           double acc[kNComp])
{
    if (!I.own) return;
    const int nr = T.nr, nc = T.nc, r = I.r, so = I.so;
    float pn[4], up[4], dn[4], wdn[4], wup[4], wrt[4], qv[4] = {0.f, 0.f, 0.f, 0.f};
    sld4(Pn + so, pn);
    sld4(Pn + so - kSegW, up);
    sld4(Pn + so + kSegW, dn);
    const float lf = Pn[so - 1], rt = Pn[so + 4];
    sld4(I.WD + I.sd, wdn);
    sld4(I.WD + I.sd - kSegW, wup);
    sld4(I.WR + so, wrt);
    const float wlf = I.WR[so - 1];
    float mq[4] = {0.f, 0.f, 0.f, 0.f};
    if (I.in) {
        /* interior: the stencil without the tile-edge tests, two pixels per
         * instruction (the same operations in the same order per pixel) */
#pragma unroll
        for (int j = 0; j < kItemVx; j += 2) {
            const float2 xa = pf2(pn[j], pn[j + 1]);
            const float2 xl = pf2(j == 0 ? lf : pn[j - 1], pn[j]);
            const float2 xr = pf2(pn[j + 1], j + 2 == kItemVx ? rt : pn[j + 2]);
            const float2 wl = pf2(j == 0 ? wlf : wrt[j - 1], wrt[j]);
            float2 y = __fmul2_rn(pf2(kLapEpsF, kLapEpsF), xa);
            y = __ffma2_rn(pf2(wdn[j], wdn[j + 1]), psub(xa, pf2(dn[j], dn[j + 1])), y);
            y = __ffma2_rn(pf2(wup[j], wup[j + 1]), psub(xa, pf2(up[j], up[j + 1])), y);
            y = __ffma2_rn(pf2(wrt[j], wrt[j + 1]), psub(xa, xr), y);
            y = __ffma2_rn(wl, psub(xa, xl), y);
            const float2 m = __fmul2_rn(y, pf2(rd[j], rd[j + 1]));
            qv[j] = y.x; qv[j + 1] = y.y;
            mq[j] = m.x; mq[j + 1] = m.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < kItemVx; ++j) {
            const int c = I.c0 + j;
            if (c >= nc) {
                pn[j] = 0.f;
                continue;
            }
            const float xl = j == 0 ? lf : pn[j - 1];
            const float xr = j == kItemVx - 1 ? rt : pn[j + 1];
            const float wl = j == 0 ? wlf : wrt[j - 1];
            const float xa = pn[j];
            float y = __fmul_rn(kLapEpsF, xa);
            if (r < nr - 1) y = __fmaf_rn(wdn[j], __fsub_rn(xa, dn[j]), y);
            if (r > 0)      y = __fmaf_rn(wup[j], __fsub_rn(xa, up[j]), y);
            if (c < nc - 1) y = __fmaf_rn(wrt[j], __fsub_rn(xa, xr), y);
            if (c > 0)      y = __fmaf_rn(wl, __fsub_rn(xa, xl), y);
            qv[j] = y;
            mq[j] = __fmul_rn(y, rd[j]);
        }
    }
    dot4_df2(pn, qv, zn, qv, acc[1], acc[2]);
    if (fresh) acc[3] = dot4_df(qv, mq);
    else dot4_df2(qv, mq, rv, zn, acc[3], acc[0]);
    st4(pnew_all + I.o, pn);
    st4(qnew_all + I.o, qv);
}

/* mixed precision: fold the FP32 increment into the FP64 solution, optionally
 * applying this iteration's update first (x = x + (dx + alpha p), dx = 0) */
template <typename V>
__device__ void phase_fold(const TileDesc &T, int li, const SolverPlanes &P, const V *pnew_all,
                           bool with_update, double alpha)
{
    ItemXY q = item_xy(T, li);
    if (q.r >= T.nr || q.c0 >= T.nc) return;
    const size_t o = T.pix + (size_t)q.r * T.pitch + q.c0;
    float dxv[4], pv[4];
    double xv[4];
    ld4(P.dx + o, dxv);
    ld4(P.x + o, xv);
    if (with_update) ld4((const float *)pnew_all + o, pv);
    const float alphaf = (float)alpha;
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        if (q.c0 + j >= T.nc) continue;
        float d = with_update ? __fmaf_rn(alphaf, pv[j], dxv[j]) : dxv[j];
        xv[j] = xv[j] + (double)d;
    }
    const float zero[4] = {0.f, 0.f, 0.f, 0.f};
    st4(P.x + o, xv);
    st4(P.dx + o, zero);
}

/* ── IRLS reweight (A13): w = w0 / sqrt(e^2 + delta^2) ───────────────────── */
template <typename V>
__device__ void phase_rw(const TileDesc &T, int li, const SolverPlanes &P, float delta)
{
    ItemXY q = item_xy(T, li);
    if (q.r >= T.nr || q.c0 >= T.nc) return;
    const double *x = P.x + T.pix;
    const double dd = (double)delta * (double)delta;
    const int r = q.r, nr = T.nr, nc = T.nc, pitch = T.pitch, pp = T.ph_pitch;
    size_t prow = (size_t)r * pitch;
    float wdo[4], wro[4];
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        int c = q.c0 + j;
        wdo[j] = 0.0f; wro[j] = 0.0f;
        if (c >= nc) continue;
        size_t pi = prow + c, gi = (size_t)r * pp + c;
        double xa = ldc(x + pi);
        float pa = __ldg(T.ph + gi);
        if (r < nr - 1) {
            float w0 = __ldg(P.w0d + T.pix + pi);
            if (w0 > 0.0f) {
                float g = lap_wrap_pi(__ldg(T.ph + gi + pp) - pa);
                double e = (ldc(x + pi + pitch) - xa) - (double)g;
                wdo[j] = (float)((double)w0 / __dsqrt_rn(__fma_rn(e, e, dd)));
            }
        }
        if (c < nc - 1) {
            float w0 = __ldg(P.w0r + T.pix + pi);
            if (w0 > 0.0f) {
                float g = lap_wrap_pi(__ldg(T.ph + gi + 1) - pa);
                double e = (ldc(x + pi + 1) - xa) - (double)g;
                wro[j] = (float)((double)w0 / __dsqrt_rn(__fma_rn(e, e, dd)));
            }
        }
    }
    st4(P.wd + T.pix + prow + q.c0, wdo);
    st4(P.wr + T.pix + prow + q.c0, wro);
}

/* ── anchor + congruence (A14) ────────────────────────────────────────── */
template <typename V>
__device__ void phase_final(const TileDesc &T, int li, const SolverPlanes &P)
{
    ItemXY q = item_xy(T, li);
    if (q.r >= T.nr || q.c0 >= T.nc) return;
    const double *x = P.x + T.pix;
    double off = (double)__ldg(T.ph) - ldc(x);
    size_t prow = (size_t)q.r * T.pitch;
    float uo[4] = {0.f, 0.f, 0.f, 0.f}, co[4] = {0.f, 0.f, 0.f, 0.f};
    int ko[4] = {0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        int c = q.c0 + j;
        if (c >= T.nc) continue;
        float ph = __ldg(T.ph + (size_t)q.r * T.ph_pitch + c);
        double u = ldc(x + prow + c) + off;
        double d = u - (double)ph;
        double k = rint(d / kTwoPiD);
        co[j] = (float)u;
        uo[j] = __fmaf_rn(kTwoPiF, (float)k, ph);
        ko[j] = (int)k;
    }
    *reinterpret_cast<float4 *>(P.unw + T.pix + prow + q.c0) = make_float4(uo[0], uo[1], uo[2], uo[3]);
    if (P.cyc)
        *reinterpret_cast<int4 *>(P.cyc + T.pix + prow + q.c0) = make_int4(ko[0], ko[1], ko[2], ko[3]);
    if (P.cont)
        *reinterpret_cast<float4 *>(P.cont + T.pix + prow + q.c0) = make_float4(co[0], co[1], co[2], co[3]);
}

/* ── work distribution ─────────────────────────────────────────────────────
 * At every phase each block takes an equal slice of the items of the tiles
 * that are still active (tile-major order), so tiles that converge late get
 * the whole GPU instead of the few blocks that own them.  The active flags
 * were published before the last grid barrier; every block computes the same
 * prefix sum of active item counts in shared memory.  Tile scalars are
 * reduced redundantly (and identically) by every block whose slice touches
 * the tile; the block whose slice holds the tile's first item is its owner
 * for the global active-tile count. */
constexpr int kMaxTiles = 1024;
constexpr int kCacheTiles = 16;

struct SliceCtl {
    int pre[kMaxTiles + 1];          /* exclusive prefix of counted item numbers */
    int s0, s1, t0, t1;              /* my slice in counted order, tiles it spans */
    int ncached;
    TileDesc d[kCacheTiles];
    double alpha[kCacheTiles], beta[kCacheTiles];
    int active[kCacheTiles];
};

__device__ __forceinline__ const TileDesc &stile(const SliceCtl &sc, const TileDesc *g, int t)
{
    int k = t - sc.t0;
    return (k >= 0 && k < sc.ncached) ? sc.d[k] : g[t];
}
__device__ __forceinline__ int sactive(const SliceCtl &sc, const TileState *st, int t)
{
    int k = t - sc.t0;
    return (k >= 0 && k < sc.ncached) ? sc.active[k] : __ldcg(&st[t].active);
}
__device__ __forceinline__ double sbeta(const SliceCtl &sc, const TileState *st, int t)
{
    int k = t - sc.t0;
    return (k >= 0 && k < sc.ncached) ? sc.beta[k] : __ldcg(&st[t].beta);
}
__device__ __forceinline__ double salpha(const SliceCtl &sc, const TileState *st, int t)
{
    int k = t - sc.t0;
    return (k >= 0 && k < sc.ncached) ? sc.alpha[k] : __ldcg(&st[t].alpha);
}
/* Every block touching a tile derives the same scalars; only the tile's owner
 * publishes them (hundreds of blocks storing one line serialise in L2 when a
 * single tile is left).  A block reads its own copy from the cache, or, for a
 * tile beyond the cache, from the global state it then writes itself. */
__device__ __forceinline__ bool scached(const SliceCtl &sc, int t)
{
    int k = t - sc.t0;
    return k >= 0 && k < sc.ncached;
}
__device__ __forceinline__ void sput(SliceCtl &sc, int t, const TileState &S)
{
    int k = t - sc.t0;
    if (k >= 0 && k < sc.ncached) {
        sc.active[k] = S.active;
        sc.alpha[k] = S.alpha;
        sc.beta[k] = S.beta;
    }
}

/* tile containing counted position p (pre[t] <= p < pre[t+1]) */
__device__ __forceinline__ int slice_tile(const SliceCtl &sc, int ntiles, int p)
{
    int lo = 0, hi = ntiles - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (sc.pre[mid] <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* Build the prefix sum of item counts (all tiles, or only the tiles active in
 * `st`) and this block's slice; caches the descriptors of the slice's tiles
 * and, with `st`, their scalars. */
__device__ void setup_slice(SliceCtl &sc, const TileDesc *tiles, const TileState *st,
                            int ntiles, double *swd)
{
    int *sw = reinterpret_cast<int *>(swd);
    const int per = (ntiles + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per;
    int loc = 0;
    for (int k = 0; k < per; ++k) {
        int t = b0 + k;
        if (t < ntiles && (!st || __ldcg(&st[t].active))) loc += tiles[t].nitems;
    }
    /* block exclusive scan of loc */
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = loc;
    for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    __syncthreads();
    if (lane == 31) sw[w] = x;
    __syncthreads();
    if (w == 0) {
        int v = lane < (int)(blockDim.x >> 5) ? sw[lane] : 0;
        for (int off = 1; off < 32; off <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, v, off);
            if (lane >= off) v += y;
        }
        sw[lane] = v;
    }
    __syncthreads();
    int run = x - loc + (w > 0 ? sw[w - 1] : 0);
    for (int k = 0; k < per; ++k) {
        int t = b0 + k;
        if (t < ntiles) {
            sc.pre[t] = run;
            if (!st || __ldcg(&st[t].active)) run += tiles[t].nitems;
        }
    }
    if (threadIdx.x == blockDim.x - 1) sc.pre[ntiles] = run;
    __syncthreads();
    if (threadIdx.x == 0) {
        int total = sc.pre[ntiles];
        sc.s0 = (int)((long long)blockIdx.x * total / gridDim.x);
        sc.s1 = (int)((long long)(blockIdx.x + 1) * total / gridDim.x);
        if (sc.s0 < sc.s1) {
            sc.t0 = slice_tile(sc, ntiles, sc.s0);
            sc.t1 = slice_tile(sc, ntiles, sc.s1 - 1);
        } else {
            sc.t0 = 0;
            sc.t1 = -1;
        }
        sc.ncached = min(max(sc.t1 - sc.t0 + 1, 0), kCacheTiles);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < sc.ncached; k += blockDim.x) {
        int t = sc.t0 + k;
        sc.d[k] = tiles[t];
        if (st) {
            sc.active[k] = __ldcg(&st[t].active);
            sc.alpha[k] = __ldcg(&st[t].alpha);
            sc.beta[k] = __ldcg(&st[t].beta);
        }
    }
    __syncthreads();
}

/* this block's items of tile t in counted order: [a, b) of local indices */
__device__ __forceinline__ void slice_items(const SliceCtl &sc, const TileDesc &T, int t, int &a,
                                            int &b)
{
    a = max(sc.s0, sc.pre[t]) - sc.pre[t];
    b = min(sc.s1, sc.pre[t] + T.nitems) - sc.pre[t];
}

/* position in the slice: counted position p, tile t */
struct Cursor {
    int p, t;
};

__device__ __forceinline__ Cursor cursor_active(Cursor c, const SliceCtl &sc, const TileDesc *g,
                                                const TileState *st, int ntiles)
{
    while (c.p < sc.s1) {
        while (c.t + 1 <= ntiles && sc.pre[c.t + 1] <= c.p) ++c.t;
        if (sactive(sc, st, c.t)) return c;
        c.p = sc.pre[c.t + 1];
    }
    return c;
}

/* run a staged FP64 pass over this block's slice.  KIND 0: the stencil
 * pass, KIND 1: the update pass.  NS items are in flight; the stage of
 * item k is refilled with item k+NS right after the barrier of item k's
 * reduction, which every thread reaches only after its last read of the
 * stage and Pn. */
template <int KIND, int NS>
__device__ void run_pass(const SliceCtl &sc, const TileDesc *gt, const TileState *st, int ntiles,
                         const SolverPlanes &P, const SolveMaps &M, int psel, double *pvec,
                         bool flag, double *part, double *tot, unsigned *cnt, double *sw,
                         double *s_bcast, int *s_flag, double *Pn, char *stages, uint64_t *bars,
                         uint32_t &parity, SolverCtl *ctl, long long timeout_ns)
{
    constexpr size_t SB = stage_bytes<double>();
    const bool red = KIND == 0 || flag;
    if (sc.s0 >= sc.s1) return;
    Cursor ci = cursor_active(Cursor{sc.s0, sc.t0}, sc, gt, st, ntiles);
    if (ci.p >= sc.s1) return;
    Cursor cc = ci;
    if (threadIdx.x == 0) {
        fence_async_global();
        fence_async_smem();
    }
    for (int k = 0; k < NS && ci.p < sc.s1; ++k) {
        if (threadIdx.x == 0) {
            const TileDesc &T = stile(sc, gt, ci.t);
            int li = ci.p - sc.pre[ci.t];
            if (KIND == 0) issue_a(T, li, M, psel, flag, stages + k * SB, bars + k);
            else issue_b(T, li, M, psel, flag, stages + k * SB, bars + k);
        }
        ci = cursor_active(Cursor{ci.p + 1, ci.t}, sc, gt, st, ntiles);
    }
    int done = 0;
    while (cc.p < sc.s1) {
        int s = done % NS;
        mbar_wait(bars + s, (parity >> s) & 1u, ctl, timeout_ns);
        parity ^= 1u << s;
        ++done;
        const TileDesc &T = stile(sc, gt, cc.t);
        int li = cc.p - sc.pre[cc.t];
        double acc;
        if (KIND == 0)
            acc = compute_a(T, li, P, pvec, flag, sbeta(sc, st, cc.t), stages + s * SB, Pn);
        else
            acc = compute_b(T, li, P, salpha(sc, st, cc.t), flag, stages + s * SB);
        double bs = block_sum_item(acc, sw + 8 * (done & 1));   /* contains the item barrier */
        if (threadIdx.x == 0) {
            if (red) part[T.item0 + li] = bs;
            if (ci.p < sc.s1) {
                fence_async_smem();
                const TileDesc &Tn = stile(sc, gt, ci.t);
                int ln = ci.p - sc.pre[ci.t];
                if (KIND == 0) issue_a(Tn, ln, M, psel, flag, stages + s * SB, bars + s);
                else issue_b(Tn, ln, M, psel, flag, stages + s * SB, bars + s);
            }
        }
        if (ci.p < sc.s1) ci = cursor_active(Cursor{ci.p + 1, ci.t}, sc, gt, st, ntiles);
        Cursor nx = cursor_active(Cursor{cc.p + 1, cc.t}, sc, gt, st, ntiles);
        if (red && (nx.p >= sc.s1 || nx.t != cc.t)) {
            int a, b;
            slice_items(sc, T, cc.t, a, b);
            seg_done(T, cc.t, b - a, part, tot, cnt, sw, s_bcast, s_flag);
        }
        cc = nx;
    }
    __syncthreads();
}

/* The mixed pass over this block's slice, staged like run_pass but with one
 * block barrier per item.  Pn and the warp partials alternate between two
 * buffers by item parity.  After the barrier of item k (between its two
 * halves), every thread has finished item k-1, so then one thread of warp
 * 7 refills item k-1's stage with item k-1+NS (the boxes of the next NS-1 items are in
 * flight while item k computes) and warps 0-3 form and store item k-1's
 * four partials (cross-warp sums, one component per warp).  Tile totals of the pass are formed at its
 * end, for every tile of the block's slice. */
/* cross-warp sum of component c of one item's eight warp partials (a fixed
 * three-level tree), stored as the item's partial; warp c calls it */
__device__ __forceinline__ void store_item_comp(const double (*red)[8], int c, double *part,
                                                int nitems, int item)
{
    const int lane = threadIdx.x & 31;
    double x = lane < kItemThreads / 32 ? red[c][lane] : 0.0;
    for (int off = kItemThreads / 64; off > 0; off >>= 1)
        x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) part[(size_t)c * nitems + item] = x;
}

template <int NS>
__device__ void run_pass_s(const SliceCtl &sc, const TileDesc *gt, const TileState *st, int ntiles,
                           int nitems, const SolveMaps &M, int zsel, int ksel, bool first,
                           bool fresh, float *pnew, float *rnew, float *qnew, float *dx,
                           double *part, double *tot, unsigned *cnt, double *sw,
                           double (*red)[kNComp][8], double *s_bcast, int *s_flag, float *Pn2,
                           char *stages, uint64_t *bars, uint32_t &parity, SolverCtl *ctl,
                           long long timeout_ns)
{
    constexpr size_t SB = stage_bytes<float>();
    constexpr size_t PNE = pn_bytes<float>() / sizeof(float);
    if (sc.s0 >= sc.s1) return;
    Cursor ci = cursor_active(Cursor{sc.s0, sc.t0}, sc, gt, st, ntiles);
    if (ci.p >= sc.s1) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    /* the issuing thread: warp 7, whose post-barrier work is lightest */
    const bool issuer = threadIdx.x == kItemThreads - 32;
    Cursor cc = ci;
    if (issuer) {
        fence_async_global();
        fence_async_smem();
    }
    for (int k = 0; k < NS && ci.p < sc.s1; ++k) {
        if (issuer)
            issue_s(stile(sc, gt, ci.t), ci.p - sc.pre[ci.t], M, zsel, ksel, first, fresh,
                    stages + k * SB, bars + k);
        ci = cursor_active(Cursor{ci.p + 1, ci.t}, sc, gt, st, ntiles);
    }
    int k = 0, prev = -1;   /* item number in the pass; partial index of item k-1 */
    while (cc.p < sc.s1) {
        const int s = k % NS;
        mbar_wait(bars + s, (parity >> s) & 1u, ctl, timeout_ns);
        parity ^= 1u << s;
        const TileDesc &T = stile(sc, gt, cc.t);
        const int li = cc.p - sc.pre[cc.t];
        const ItemS I = item_s(T, li, stages + s * SB);
        float *Pn = Pn2 + (k & 1) * PNE;
        double acc[kNComp] = {0.0, 0.0, 0.0, 0.0};
        float zn[4] = {0.f, 0.f, 0.f, 0.f}, rd[4] = {0.f, 0.f, 0.f, 0.f};
        float rv[4] = {0.f, 0.f, 0.f, 0.f};
        compute_s1(T, I, rnew, dx, first, fresh, (float)salpha(sc, st, cc.t),
                   (float)sbeta(sc, st, cc.t), Pn, zn, rd, rv);
        __syncthreads();
        if (prev >= 0) {
            if (ci.p < sc.s1) {
                if (issuer) {
                    const int sp = (k - 1) % NS;
                    fence_async_smem();
                    issue_s(stile(sc, gt, ci.t), ci.p - sc.pre[ci.t], M, zsel, ksel, first,
                            fresh, stages + sp * SB, bars + sp);
                }
                ci = cursor_active(Cursor{ci.p + 1, ci.t}, sc, gt, st, ntiles);
            }
            if (warp < kNComp) store_item_comp(red[(k - 1) & 1], warp, part, nitems, prev);
        }
        compute_s2(T, I, pnew, qnew, Pn, zn, rd, rv, fresh, acc);
        {
            const double v = warp_scatter4(acc);   /* lane 8c: the warp's component c */
            if ((lane & 7) == 0) red[k & 1][lane >> 3][warp] = v;
        }
        prev = T.item0 + li;
        ++k;
        cc = cursor_active(Cursor{cc.p + 1, cc.t}, sc, gt, st, ntiles);
    }
    __syncthreads();
    if (warp < kNComp) store_item_comp(red[(k - 1) & 1], warp, part, nitems, prev);
    __syncthreads();
    /* the block's partials of every active tile of its slice are stored */
    for (int t = sc.t0; t <= sc.t1; ++t) {
        if (sc.pre[t + 1] == sc.pre[t] || !sactive(sc, st, t)) continue;
        const TileDesc &T = stile(sc, gt, t);
        int a, b;
        slice_items(sc, T, t, a, b);
        if (b > a) seg_done4(T, t, b - a, part, nitems, tot, ntiles, cnt, sw, s_bcast, s_flag);
    }
}

/* state written by other blocks before the last grid barrier: read from L2 */
__device__ __forceinline__ TileState load_state(const TileState *p)
{
    TileState S;
    S.rz = __ldcg(&p->rz);
    S.rz0 = __ldcg(&p->rz0);
    S.thr = __ldcg(&p->thr);
    S.alpha = __ldcg(&p->alpha);
    S.beta = __ldcg(&p->beta);
    S.active = __ldcg(&p->active);
    S.iter = __ldcg(&p->iter);
    return S;
}


/* A tile leaves the solve: the owner block updates the active count and the
 * statistics (pixel-iterations, the pass's largest iteration count). */
__device__ __forceinline__ void tile_stop(TileState &S, const TileDesc &T, bool owner,
                                          SolverCtl *ctl)
{
    S.active = 0;
    if (owner && threadIdx.x == 0) {
        atomicSub(&ctl->n_active, 1);
        atomicAdd(&ctl->px_iters,
                  (unsigned long long)S.iter * (unsigned long long)((long long)T.nr * T.nc));
        atomicMax(&ctl->pass_max, S.iter);
    }
}

/* first scalars of a solve from the tile's initial r.z */
__device__ __forceinline__ TileState start_state(double rz, const SolveParams &sp)
{
    TileState S;
    S.rz = rz;
    S.rz0 = rz;
    S.thr = (double)sp.tol * (double)sp.tol * rz;
    S.alpha = 0.0;
    S.beta = 0.0;
    S.iter = 0;
    S.active = (rz > 0.0 && sp.max_iter > 0) ? 1 : 0;
    return S;
}

/* publish a tile's new scalars: the owner (or a block beyond its cache)
 * stores them; every block touching the tile caches its own copy */
__device__ __forceinline__ void put_state(SliceCtl &sc, TileState *dst, int t, const TileState &S,
                                          bool owner)
{
    if (threadIdx.x == 0) {
        if (owner || !scached(sc, t)) dst[t] = S;
        sput(sc, t, S);
    }
}

/* tiles not counted by a phase that slices over the active tiles of `from`
 * keep their inactive flag in `to` */
__device__ __forceinline__ void carry_inactive(const TileState *from, TileState *to, int ntiles)
{
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < ntiles; t += blockDim.x)
            if (!__ldcg(&from[t].active)) to[t].active = 0;
}

/* WLS = true: the WLS-mode instance (explicit arc targets / right-hand
 * side, optional warm start, no anchoring); a separate instantiation so the
 * main path's register allocation does not carry its extra inputs */
template <typename V, bool WLS, int NS, int MINB>
__global__ void __launch_bounds__(kItemThreads, MINB)
    k_solve(const TileDesc *__restrict__ tiles, const int *__restrict__ item_tile, int nitems,
            int ntiles, SolverPlanes P, TileState *st, double *part, SolverCtl *ctl,
            SolveParams sp, long long timeout_ns, const __grid_constant__ SolveMaps M)
{
    extern __shared__ __align__(128) char dsm_raw[];
    __shared__ double sw[32];
    __shared__ double red[2][kNComp][8];   /* mixed: warp partials by item parity */
    __shared__ double sgrp[kItemGroup][8];   /* warp sums of a group of items */
    __shared__ double s_bcast;
    __shared__ int s_flag;
    __shared__ __align__(8) uint64_t bars[NS];
    __shared__ SliceCtl sc;
    char *dsm = (char *)(((uintptr_t)dsm_raw + 127) & ~(uintptr_t)127);
    constexpr bool mixed = sizeof(V) == 4;
    V *pb[2] = {(V *)P.p0, (V *)P.p1};
    /* per-item partials (kNComp components, component-major) and published
     * tile totals, both double-buffered by phase parity, and the per-tile
     * item tickets */
    double *pbuf[2] = {part, part + (size_t)kNComp * nitems};
    double *tbuf[2] = {part + 2 * (size_t)kNComp * nitems,
                       part + 2 * (size_t)kNComp * nitems + (size_t)kNComp * ntiles};
    unsigned *tick = reinterpret_cast<unsigned *>(part + 2 * (size_t)kNComp * nitems +
                                                  2 * (size_t)kNComp * ntiles);
    V *Pn = (V *)(dsm + NS * stage_bytes<V>());
    /* FP64: z (written by the assembly); mixed: the residual r, double-
     * buffered in the z and r planes */
    V *zb[2] = {(V *)P.z, (V *)P.r};
    uint32_t parity = 0u;   /* phase bit per stage of the ring */
    (void)item_tile;
    if (threadIdx.x == 0) {
        for (int k = 0; k < NS; ++k) mbar_init(&bars[k]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int pc = 0;   /* phase counter selecting the partial buffer */

    for (int outer = 0; outer <= sp.n_irls; ++outer) {
        /* assemble b, diag; r = b - A x; partial r.z (all tiles) */
        setup_slice(sc, tiles, nullptr, ntiles, sw);
        for (int t = sc.t0; t <= sc.t1; ++t) {
            const TileDesc &T = stile(sc, tiles, t);
            int a, b;
            slice_items(sc, T, t, a, b);
            const bool zx = outer == 0 && !(WLS && sp.warm);
            item_partials(T, a, b, pbuf[pc & 1], sgrp,
                          [&](int li) { return phase_init<V, WLS>(T, li, P, zx, true, zb[0]); });
            if (b > a) seg_done(T, t, b - a, pbuf[pc & 1], tbuf[pc & 1], tick, sw, &s_bcast, &s_flag);
        }
        ++pc;
        if (!grid_sync(ctl, timeout_ns, !(outer == 0 && (int)blockIdx.x == sp.skip_block))) return;

        int it = 0;
        if constexpr (!mixed) {
            /* ── FP64: stencil pass + update pass per iteration ──
             * stA: scalars after the stencil-pass decisions, stB: after the
             * update-pass decisions; each phase reads one and writes the
             * other, so the active flags a phase slices on never change
             * under it */
            TileState *stA = st, *stB = st + ntiles;
            while (true) {
                double *pnew = (double *)pb[(it + 1) & 1];
                /* slice over the tiles active in the previous phase; reduce
                 * r.z, update the tile scalars, then the stencil pass */
                setup_slice(sc, tiles, it == 0 ? nullptr : stB, ntiles, sw);
                if (it > 0) carry_inactive(stB, stA, ntiles);
                for (int t = sc.t0; t <= sc.t1; ++t) {
                    const TileDesc &T = stile(sc, tiles, t);
                    if (sc.pre[t + 1] == sc.pre[t]) continue;          /* not counted */
                    const bool owner = sc.pre[t] >= sc.s0 && sc.pre[t] < sc.s1;
                    TileState S;
                    double tot = __ldcg(tbuf[(pc - 1) & 1] + t);
                    if (it == 0) {
                        S = start_state(tot, sp);
                        if (owner && threadIdx.x == 0 && S.active) atomicAdd(&ctl->n_active, 1);
                    } else {
                        S = load_state(stB + t);
                        S.iter += 1;
                        if (tot < S.thr || S.iter >= sp.max_iter) {
                            tile_stop(S, T, owner, ctl);
                        } else {
                            S.beta = tot / S.rz;
                            S.rz = tot;
                        }
                    }
                    put_state(sc, stA, t, S, owner);
                }
                __syncthreads();
                run_pass<0, NS>(sc, tiles, stA, ntiles, P, M, it & 1, pnew, it == 0, pbuf[pc & 1],
                            tbuf[pc & 1], tick, sw, &s_bcast, &s_flag, (double *)Pn, dsm, bars,
                            parity, ctl, timeout_ns);
                ++pc;
                if (!grid_sync(ctl, timeout_ns)) return;
                if (*(volatile int *)&ctl->snap <= 0) break;

                /* slice over the tiles active in the stencil pass; reduce
                 * p.q, alpha; then the update pass */
                setup_slice(sc, tiles, stA, ntiles, sw);
                carry_inactive(stA, stB, ntiles);
                for (int t = sc.t0; t <= sc.t1; ++t) {
                    const TileDesc &T = stile(sc, tiles, t);
                    if (sc.pre[t + 1] == sc.pre[t]) continue;
                    const bool owner = sc.pre[t] >= sc.s0 && sc.pre[t] < sc.s1;
                    TileState S = load_state(stA + t);
                    double pq = __ldcg(tbuf[(pc - 1) & 1] + t);
                    if (pq <= 0.0) {
                        tile_stop(S, T, owner, ctl);
                        S.alpha = 0.0;
                    } else {
                        S.alpha = S.rz / pq;
                    }
                    put_state(sc, stB, t, S, owner);
                }
                __syncthreads();
                run_pass<1, NS>(sc, tiles, stB, ntiles, P, M, (it + 1) & 1, pnew, true, pbuf[pc & 1],
                            tbuf[pc & 1], tick, sw, &s_bcast, &s_flag, (double *)Pn, dsm, bars,
                            parity, ctl, timeout_ns);
                ++pc;
                if (!grid_sync(ctl, timeout_ns)) return;
                ++it;
            }
        } else {
            /* ── mixed: one pass per iteration ──
             * Before pass k the tile scalars take the totals of the last
             * reduction: after a pass that updated z, its true r.z (stop
             * test), then alpha_{k-1} = r.z / p.q and the recurrence for
             * beta_k; after a true-residual assembly, its r.z.  Each such
             * step reads st[cur] and writes st[cur ^ 1]. */
            float *qb[2] = {(float *)P.q, P.q1};
            int zsel = 0, cur = 0;
            bool prev_fresh = true;
            for (int k = 0;; ++k) {
                const bool repl = k > 0 && sp.replace_every > 0 && (k % sp.replace_every) == 0;
                {
                    TileState *sP = st + (size_t)cur * ntiles, *sN = st + (size_t)(cur ^ 1) * ntiles;
                    setup_slice(sc, tiles, k == 0 ? nullptr : sP, ntiles, sw);
                    if (k > 0) carry_inactive(sP, sN, ntiles);
                    const double *tt = tbuf[(pc - 1) & 1];
                    for (int t = sc.t0; t <= sc.t1; ++t) {
                        const TileDesc &T = stile(sc, tiles, t);
                        if (sc.pre[t + 1] == sc.pre[t]) continue;
                        const bool owner = sc.pre[t] >= sc.s0 && sc.pre[t] < sc.s1;
                        TileState S;
                        if (k == 0) {
                            S = start_state(__ldcg(tt + t), sp);
                            if (owner && threadIdx.x == 0 && S.active) atomicAdd(&ctl->n_active, 1);
                        } else {
                            S = load_state(sP + t);
                            if (!prev_fresh) {
                                const double rz = __ldcg(tt + t);
                                S.iter += 1;
                                if (rz < S.thr || S.iter >= sp.max_iter) tile_stop(S, T, owner, ctl);
                                else S.rz = rz;
                            }
                            if (S.active) {
                                const double pq = __ldcg(tt + (size_t)ntiles + t);
                                if (pq <= 0.0) {
                                    tile_stop(S, T, owner, ctl);
                                    S.alpha = 0.0;
                                } else {
                                    S.alpha = S.rz / pq;
                                    const double zq = __ldcg(tt + 2 * (size_t)ntiles + t);
                                    const double qq = __ldcg(tt + 3 * (size_t)ntiles + t);
                                    const double rzn = __fma_rn(S.alpha * S.alpha, qq,
                                                                __fma_rn(-2.0 * S.alpha, zq, S.rz));
                                    S.beta = rzn > 0.0 ? rzn / S.rz : 0.0;
                                }
                            }
                        }
                        put_state(sc, sN, t, S, owner);
                    }
                    __syncthreads();
                    cur ^= 1;
                }
                bool fresh = k == 0;
                if (repl) {
                    /* fold x += dx + alpha_{k-1} p_{k-1} (dx = 0), then the true
                     * residual b - A x replaces the recursive one */
                    const TileState *sC = st + (size_t)cur * ntiles;
                    for (int t = sc.t0; t <= sc.t1; ++t) {
                        const TileDesc &T = stile(sc, tiles, t);
                        if (sc.pre[t + 1] == sc.pre[t] || !sactive(sc, sC, t)) continue;
                        int a, b;
                        slice_items(sc, T, t, a, b);
                        const double alpha = salpha(sc, sC, t);
                        for (int li = a; li < b; ++li)
                            phase_fold<float>(T, li, P, (const float *)pb[k & 1], true, alpha);
                    }
                    if (!grid_sync(ctl, timeout_ns)) return;
                    setup_slice(sc, tiles, sC, ntiles, sw);
                    for (int t = sc.t0; t <= sc.t1; ++t) {
                        const TileDesc &T = stile(sc, tiles, t);
                        if (sc.pre[t + 1] == sc.pre[t]) continue;
                        int a, b;
                        slice_items(sc, T, t, a, b);
                        item_partials(T, a, b, pbuf[pc & 1], sgrp, [&](int li) {
                            return phase_init<V, WLS>(T, li, P, false, false, zb[zsel]);
                        });
                        if (b > a)
                            seg_done(T, t, b - a, pbuf[pc & 1], tbuf[pc & 1], tick, sw, &s_bcast,
                                     &s_flag);
                    }
                    ++pc;
                    if (!grid_sync(ctl, timeout_ns)) return;
                    /* stop test on the true r.z, beta from it */
                    TileState *sP = st + (size_t)cur * ntiles, *sN = st + (size_t)(cur ^ 1) * ntiles;
                    setup_slice(sc, tiles, sP, ntiles, sw);
                    carry_inactive(sP, sN, ntiles);
                    for (int t = sc.t0; t <= sc.t1; ++t) {
                        const TileDesc &T = stile(sc, tiles, t);
                        if (sc.pre[t + 1] == sc.pre[t]) continue;
                        const bool owner = sc.pre[t] >= sc.s0 && sc.pre[t] < sc.s1;
                        TileState S = load_state(sP + t);
                        const double rz = __ldcg(tbuf[(pc - 1) & 1] + t);
                        S.iter += 1;
                        if (rz < S.thr || S.iter >= sp.max_iter) {
                            tile_stop(S, T, owner, ctl);
                        } else {
                            S.beta = rz / S.rz;
                            S.rz = rz;
                        }
                        S.alpha = 0.0;
                        put_state(sc, sN, t, S, owner);
                    }
                    __syncthreads();
                    cur ^= 1;
                    fresh = true;
                }
                run_pass_s<NS>(sc, tiles, st + (size_t)cur * ntiles, ntiles, nitems, M, zsel, k & 1,
                           k == 0, fresh, (float *)pb[(k + 1) & 1], (float *)zb[zsel ^ 1],
                           qb[(k + 1) & 1], P.dx, pbuf[pc & 1], tbuf[pc & 1], tick, sw, red,
                           &s_bcast, &s_flag, (float *)Pn, dsm, bars, parity, ctl, timeout_ns);
                ++pc;
                if (!fresh) zsel ^= 1;
                prev_fresh = fresh;
                if (!grid_sync(ctl, timeout_ns)) return;
                if (*(volatile int *)&ctl->snap <= 0) break;
            }
            /* fold the FP32 increments of the pass into the FP64 solution
             * (every update has been applied to dx by then) */
            setup_slice(sc, tiles, nullptr, ntiles, sw);
            for (int t = sc.t0; t <= sc.t1; ++t) {
                const TileDesc &T = stile(sc, tiles, t);
                int a, b;
                slice_items(sc, T, t, a, b);
                for (int li = a; li < b; ++li) phase_fold<float>(T, li, P, nullptr, false, 0.0);
            }
            if (!grid_sync(ctl, timeout_ns)) return;
            it = *(volatile int *)&ctl->pass_max;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            if (sp.pass_iters) sp.pass_iters[outer] = it;
            ctl->total_iters += it;
            if (it > ctl->max_pass_iters) ctl->max_pass_iters = it;
            ctl->pass_max = 0;
        }
        if (outer < sp.n_irls) {
            float delta = sp.deltas[outer];
            setup_slice(sc, tiles, nullptr, ntiles, sw);
            for (int t = sc.t0; t <= sc.t1; ++t) {
                const TileDesc &T = stile(sc, tiles, t);
                int a, b;
                slice_items(sc, T, t, a, b);
                for (int li = a; li < b; ++li) phase_rw<V>(T, li, P, delta);
            }
            if (!grid_sync(ctl, timeout_ns)) return;
        }
    }
    if (WLS) return;   /* WLS mode: the caller reads the raw solution x */
    setup_slice(sc, tiles, nullptr, ntiles, sw);
    for (int t = sc.t0; t <= sc.t1; ++t) {
        const TileDesc &T = stile(sc, tiles, t);
        int a, b;
        slice_items(sc, T, t, a, b);
        for (int li = a; li < b; ++li) phase_final<V>(T, li, P);
    }
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

/* 2-D map of a stacked plane: dim0 = pitch elements, dim1 = rows */
static int make_map(CUtensorMap &m, const void *base, size_t esize, int pitch, int rows, int bx,
                    int by)
{
    auto enc = tensor_map_encoder();
    if (!enc) return fail(CUPHU_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {(cuuint64_t)pitch, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * esize};
    cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
    cuuint32_t es[2] = {1, 1};
    CUtensorMapDataType dt = esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                        : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUresult r = enc(&m, dt, 2, const_cast<void *>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(CUPHU_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return 0;
}

template <typename V>
static int make_maps(SolveMaps &M, const SolverPlanes &P, int pitch, int rows)
{
    int rc = 0;
    rc |= make_map(M.zA, P.z, sizeof(V), pitch, rows, kSegW, kItemBy + 2);
    rc |= make_map(M.p0A, P.p0, sizeof(V), pitch, rows, kSegW, kItemBy + 2);
    rc |= make_map(M.p1A, P.p1, sizeof(V), pitch, rows, kSegW, kItemBy + 2);
    if (sizeof(V) == 8) {
        rc |= make_map(M.wdA, P.wd, 4, pitch, rows, kItemBx, kItemBy + 1);
        rc |= make_map(M.wrA, P.wr, 4, pitch, rows, kWrW, kItemBy);
        rc |= make_map(M.xB, P.x, 8, pitch, rows, kItemBx, kItemBy);
        rc |= make_map(M.p0B, P.p0, 8, pitch, rows, kItemBx, kItemBy);
        rc |= make_map(M.p1B, P.p1, 8, pitch, rows, kItemBx, kItemBy);
        rc |= make_map(M.qB, P.q, 8, pitch, rows, kItemBx, kItemBy);
        rc |= make_map(M.rB, P.r, 8, pitch, rows, kItemBx, kItemBy);
        rc |= make_map(M.dB, P.diag, 8, pitch, rows, kItemBx, kItemBy);
    } else {
        rc |= make_map(M.zS1, P.r, 4, pitch, rows, kSegW, StageS::kBoxH);
        rc |= make_map(M.qS0, P.q, 4, pitch, rows, kSegW, StageS::kBoxH);
        rc |= make_map(M.qS1, P.q1, 4, pitch, rows, kSegW, StageS::kBoxH);
        rc |= make_map(M.wdS, P.wd, 4, pitch, rows, kSegW, StageS::kWdH);
        rc |= make_map(M.wrS, P.wr, 4, pitch, rows, kSegW, StageS::kBoxH);
        rc |= make_map(M.xB, P.dx, 4, pitch, rows, kItemBx, kItemBy);
    }
    return rc ? CUPHU_ERR_CUDA : 0;
}

/* Launch shapes of the persistent solver: the stages of each block's
 * shared-memory ring (items whose boxes are in flight) and the resident
 * blocks per SM it is compiled for (the launch bound, which sets the
 * registers a thread may use).  Deeper rings keep more bytes in flight per
 * SM; more blocks hide more latency.  The arithmetic and its order do not
 * depend on the shape, so every shape gives identical results; the
 * autotuner times them and keeps the fastest per job size. */
template <typename V, bool WLS, int NS, int MINB>
static int launch_solve_shape(const TileDesc *tiles, const int *item_tile, int nitems,
                              int ntiles, const SolverPlanes &P, int pitch, int rows,
                              TileState *st, double *part, SolverCtl *ctl, const SolveParams &sp,
                              long long timeout_ns, int device, cudaStream_t s)
{
    SolveMaps M;
    std::memset(&M, 0, sizeof(M));
    int rcm = make_maps<V>(M, P, pitch, rows);
    if (rcm) return rcm;
    int nsm = 0, per_sm = 0;
    CUPHU_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    const size_t smem = solve_smem_bytes<V, NS>();
    auto kern = k_solve<V, WLS, NS, MINB>;
    CUPHU_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    CUPHU_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kItemThreads,
                                                                 smem));
    if (per_sm < 1) return fail(CUPHU_ERR_CUDA, "solver kernel cannot be resident");
    per_sm = std::min(per_sm, MINB);
    int grid = std::min(nsm * per_sm, std::max(nitems, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kItemThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUPHU_TRY_CUDA(cudaLaunchKernelEx(&cfg, kern, tiles, item_tile, nitems, ntiles, P, st, part,
                                      ctl, sp, timeout_ns, M));
    return 0;
}

template <typename V, bool WLS>
static int launch_solve_kernel(const TileDesc *tiles, const int *item_tile, int nitems, int ntiles,
                          const SolverPlanes &P, int pitch, int rows, TileState *st, double *part,
                          SolverCtl *ctl, const SolveParams &sp, long long timeout_ns, int device,
                          cudaStream_t s)
{
    if (ntiles > kMaxTiles)
        return fail(CUPHU_ERR_INVALID, "at most 1024 tiles per solver launch");
    /* the shape from the autotuner (job size = item count) */
    tune_note_items(nitems);
    const int v = tune_get(device, sizeof(V) == 8 ? 2 : 1, (long long)nitems);
#define CUPHU_SOLVE_SHAPE(NS, MINB)                                                            \
    return launch_solve_shape<V, WLS, NS, MINB>(tiles, item_tile, nitems, ntiles, P, pitch,    \
                                                rows, st, part, ctl, sp, timeout_ns, device, s)
    if constexpr (sizeof(V) == 4) {
        switch (v) {
        case 1: CUPHU_SOLVE_SHAPE(2, 2);
        case 2: CUPHU_SOLVE_SHAPE(6, 1);
        default: CUPHU_SOLVE_SHAPE(3, 2);
        }
    } else {
        switch (v) {
        case 1: CUPHU_SOLVE_SHAPE(3, 1);
        default: CUPHU_SOLVE_SHAPE(2, 2);
        }
    }
#undef CUPHU_SOLVE_SHAPE
}

int solve_shape_count(bool fp64) { return fp64 ? 2 : 3; }

void solve_shape_of(bool fp64, int v, int *stages, int *blocks_per_sm)
{
    static const int mixed[3][2] = {{3, 2}, {2, 2}, {6, 1}};
    static const int f64[2][2] = {{2, 2}, {3, 1}};
    const int(*t)[2] = fp64 ? f64 : mixed;
    const int n = solve_shape_count(fp64);
    if (v < 0 || v >= n) v = 0;
    *stages = t[v][0];
    *blocks_per_sm = t[v][1];
}

template <typename V>
static int launch_solve_t(const TileDesc *tiles, const int *item_tile, int nitems, int ntiles,
                          const SolverPlanes &P, int pitch, int rows, TileState *st, double *part,
                          SolverCtl *ctl, const SolveParams &sp, long long timeout_ns, int device,
                          cudaStream_t s)
{
    if (sp.wls)
        return launch_solve_kernel<V, true>(tiles, item_tile, nitems, ntiles, P, pitch, rows, st,
                                            part, ctl, sp, timeout_ns, device, s);
    return launch_solve_kernel<V, false>(tiles, item_tile, nitems, ntiles, P, pitch, rows, st, part,
                                         ctl, sp, timeout_ns, device, s);
}

/* the failure test's one-shot switch, per device */
static std::atomic<int> g_skip_block[64];
static std::once_flag g_skip_init;

void solver_skip_barrier_once(int dev, int block)
{
    std::call_once(g_skip_init, [] { for (auto &v : g_skip_block) v.store(-1); });
    if (dev >= 0 && dev < 64) g_skip_block[dev].store(block);
}

int launch_solve(bool fp64, const TileDesc *tiles, const int *item_tile, int nitems,
                 int ntiles, const SolverPlanes &P, int plane_pitch, int plane_rows,
                 TileState *st, double *part, SolverCtl *ctl, const SolveParams &sp_in,
                 int device, cudaStream_t s)
{
    std::call_once(g_skip_init, [] { for (auto &v : g_skip_block) v.store(-1); });
    SolveParams sp = sp_in;
    if (device >= 0 && device < 64) sp.skip_block = g_skip_block[device].exchange(-1);
    long long timeout_ns = sp.timeout_ns;
    if (fp64)
        return launch_solve_t<double>(tiles, item_tile, nitems, ntiles, P, plane_pitch, plane_rows,
                                      st, part, ctl, sp, timeout_ns, device, s);
    return launch_solve_t<float>(tiles, item_tile, nitems, ntiles, P, plane_pitch, plane_rows, st,
                                 part, ctl, sp, timeout_ns, device, s);
}

}  // namespace cuphu
