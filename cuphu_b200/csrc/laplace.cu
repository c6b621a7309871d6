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
 *  - The p = z + beta p update is folded into the next stencil pass: each
 *    work item rebuilds p for its halo from r, diag and the previous p in
 *    shared memory (p is double-buffered so neighbours never race).
 *  - FP64 mode keeps every vector in double and is bit-identical to the CPU
 *    FP64 oracle (same operation order, explicit fma, same reduction tree).
 *    Mixed mode stores x, r, p, q, diag in FP32 (half the bytes) with FP64
 *    scalars and dots, and replaces the recursive residual by the true
 *    residual b - A x every `replace_every` iterations.
 */
#include "kernels.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda/atomic>
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

__device__ __forceinline__ void store_partial(double acc, double *part, int item, double *sw)
{
    double bs = block_sum(acc, sw);
    if (threadIdx.x == 0) part[item] = bs;
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

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* Grid barrier with a bounded wait.  The last arriving block snapshots the
 * active-tile count, so every block takes the same loop decision. */
__device__ __forceinline__ bool grid_sync(SolverCtl *ctl, long long timeout_ns)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(ctl->bar_gen);
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(ctl->bar_count);
        cuda::atomic_ref<int, cuda::thread_scope_device> act(ctl->n_active);
        __threadfence();
        unsigned g = gen.load(cuda::memory_order_acquire);
        unsigned prev = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
        if (prev == gridDim.x - 1u) {
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

/* ── INIT / true residual: b, diag (A10) and r = b - A x, rz partial ────────
 * zero_x: first pass (x = 0, r = b).  write_diag: assemble pass (else the
 * stored diag is reused: residual replacement). */
template <typename V, bool WLS>
__device__ double phase_init(const TileDesc &T, int li, const SolverPlanes &P, bool zero_x,
                             bool write_diag)
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
    size_t prow = (size_t)r * pitch;
    double xv[4];
    V rv[4], dv[4], zv[4];
    if (!zero_x) ld4(x + prow + q.c0, xv);
    if (!write_diag) ld4(dg + prow + q.c0, dv);
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        int c = q.c0 + j;
        if (c >= nc) {
            rv[j] = (V)0;
            zv[j] = (V)0;
            if (write_diag) dv[j] = (V)0;
            if (zero_x) xv[j] = 0.0;
            continue;
        }
        size_t gi = (size_t)r * pp + c, pi = prow + c;
        float pa = gdp ? 0.0f : __ldg(ph + gi);
        double bv = 0.0, ws = 0.0;
        if (r < nr - 1) {
            float w = ldc(wd + pi);
            if (w > 0.0f) {
                float g = gdp ? ldc(gdp + pi) : lap_wrap_pi(__ldg(ph + gi + pp) - pa);
                bv = __fma_rn(-(double)w, (double)g, bv);
                ws += w;
            }
        }
        if (r > 0) {
            float w = ldc(wd + pi - pitch);
            if (w > 0.0f) {
                float g = gdp ? ldc(gdp + pi - pitch) : lap_wrap_pi(pa - __ldg(ph + gi - pp));
                bv = __fma_rn((double)w, (double)g, bv);
                ws += w;
            }
        }
        if (c < nc - 1) {
            float w = ldc(wr + pi);
            if (w > 0.0f) {
                float g = grp ? ldc(grp + pi) : lap_wrap_pi(__ldg(ph + gi + 1) - pa);
                bv = __fma_rn(-(double)w, (double)g, bv);
                ws += w;
            }
        }
        if (c > 0) {
            float w = ldc(wr + pi - 1);
            if (w > 0.0f) {
                float g = grp ? ldc(grp + pi - 1) : lap_wrap_pi(pa - __ldg(ph + gi - 1));
                bv = __fma_rn((double)w, (double)g, bv);
                ws += w;
            }
        }
        if (rhsp) bv = (double)ldc(rhsp + pi);
        double d = write_diag ? ws + eps : (double)dv[j];
        double y;
        if (zero_x) {
            y = 0.0;
            xv[j] = 0.0;
        } else {
            double xa = xv[j];
            y = eps * xa;
            if (r < nr - 1) y = __fma_rn((double)ldc(wd + pi), xa - ldc(x + pi + pitch), y);
            if (r > 0)      y = __fma_rn((double)ldc(wd + pi - pitch), xa - ldc(x + pi - pitch), y);
            if (c < nc - 1) y = __fma_rn((double)ldc(wr + pi), xa - ldc(x + pi + 1), y);
            if (c > 0)      y = __fma_rn((double)ldc(wr + pi - 1), xa - ldc(x + pi - 1), y);
        }
        V rs = (V)(bv - y);
        V ds = (V)d;
        double z = (double)rs / (double)ds;
        acc = __fma_rn((double)rs, z, acc);
        rv[j] = rs;
        zv[j] = (V)z;
        if (write_diag) dv[j] = ds;
    }
    if (sizeof(V) == 8) st4(rr + prow + q.c0, rv);
    st4((V *)P.z + T.pix + prow + q.c0, zv);
    if (write_diag) st4(dg + prow + q.c0, dv);
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
    CUtensorMap zA, p0A, p1A, wdA, wrA;        /* stencil pass boxes */
    CUtensorMap xB, p0B, p1B, qB, rB, dB;      /* update pass boxes  */
    CUtensorMap zB;                            /* mixed: z in place of r, dx in xB */
};

__host__ __device__ constexpr size_t al128(size_t b) { return (b + 127) & ~(size_t)127; }

template <typename V> struct StageA {
    static constexpr size_t kVec = al128((size_t)(kItemBy + 2) * kSegW * sizeof(V));
    static constexpr size_t kWd = al128((size_t)(kItemBy + 1) * kItemBx * sizeof(float));
    static constexpr size_t kWr = al128((size_t)kItemBy * kWrW * sizeof(float));
    /* mixed mode: the item's FP32 increment dx, which takes the previous
     * iteration's deferred dx += alpha p_old */
    static constexpr size_t kDx = sizeof(V) == 4 ? (size_t)kItemBy * kItemBx * 4 : 0;
    static constexpr size_t kBytes = 2 * kVec + kWd + kWr + kDx;
    static constexpr uint32_t kTx = (uint32_t)(2 * (kItemBy + 2) * kSegW * sizeof(V) +
                                               (kItemBy + 1) * kItemBx * 4 + kItemBy * kWrW * 4);
};
/* update-pass stage: FP64 mode x, p, q, r, diag; mixed mode q, z (r = z diag
 * is not stored) and diag, back to back */
template <typename V> struct StageB {
    static constexpr size_t kX = (size_t)kItemBy * kItemBx * sizeof(double);
    static constexpr size_t kV = (size_t)kItemBy * kItemBx * sizeof(V);
    static constexpr size_t kBytes = kX + 4 * kV;
    static constexpr uint32_t kTxFull = (uint32_t)(sizeof(V) == 4 ? 3 * kV : kX + 4 * kV);
    static constexpr uint32_t kTxX = (uint32_t)(kX + kV);
};
#ifndef CUPHU_SOLVE_STAGES_F32
#define CUPHU_SOLVE_STAGES_F32 2
#endif
template <typename V> __host__ __device__ constexpr int n_stages()
{
    return sizeof(V) == 4 ? CUPHU_SOLVE_STAGES_F32 : 2;
}
template <typename V> __host__ __device__ constexpr size_t stage_bytes()
{
    return al128(StageA<V>::kBytes > StageB<V>::kBytes ? StageA<V>::kBytes : StageB<V>::kBytes);
}
/* ring shape of a pass: the mixed update pass stages only q, z and diag
 * (12 KB per item), so it runs four shallow stages in the memory of the two
 * deep ones */
constexpr size_t kStageBm = 3 * (size_t)kItemBy * kItemBx * 4;
template <int KIND, typename V> __host__ __device__ constexpr int pass_stages()
{
    return (KIND == 1 && sizeof(V) == 4) ? 4 : n_stages<V>();
}
template <int KIND, typename V> __host__ __device__ constexpr size_t pass_stage_bytes()
{
    return (KIND == 1 && sizeof(V) == 4) ? kStageBm : stage_bytes<V>();
}
static_assert(pass_stages<1, float>() * pass_stage_bytes<1, float>() <=
                  n_stages<float>() * stage_bytes<float>(),
              "mixed update-pass ring exceeds the stage memory");
/* p_new of an item with its halo ring, rows of kSegW elements laid out like
 * the staged boxes (column 0 <-> c0b - 4), so own columns start 16-byte
 * aligned at column 4 */
template <typename V> __host__ __device__ constexpr size_t pn_bytes()
{
    return al128((size_t)kHaloH * kSegW * sizeof(V));
}
template <typename V> __host__ __device__ constexpr size_t solve_smem_bytes()
{
    return n_stages<V>() * stage_bytes<V>() + pn_bytes<V>() + 128;
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
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
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

template <typename V>
__device__ __forceinline__ void issue_a(const TileDesc &T, int li, const SolveMaps &M, int pold_sel,
                                        bool first, bool upd, char *stage, uint64_t *bar)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const int y = T.row0 + r0b;
    char *Z = stage;
    char *PO = stage + StageA<V>::kVec;
    char *WD = PO + StageA<V>::kVec;
    char *WR = WD + StageA<V>::kWd;
    char *DX = WR + StageA<V>::kWr;
    uint32_t tx = StageA<V>::kTx - (first ? (uint32_t)((kItemBy + 2) * kSegW * sizeof(V)) : 0u);
    if (upd) tx += (uint32_t)StageA<V>::kDx;
    mbar_expect(bar, tx);
    tma_load_2d(Z, &M.zA, c0b - 4, y - 1, bar);
    if (!first) tma_load_2d(PO, pold_sel ? &M.p1A : &M.p0A, c0b - 4, y - 1, bar);
    tma_load_2d(WD, &M.wdA, c0b, y - 1, bar);
    tma_load_2d(WR, &M.wrA, c0b - 4, y, bar);
    if (upd) tma_load_2d(DX, &M.xB, c0b, y, bar);
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

/* p_new = z + beta p_old: FP32 arithmetic in mixed mode, FP64 in FP64 mode */
template <typename V>
__device__ __forceinline__ V pupdate(bool first, double beta, float betaf, V po, V z)
{
    if (first) return z;
    if (sizeof(V) == 4) return (V)__fmaf_rn(betaf, (float)po, (float)z);
    return (V)__fma_rn(beta, (double)po, (double)z);
}

/* stencil pass on a staged item: p_new = z + beta p_old (own + halo ring),
 * q = A p_new, thread partial of p.q (FP64 accumulation).  FP64 mode: FP64
 * arithmetic in the oracle's operation order.  Mixed mode: FP32 arithmetic
 * (the SpMV and vector update), FP64 only for the dot; with upd it also
 * applies the previous iteration's solution update dx += alpha_prev p_old,
 * which the update pass leaves to this pass because p_old is staged here
 * anyway. */
template <typename V>
__device__ double compute_a(const TileDesc &T, int li, const SolverPlanes &P, V *pnew_all,
                            bool first, double beta, bool upd, double alpha_prev,
                            const char *stage, V *Pn)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const V *Z = (const V *)stage;
    const V *PO = (const V *)(stage + StageA<V>::kVec);
    const float *WD = (const float *)(stage + 2 * StageA<V>::kVec);
    const float *WR = (const float *)(stage + 2 * StageA<V>::kVec + StageA<V>::kWd);
    const int nr = T.nr, nc = T.nc;
    const float betaf = (float)beta;
    const int ty = threadIdx.x / kItemTx, tx = threadIdx.x % kItemTx;
    const int r = r0b + ty, c0 = c0b + tx * kItemVx;
    const bool own = r < nr && c0 < nc;
    /* own p_new: row ty+1, columns 4 + 4 tx .. +3 */
    V pn[4] = {(V)0, (V)0, (V)0, (V)0};
    const int so = (ty + 1) * kSegW + 4 + tx * kItemVx;
    if (own) {
        V zv[4], pv[4] = {(V)0, (V)0, (V)0, (V)0};
        sld4(Z + so, zv);
        if (!first) sld4(PO + so, pv);
#pragma unroll
        for (int j = 0; j < kItemVx; ++j)
            if (c0 + j < nc) pn[j] = pupdate<V>(first, beta, betaf, pv[j], zv[j]);
        if constexpr (sizeof(V) == 4) {
            if (upd) {
                const float *DX = (const float *)(stage + 2 * StageA<V>::kVec + StageA<V>::kWd +
                                                  StageA<V>::kWr);
                float dxv[4];
                sld4(DX + ty * kItemBx + tx * kItemVx, dxv);
                const float af = (float)alpha_prev;
#pragma unroll
                for (int j = 0; j < kItemVx; ++j)
                    if (c0 + j < nc) dxv[j] = __fmaf_rn(af, (float)pv[j], dxv[j]);
                st4(P.dx + T.pix + (size_t)r * T.pitch + c0, dxv);
            }
        }
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
        V v = (V)0;
        if (gr >= 0 && gr < nr && gc >= 0 && gc < nc) {
            int sidx = i * kSegW + jc;
            v = pupdate<V>(first, beta, betaf, first ? (V)0 : PO[sidx], Z[sidx]);
        }
        Pn[i * kSegW + jc] = v;
    }
    __syncthreads();
    double acc = 0.0;
    if (own) {
        V up[4], dn[4], qv[4] = {(V)0, (V)0, (V)0, (V)0};
        float wdn[4], wup[4], wrt[4];
        sld4(Pn + so - kSegW, up);
        sld4(Pn + so + kSegW, dn);
        V lf = Pn[so - 1], rt = Pn[so + 4];
        sld4(WD + (ty + 1) * kItemBx + tx * kItemVx, wdn);
        sld4(WD + ty * kItemBx + tx * kItemVx, wup);
        sld4(WR + ty * kWrW + tx * kItemVx + 4, wrt);
        float wlf = WR[ty * kWrW + tx * kItemVx + 3];
#pragma unroll
        for (int j = 0; j < kItemVx; ++j) {
            int c = c0 + j;
            if (c >= nc) continue;
            V xl = j == 0 ? lf : pn[j - 1];
            V xr = j == kItemVx - 1 ? rt : pn[j + 1];
            float wl = j == 0 ? wlf : wrt[j - 1];
            if (sizeof(V) == 4) {
                float xa = (float)pn[j];
                float y = __fmul_rn(kLapEpsF, xa);
                if (r < nr - 1) y = __fmaf_rn(wdn[j], xa - (float)dn[j], y);
                if (r > 0)      y = __fmaf_rn(wup[j], xa - (float)up[j], y);
                if (c < nc - 1) y = __fmaf_rn(wrt[j], xa - (float)xr, y);
                if (c > 0)      y = __fmaf_rn(wl, xa - (float)xl, y);
                qv[j] = (V)y;
            } else {
                double xa = (double)pn[j];
                double y = (double)kLapEpsF * xa;
                if (r < nr - 1) y = __fma_rn((double)wdn[j], xa - (double)dn[j], y);
                if (r > 0)      y = __fma_rn((double)wup[j], xa - (double)up[j], y);
                if (c < nc - 1) y = __fma_rn((double)wrt[j], xa - (double)xr, y);
                if (c > 0)      y = __fma_rn((double)wl, xa - (double)xl, y);
                qv[j] = (V)y;
            }
            acc = __fma_rn((double)pn[j], (double)qv[j], acc);
        }
        size_t o = T.pix + (size_t)r * T.pitch + c0;
        st4(pnew_all + o, pn);
        st4((V *)P.q + o, qv);
    }
    return acc;
}

template <typename V>
__device__ __forceinline__ void issue_b(const TileDesc &T, int li, const SolveMaps &M, int pnew_sel,
                                        bool update_r, char *stage, uint64_t *bar)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const int y = T.row0 + r0b;
    if (sizeof(V) == 4) {
        /* mixed: q, z, diag back to back */
        char *QB = stage;
        mbar_expect(bar, StageB<V>::kTxFull);
        tma_load_2d(QB, &M.qB, c0b, y, bar);
        tma_load_2d(QB + StageB<V>::kV, &M.zB, c0b, y, bar);
        tma_load_2d(QB + 2 * StageB<V>::kV, &M.dB, c0b, y, bar);
        return;
    }
    char *X = stage;
    char *PB = X + StageB<V>::kX;
    char *QB = PB + StageB<V>::kV;
    char *RB = QB + StageB<V>::kV;
    char *DB = RB + StageB<V>::kV;
    mbar_expect(bar, update_r ? StageB<V>::kTxFull : StageB<V>::kTxX);
    tma_load_2d(X, &M.xB, c0b, y, bar);
    tma_load_2d(PB, pnew_sel ? &M.p1B : &M.p0B, c0b, y, bar);
    if (update_r) {
        tma_load_2d(QB, &M.qB, c0b, y, bar);
        tma_load_2d(RB, &M.rB, c0b, y, bar);
        tma_load_2d(DB, &M.dB, c0b, y, bar);
    }
}

template <typename V>
__device__ double compute_b(const TileDesc &T, int li, const SolverPlanes &P, double alpha,
                            bool update_r, const char *stage)
{
    const int r0b = (li / T.nbx) * kItemBy, c0b = (li % T.nbx) * kItemBx;
    const V *PB = (const V *)(stage + StageB<V>::kX);
    const V *QB = PB + kItemBy * kItemBx;
    const V *RB = QB + kItemBy * kItemBx;
    const V *DB = RB + kItemBy * kItemBx;
    const int ty = threadIdx.x / kItemTx, tx = threadIdx.x % kItemTx;
    const int r = r0b + ty, c0 = c0b + tx * kItemVx;
    if (r >= T.nr || c0 >= T.nc) return 0.0;
    const int s0 = ty * kItemBx + tx * kItemVx;
    const size_t o = T.pix + (size_t)r * T.pitch + c0;
    double acc = 0.0;
    if constexpr (sizeof(V) == 4) {
        /* mixed: r = z diag, r -= alpha q, z = r / diag (the solution update
         * dx += alpha p is deferred to the next stencil pass or fold) */
        const float *QM = (const float *)stage;
        float qv[4], zv[4], dv[4];
        sld4(QM + s0, qv);
        sld4(QM + kItemBy * kItemBx + s0, zv);
        sld4(QM + 2 * kItemBy * kItemBx + s0, dv);
        const float alphaf = (float)alpha;
#pragma unroll
        for (int j = 0; j < kItemVx; ++j) {
            if (c0 + j >= T.nc) continue;
            float rn = __fmaf_rn(-alphaf, qv[j], __fmul_rn(zv[j], dv[j]));
            float z = __fdiv_rn(rn, dv[j]);
            zv[j] = z;
            acc = __fma_rn((double)rn, (double)z, acc);
        }
        st4((float *)P.z + o, zv);
    } else {
        const double *X = (const double *)stage;
        double xv[4];
        V pv[4], qv[4], rv[4] = {(V)0, (V)0, (V)0, (V)0}, dv[4], zv[4] = {(V)0, (V)0, (V)0, (V)0};
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
            xv[j] = __fma_rn(alpha, (double)pv[j], xv[j]);
            if (update_r) {
                V rn = (V)__fma_rn(-alpha, (double)qv[j], (double)rv[j]);
                rv[j] = rn;
                double z = (double)rn / (double)dv[j];
                zv[j] = (V)z;
                acc = __fma_rn((double)rn, z, acc);
            }
        }
        st4(P.x + o, xv);
        if (update_r) {
            st4((V *)P.r + o, rv);
            st4((V *)P.z + o, zv);
        }
    }
    return acc;
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

/* mixed mode: the stencil pass of an iteration applies the previous
 * iteration's deferred solution update unless there is none (first
 * iteration, or alpha_prev zeroed because a fold already applied it) */
template <typename V> __device__ __forceinline__ bool defer_upd(bool first, double alpha_prev)
{
    return sizeof(V) == 4 && !first && alpha_prev != 0.0;
}

/* run a staged pass over this block's slice.  KIND 0: the stencil pass,
 * KIND 1: the update pass.  NS items are in flight; the stage of item k is
 * refilled with item k+NS right after the barrier of item k's reduction,
 * which every thread reaches only after its last read of the stage and Pn. */
template <int KIND, typename V>
__device__ void run_pass(const SliceCtl &sc, const TileDesc *gt, const TileState *st, int ntiles,
                         const SolverPlanes &P, const SolveMaps &M, int psel, V *pvec, bool flag,
                         double *part, double *tot, unsigned *cnt, double *sw, double *s_bcast,
                         int *s_flag, V *Pn, char *stages, uint64_t *bars, uint32_t &parity,
                         SolverCtl *ctl, long long timeout_ns)
{
    constexpr int NS = pass_stages<KIND, V>();
    constexpr size_t SB = pass_stage_bytes<KIND, V>();
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
            if (KIND == 0)
                issue_a<V>(T, li, M, psel, flag, defer_upd<V>(flag, salpha(sc, st, ci.t)),
                           stages + k * SB, bars + k);
            else issue_b<V>(T, li, M, psel, flag, stages + k * SB, bars + k);
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
        if (KIND == 0) {
            const double ap = salpha(sc, st, cc.t);
            acc = compute_a<V>(T, li, P, pvec, flag, sbeta(sc, st, cc.t), defer_upd<V>(flag, ap),
                               ap, stages + s * SB, Pn);
        } else
            acc = compute_b<V>(T, li, P, salpha(sc, st, cc.t), flag, stages + s * SB);
        double bs = block_sum_item(acc, sw + 8 * (done & 1));   /* contains the item barrier */
        if (threadIdx.x == 0) {
            if (red) part[T.item0 + li] = bs;
            if (ci.p < sc.s1) {
                fence_async_smem();
                const TileDesc &Tn = stile(sc, gt, ci.t);
                int ln = ci.p - sc.pre[ci.t];
                if (KIND == 0)
                    issue_a<V>(Tn, ln, M, psel, flag, defer_upd<V>(flag, salpha(sc, st, ci.t)),
                               stages + s * SB, bars + s);
                else issue_b<V>(Tn, ln, M, psel, flag, stages + s * SB, bars + s);
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

/* Mixed-precision update pass without shared-memory staging.  The pass is
 * elementwise (r = z diag - alpha q, z = r / diag) plus the r.z dot, so the
 * block sweeps its slice's pixel rows with 16-byte loads straight from HBM
 * (contiguous row spans per plane instead of 256-byte item rows), and
 * each thread accumulates r.z in FP64 over the whole tile segment: one block reduction
 * per tile segment instead of one per item, no barrier per item.  The
 * segment total goes into the partial slot of the segment's first item and
 * the segment's other slots are zeroed, so the tile total is the canonical
 * sum over the tile's partials as in the other phases (deterministic for a
 * given grid; mixed mode does not follow the oracle's summation order). */
__device__ void run_update_direct(const SliceCtl &sc, const TileDesc *gt, const TileState *st,
                                  const SolverPlanes &P, double *part, double *tot,
                                  unsigned *cnt, double *sw, double *s_bcast, int *s_flag)
{
    for (int t = sc.t0; t <= sc.t1; ++t) {
        if (sc.pre[t + 1] == sc.pre[t] || !sactive(sc, st, t)) continue;
        const TileDesc &T = stile(sc, gt, t);
        int a, b;
        slice_items(sc, T, t, a, b);
        if (a >= b) continue;
        const float alphaf = (float)salpha(sc, st, t);
        const int nr = T.nr, nc = T.nc, nbx = T.nbx;
        float *zp = (float *)P.z + T.pix;
        const float *qp = (const float *)P.q + T.pix, *dp = (const float *)P.diag + T.pix;
        double acc = 0.0;
        /* the segment's items, band by band (16-row strips), each strip swept
         * one pixel row at a time across the segment's columns of the band */
        for (int band = a / nbx; band <= (b - 1) / nbx; ++band) {
            const int i0 = max(a, band * nbx) - band * nbx, i1 = min(b, (band + 1) * nbx) - band * nbx;
            const int clo = i0 * kItemBx, chi = min(i1 * kItemBx, nc);
            const int rlo = band * kItemBy, rhi = min(rlo + kItemBy, nr);
            /* the band's (row, 4-column group) pairs spread over all threads,
             * row-major, so partial bands keep every thread busy */
            const int qw = (chi - clo + kItemVx - 1) / kItemVx;
            const int nq = (rhi - rlo) * qw;
            for (int u = threadIdx.x; u < nq; u += blockDim.x) {
                {
                    const int r = rlo + u / qw, c0 = clo + (u - (u / qw) * qw) * kItemVx;
                    const size_t o = (size_t)r * T.pitch + c0;
                    float4 qv = __ldcs(reinterpret_cast<const float4 *>(qp + o));
                    float4 zv = __ldcg(reinterpret_cast<const float4 *>(zp + o));
                    float4 dv = __ldcg(reinterpret_cast<const float4 *>(dp + o));
                    const int n4 = min(chi - c0, kItemVx);
                    float q4[4] = {qv.x, qv.y, qv.z, qv.w};
                    float z4[4] = {zv.x, zv.y, zv.z, zv.w};
                    float d4[4] = {dv.x, dv.y, dv.z, dv.w};
#pragma unroll
                    for (int j = 0; j < kItemVx; ++j) {
                        if (j >= n4) continue;
                        float rn = __fmaf_rn(-alphaf, q4[j], __fmul_rn(z4[j], d4[j]));
                        float z = __fdiv_rn(rn, d4[j]);
                        z4[j] = z;
                        acc = __fma_rn((double)rn, (double)z, acc);
                    }
                    st4(zp + o, z4);
                }
            }
        }
        double v = block_sum(acc, sw);
        if (threadIdx.x == 0) part[T.item0 + a] = v;
        for (int li = a + 1 + (int)threadIdx.x; li < b; li += blockDim.x) part[T.item0 + li] = 0.0;
        __threadfence();
        seg_done(T, t, b - a, part, tot, cnt, sw, s_bcast, s_flag);
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

#ifndef CUPHU_SOLVE_MIN_BLOCKS
#define CUPHU_SOLVE_MIN_BLOCKS 3
#endif

/* WLS = true: the WLS-mode instance (explicit arc targets / right-hand
 * side, optional warm start, no anchoring); a separate instantiation so the
 * main path's register allocation does not carry its extra inputs */
template <typename V, bool WLS>
__global__ void __launch_bounds__(kItemThreads, CUPHU_SOLVE_MIN_BLOCKS)
    k_solve(const TileDesc *__restrict__ tiles, const int *__restrict__ item_tile, int nitems,
            int ntiles, SolverPlanes P, TileState *st, double *part, SolverCtl *ctl,
            SolveParams sp, long long timeout_ns, const __grid_constant__ SolveMaps M)
{
    extern __shared__ __align__(128) char dsm_raw[];
    __shared__ double sw[32];
    __shared__ double s_bcast;
    __shared__ int s_flag;
    __shared__ __align__(8) uint64_t bars[4];
    __shared__ SliceCtl sc;
    constexpr int NS = n_stages<V>();
    constexpr int NBAR = pass_stages<1, V>() > NS ? pass_stages<1, V>() : NS;
    char *dsm = (char *)(((uintptr_t)dsm_raw + 127) & ~(uintptr_t)127);
    const bool mixed = sizeof(V) == 4;
    V *pb[2] = {(V *)P.p0, (V *)P.p1};
    /* per-item partials and published tile totals, both double-buffered by
     * phase parity, and the per-tile item tickets */
    double *pbuf[2] = {part, part + nitems};
    double *tbuf[2] = {part + 2 * (size_t)nitems, part + 2 * (size_t)nitems + ntiles};
    unsigned *tick = reinterpret_cast<unsigned *>(part + 2 * (size_t)nitems + 2 * (size_t)ntiles);
    V *Pn = (V *)(dsm + NS * stage_bytes<V>());
    uint32_t parity = 0u;
    (void)item_tile;
    if (threadIdx.x == 0) {
        for (int k = 0; k < NBAR; ++k) mbar_init(&bars[k]);
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
            for (int li = a; li < b; ++li)
                store_partial(phase_init<V, WLS>(T, li, P, outer == 0 && !(WLS && sp.warm), true),
                              pbuf[pc & 1], T.item0 + li, sw);
            if (b > a) seg_done(T, t, b - a, pbuf[pc & 1], tbuf[pc & 1], tick, sw, &s_bcast, &s_flag);
        }
        ++pc;
        if (!grid_sync(ctl, timeout_ns)) return;

        /* stA: scalars after the stencil-pass decisions, stB: after the
         * update-pass decisions; each phase reads one and writes the other,
         * so the active flags a phase slices on never change under it */
        TileState *stA = st, *stB = st + ntiles;
        int it = 0;
        while (true) {
            V *pnew = pb[(it + 1) & 1];
            /* slice over the tiles active in the previous phase; reduce r.z,
             * update the tile scalars, then the stencil pass */
            setup_slice(sc, tiles, it == 0 ? nullptr : stB, ntiles, sw);
            /* tiles not counted this phase keep their inactive flag in stA */
            if (it > 0 && blockIdx.x == 0)
                for (int t = threadIdx.x; t < ntiles; t += blockDim.x)
                    if (!__ldcg(&stB[t].active)) stA[t].active = 0;
            for (int t = sc.t0; t <= sc.t1; ++t) {
                const TileDesc &T = stile(sc, tiles, t);
                if (sc.pre[t + 1] == sc.pre[t]) continue;          /* not counted */
                const bool owner = sc.pre[t] >= sc.s0 && sc.pre[t] < sc.s1;
                TileState S;
                if (it == 0) {
                    double tot = __ldcg(tbuf[(pc - 1) & 1] + t);
                    S.rz = tot;
                    S.rz0 = tot;
                    S.thr = (double)sp.tol * (double)sp.tol * tot;
                    S.alpha = 0.0;
                    S.beta = 0.0;
                    S.iter = 0;
                    S.active = (tot > 0.0 && sp.max_iter > 0) ? 1 : 0;
                    if (owner && threadIdx.x == 0 && S.active) atomicAdd(&ctl->n_active, 1);
                } else {
                    S = load_state(stB + t);
                    double tot = __ldcg(tbuf[(pc - 1) & 1] + t);
                    /* a replacement iteration folded its update already */
                    if (mixed && sp.replace_every > 0 && (it % sp.replace_every) == 0)
                        S.alpha = 0.0;
                    S.iter += 1;
                    if (tot < S.thr || S.iter >= sp.max_iter) {
                        S.active = 0;
                        if (owner && threadIdx.x == 0) {
                            atomicSub(&ctl->n_active, 1);
                            atomicAdd(&ctl->px_iters, (unsigned long long)S.iter *
                                                          (unsigned long long)((long long)T.nr * T.nc));
                        }
                    } else {
                        S.beta = tot / S.rz;
                        S.rz = tot;
                    }
                }
                if (threadIdx.x == 0) {
                    if (owner || !scached(sc, t)) stA[t] = S;
                    sput(sc, t, S);
                }
            }
            __syncthreads();
            run_pass<0, V>(sc, tiles, stA, ntiles, P, M, it & 1, pnew, it == 0, pbuf[pc & 1],
                           tbuf[pc & 1], tick, sw, &s_bcast, &s_flag, Pn, dsm, bars, parity, ctl,
                           timeout_ns);
            ++pc;
            if (!grid_sync(ctl, timeout_ns)) return;
            if (*(volatile int *)&ctl->snap <= 0) break;

            /* slice over the tiles active in the stencil pass; reduce p.q, alpha */
            const bool repl = mixed && sp.replace_every > 0 && ((it + 1) % sp.replace_every) == 0;
            setup_slice(sc, tiles, stA, ntiles, sw);
            if (blockIdx.x == 0)
                for (int t = threadIdx.x; t < ntiles; t += blockDim.x)
                    if (!__ldcg(&stA[t].active)) stB[t].active = 0;
            for (int t = sc.t0; t <= sc.t1; ++t) {
                const TileDesc &T = stile(sc, tiles, t);
                if (sc.pre[t + 1] == sc.pre[t]) continue;
                const bool owner = sc.pre[t] >= sc.s0 && sc.pre[t] < sc.s1;
                TileState S = load_state(stA + t);
                double pq = __ldcg(tbuf[(pc - 1) & 1] + t);
                if (pq <= 0.0) {
                    S.active = 0;
                    S.alpha = 0.0;
                    if (owner && threadIdx.x == 0) {
                        atomicSub(&ctl->n_active, 1);
                        atomicAdd(&ctl->px_iters, (unsigned long long)S.iter *
                                                      (unsigned long long)((long long)T.nr * T.nc));
                    }
                } else {
                    S.alpha = S.rz / pq;
                }
                if (threadIdx.x == 0) {
                    if (owner || !scached(sc, t)) stB[t] = S;
                    sput(sc, t, S);
                }
            }
            __syncthreads();
            if (!repl) {
                if (mixed)
                    run_update_direct(sc, tiles, stB, P, pbuf[pc & 1], tbuf[pc & 1], tick, sw,
                                      &s_bcast, &s_flag);
                else
                    run_pass<1, V>(sc, tiles, stB, ntiles, P, M, (it + 1) & 1, pnew, true,
                                   pbuf[pc & 1], tbuf[pc & 1], tick, sw, &s_bcast, &s_flag, Pn, dsm,
                                   bars, parity, ctl, timeout_ns);
                ++pc;
            } else {
                /* fold this iteration's update into the FP64 solution; the
                 * true residual follows once every neighbour has folded */
                for (int t = sc.t0; t <= sc.t1; ++t) {
                    const TileDesc &T = stile(sc, tiles, t);
                    if (sc.pre[t + 1] == sc.pre[t] || !sactive(sc, stB, t)) continue;
                    int a, b;
                    slice_items(sc, T, t, a, b);
                    double alpha = salpha(sc, stB, t);
                    for (int li = a; li < b; ++li) phase_fold<V>(T, li, P, pnew, true, alpha);
                }
            }
            if (!grid_sync(ctl, timeout_ns)) return;
            if (repl) {
                setup_slice(sc, tiles, stB, ntiles, sw);
                for (int t = sc.t0; t <= sc.t1; ++t) {
                    const TileDesc &T = stile(sc, tiles, t);
                    int a, b;
                    if (sc.pre[t + 1] == sc.pre[t]) continue;
                    slice_items(sc, T, t, a, b);
                    for (int li = a; li < b; ++li)
                        store_partial(phase_init<V, WLS>(T, li, P, false, false), pbuf[pc & 1],
                                      T.item0 + li, sw);
                    if (b > a)
                        seg_done(T, t, b - a, pbuf[pc & 1], tbuf[pc & 1], tick, sw, &s_bcast,
                                 &s_flag);
                }
                ++pc;
                if (!grid_sync(ctl, timeout_ns)) return;
            }
            ++it;
        }
        if (mixed) {
            /* fold the FP32 increments of the pass into the FP64 solution,
             * with each tile's deferred last update: a tile that stopped in
             * an r.z reduction at iteration i (stA.iter = i, stB.iter = i-1)
             * still owes alpha_{i-1} p_{i-1} (p in pb[i & 1]; alpha zeroed
             * when a replacement fold applied it); one that stopped in a p.q
             * reduction (stA.iter = stB.iter) owes nothing */
            setup_slice(sc, tiles, nullptr, ntiles, sw);
            for (int t = sc.t0; t <= sc.t1; ++t) {
                const TileDesc &T = stile(sc, tiles, t);
                int a, b;
                slice_items(sc, T, t, a, b);
                if (a >= b) continue;
                const int ia = __ldcg(&stA[t].iter), ib = __ldcg(&stB[t].iter);
                const double ap = ia == ib ? 0.0 : __ldcg(&stA[t].alpha);
                const V *pl = pb[ia & 1];
                for (int li = a; li < b; ++li) phase_fold<V>(T, li, P, pl, ap != 0.0, ap);
            }
            if (!grid_sync(ctl, timeout_ns)) return;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            if (sp.pass_iters) sp.pass_iters[outer] = it;
            ctl->total_iters += it;
            if (it > ctl->max_pass_iters) ctl->max_pass_iters = it;
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
    const size_t v = sizeof(V);
    int rc = 0;
    rc |= make_map(M.zA, P.z, v, pitch, rows, kSegW, kItemBy + 2);
    rc |= make_map(M.p0A, P.p0, v, pitch, rows, kSegW, kItemBy + 2);
    rc |= make_map(M.p1A, P.p1, v, pitch, rows, kSegW, kItemBy + 2);
    rc |= make_map(M.wdA, P.wd, 4, pitch, rows, kItemBx, kItemBy + 1);
    rc |= make_map(M.wrA, P.wr, 4, pitch, rows, kWrW, kItemBy);
    if (v == 4) rc |= make_map(M.xB, P.dx, 4, pitch, rows, kItemBx, kItemBy);
    else rc |= make_map(M.xB, P.x, 8, pitch, rows, kItemBx, kItemBy);
    rc |= make_map(M.zB, P.z, v, pitch, rows, kItemBx, kItemBy);
    rc |= make_map(M.p0B, P.p0, v, pitch, rows, kItemBx, kItemBy);
    rc |= make_map(M.p1B, P.p1, v, pitch, rows, kItemBx, kItemBy);
    rc |= make_map(M.qB, P.q, v, pitch, rows, kItemBx, kItemBy);
    rc |= make_map(M.rB, v == 8 ? P.r : P.z, v, pitch, rows, kItemBx, kItemBy);
    rc |= make_map(M.dB, P.diag, v, pitch, rows, kItemBx, kItemBy);
    return rc ? CUPHU_ERR_CUDA : 0;
}

template <typename V, bool WLS>
static int launch_solve_kernel(const TileDesc *tiles, const int *item_tile, int nitems, int ntiles,
                          const SolverPlanes &P, int pitch, int rows, TileState *st, double *part,
                          SolverCtl *ctl, const SolveParams &sp, long long timeout_ns, int device,
                          cudaStream_t s)
{
    if (ntiles > kMaxTiles)
        return fail(CUPHU_ERR_INVALID, "at most 1024 tiles per solver launch");
    SolveMaps M;
    int rcm = make_maps<V>(M, P, pitch, rows);
    if (rcm) return rcm;
    int nsm = 0, per_sm = 0;
    CUPHU_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    const size_t smem = solve_smem_bytes<V>();
    CUPHU_TRY_CUDA(cudaFuncSetAttribute(k_solve<V, WLS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    CUPHU_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve<V, WLS>,
                                                                 kItemThreads, smem));
    if (per_sm < 1) return fail(CUPHU_ERR_CUDA, "solver kernel cannot be resident");
    /* blocks per SM from the autotuner (job size = item count) */
    tune_note_items(nitems);
    const int tuned = tune_get(device, 1, (long long)nitems);
    if (tuned >= 1) per_sm = std::min(per_sm, tuned);
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
    CUPHU_TRY_CUDA(cudaLaunchKernelEx(&cfg, k_solve<V, WLS>, tiles, item_tile, nitems, ntiles, P, st,
                                      part, ctl, sp, timeout_ns, M));
    return 0;
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

int launch_solve(bool fp64, const TileDesc *tiles, const int *item_tile, int nitems,
                 int ntiles, const SolverPlanes &P, int plane_pitch, int plane_rows,
                 TileState *st, double *part, SolverCtl *ctl, const SolveParams &sp,
                 int device, cudaStream_t s)
{
    long long timeout_ns = sp.timeout_ns;
    if (fp64)
        return launch_solve_t<double>(tiles, item_tile, nitems, ntiles, P, plane_pitch, plane_rows,
                                      st, part, ctl, sp, timeout_ns, device, s);
    return launch_solve_t<float>(tiles, item_tile, nitems, ntiles, P, plane_pitch, plane_rows, st,
                                 part, ctl, sp, timeout_ns, device, s);
}

}  // namespace cuphu
