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

#include <cuda/atomic>
#include <vector>

namespace cuphu {

constexpr int kHaloW = kItemBx + 2;
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

/* Item partial -> per-tile ticket; the last block of the tile reduces the
 * tile's item partials in fixed order.  Returns true in the last block;
 * *total is valid in its thread 0. */
__device__ __forceinline__ bool item_reduce(double acc, const TileDesc &T, int t, int item,
                                            double *part, TileState *st, double *sw,
                                            int *s_last, double *total)
{
    double bs = block_sum(acc, sw);
    if (threadIdx.x == 0) {
        part[item] = bs;
        __threadfence();
        unsigned prev = atomicAdd(&st[t].ticket, 1u);
        *s_last = (prev == (unsigned)T.nitems - 1u);
    }
    __syncthreads();
    if (!*s_last) return false;
    __threadfence();
    double a = 0.0;
    for (int i = threadIdx.x; i < T.nitems; i += blockDim.x) a = a + __ldcg(part + T.item0 + i);
    double tot = block_sum(a, sw);
    if (threadIdx.x == 0) {
        st[t].ticket = 0u;
        *total = tot;
    }
    return true;
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
template <typename V>
__device__ double phase_init(const TileDesc &T, int li, const SolverPlanes &P, bool zero_x,
                             bool write_diag)
{
    ItemXY q = item_xy(T, li);
    if (q.r >= T.nr || q.c0 >= T.nc) return 0.0;
    V *x = (V *)P.x + T.pix;
    V *rr = (V *)P.r + T.pix;
    V *dg = (V *)P.diag + T.pix;
    const float *wd = P.wd + T.pix, *wr = P.wr + T.pix;
    const float *ph = T.ph;
    const double eps = (double)kLapEpsF;
    const int r = q.r, nr = T.nr, nc = T.nc, pitch = T.pitch, pp = T.ph_pitch;
    size_t prow = (size_t)r * pitch;
    V xv[4], rv[4], dv[4];
    if (!zero_x) ld4(x + prow + q.c0, xv);
    if (!write_diag) ld4(dg + prow + q.c0, dv);
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        int c = q.c0 + j;
        if (c >= nc) {
            rv[j] = (V)0;
            if (write_diag) dv[j] = (V)0;
            if (zero_x) xv[j] = (V)0;
            continue;
        }
        size_t gi = (size_t)r * pp + c, pi = prow + c;
        float pa = __ldg(ph + gi);
        double bv = 0.0, ws = 0.0;
        if (r < nr - 1) {
            float w = ldc(wd + pi);
            if (w > 0.0f) {
                float g = lap_wrap_pi(__ldg(ph + gi + pp) - pa);
                bv = __fma_rn(-(double)w, (double)g, bv);
                ws += w;
            }
        }
        if (r > 0) {
            float w = ldc(wd + pi - pitch);
            if (w > 0.0f) {
                float g = lap_wrap_pi(pa - __ldg(ph + gi - pp));
                bv = __fma_rn((double)w, (double)g, bv);
                ws += w;
            }
        }
        if (c < nc - 1) {
            float w = ldc(wr + pi);
            if (w > 0.0f) {
                float g = lap_wrap_pi(__ldg(ph + gi + 1) - pa);
                bv = __fma_rn(-(double)w, (double)g, bv);
                ws += w;
            }
        }
        if (c > 0) {
            float w = ldc(wr + pi - 1);
            if (w > 0.0f) {
                float g = lap_wrap_pi(pa - __ldg(ph + gi - 1));
                bv = __fma_rn((double)w, (double)g, bv);
                ws += w;
            }
        }
        double d = write_diag ? ws + eps : (double)dv[j];
        double y;
        if (zero_x) {
            y = 0.0;
            xv[j] = (V)0;
        } else {
            double xa = (double)xv[j];
            y = eps * xa;
            if (r < nr - 1) y = __fma_rn((double)ldc(wd + pi), xa - (double)ldc(x + pi + pitch), y);
            if (r > 0)      y = __fma_rn((double)ldc(wd + pi - pitch), xa - (double)ldc(x + pi - pitch), y);
            if (c < nc - 1) y = __fma_rn((double)ldc(wr + pi), xa - (double)ldc(x + pi + 1), y);
            if (c > 0)      y = __fma_rn((double)ldc(wr + pi - 1), xa - (double)ldc(x + pi - 1), y);
        }
        V rs = (V)(bv - y);
        V ds = (V)d;
        double z = (double)rs / (double)ds;
        acc = __fma_rn((double)rs, z, acc);
        rv[j] = rs;
        if (write_diag) dv[j] = ds;
    }
    st4(rr + prow + q.c0, rv);
    if (write_diag) st4(dg + prow + q.c0, dv);
    if (zero_x) st4(x + prow + q.c0, xv);
    return acc;
}

/* ── stencil pass: p_new = z + beta p_old (own + halo, in shared memory),
 *    q = A p_new, partial p.q ─────────────────────────────────────────── */
template <typename V>
__device__ double phase_a(const TileDesc &T, int li, const SolverPlanes &P, const V *pold_all,
                          V *pnew_all, bool first, double beta, V *smP)
{
    ItemXY q = item_xy(T, li);
    const V *rr = (const V *)P.r + T.pix;
    const V *dg = (const V *)P.diag + T.pix;
    const V *po = pold_all + T.pix;
    V *pn_out = pnew_all + T.pix;
    V *qo = (V *)P.q + T.pix;
    const float *wd = P.wd + T.pix, *wr = P.wr + T.pix;
    const int nr = T.nr, nc = T.nc, pitch = T.pitch, r = q.r;
    const bool own = r < nr && q.c0 < nc;
    size_t prow = (size_t)r * pitch;
    V pn[4] = {(V)0, (V)0, (V)0, (V)0};
    if (own) {
        V rv[4], dv[4], pv[4];
        ld4(rr + prow + q.c0, rv);
        ld4(dg + prow + q.c0, dv);
        if (!first) ld4(po + prow + q.c0, pv);
#pragma unroll
        for (int j = 0; j < kItemVx; ++j) {
            if (q.c0 + j >= nc) continue;
            double z = (double)rv[j] / (double)dv[j];
            pn[j] = (V)(first ? z : __fma_rn(beta, (double)pv[j], z));
        }
    }
    const int srow = (q.ty + 1) * kHaloW + q.tx * kItemVx + 1;
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) smP[srow + j] = pn[j];
    /* halo ring (no corners: 5-point stencil) */
    const int rb = (li / T.nbx) * kItemBy, cb = (li % T.nbx) * kItemBx;
    for (int h = threadIdx.x; h < 2 * kItemBx + 2 * kItemBy; h += blockDim.x) {
        int hr, hc, sidx;
        if (h < kItemBx) { hr = rb - 1; hc = cb + h; sidx = h + 1; }
        else if (h < 2 * kItemBx) { hr = rb + kItemBy; hc = cb + h - kItemBx; sidx = (kItemBy + 1) * kHaloW + h - kItemBx + 1; }
        else if (h < 2 * kItemBx + kItemBy) { hr = rb + h - 2 * kItemBx; hc = cb - 1; sidx = (hr - rb + 1) * kHaloW; }
        else { hr = rb + h - 2 * kItemBx - kItemBy; hc = cb + kItemBx; sidx = (hr - rb + 1) * kHaloW + kItemBx + 1; }
        V v = (V)0;
        if (hr >= 0 && hr < nr && hc >= 0 && hc < nc) {
            size_t pi = (size_t)hr * pitch + hc;
            double z = (double)ldc(rr + pi) / (double)ldc(dg + pi);
            v = (V)(first ? z : __fma_rn(beta, (double)ldc(po + pi), z));
        }
        smP[sidx] = v;
    }
    __syncthreads();
    double acc = 0.0;
    if (own) {
        float wdn[4], wup[4] = {0.f, 0.f, 0.f, 0.f}, wrt[4];
        ld4(wd + prow + q.c0, wdn);
        if (r > 0) ld4(wd + prow - pitch + q.c0, wup);
        ld4(wr + prow + q.c0, wrt);
        float wlf = q.c0 > 0 ? ldc(wr + prow + q.c0 - 1) : 0.0f;
        V qv[4] = {(V)0, (V)0, (V)0, (V)0};
        const double eps = (double)kLapEpsF;
#pragma unroll
        for (int j = 0; j < kItemVx; ++j) {
            int c = q.c0 + j;
            if (c >= nc) continue;
            int s = srow + j;
            double xa = (double)pn[j];
            double y = eps * xa;
            if (r < nr - 1) y = __fma_rn((double)wdn[j], xa - (double)smP[s + kHaloW], y);
            if (r > 0)      y = __fma_rn((double)wup[j], xa - (double)smP[s - kHaloW], y);
            if (c < nc - 1) y = __fma_rn((double)wrt[j], xa - (double)smP[s + 1], y);
            if (c > 0)      y = __fma_rn((double)(j == 0 ? wlf : wrt[j - 1]), xa - (double)smP[s - 1], y);
            qv[j] = (V)y;
            acc = __fma_rn((double)pn[j], (double)qv[j], acc);
        }
        st4(pn_out + prow + q.c0, pn);
        st4(qo + prow + q.c0, qv);
    }
    __syncthreads();
    return acc;
}

/* ── update pass: x += alpha p, r -= alpha q, z = r/diag, partial r.z ──── */
template <typename V>
__device__ double phase_b(const TileDesc &T, int li, const SolverPlanes &P, const V *pnew_all,
                          double alpha, bool update_r)
{
    ItemXY q = item_xy(T, li);
    if (q.r >= T.nr || q.c0 >= T.nc) return 0.0;
    size_t o = T.pix + (size_t)q.r * T.pitch + q.c0;
    V *x = (V *)P.x + o;
    V *rr = (V *)P.r + o;
    V xv[4], pv[4], qv[4], rv[4], dv[4];
    ld4(x, xv);
    ld4(pnew_all + o, pv);
    if (update_r) {
        ld4((const V *)P.q + o, qv);
        ld4(rr, rv);
        ld4((const V *)P.diag + o, dv);
    }
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        if (q.c0 + j >= T.nc) continue;
        xv[j] = (V)__fma_rn(alpha, (double)pv[j], (double)xv[j]);
        if (update_r) {
            V rn = (V)__fma_rn(-alpha, (double)qv[j], (double)rv[j]);
            rv[j] = rn;
            double z = (double)rn / (double)dv[j];
            acc = __fma_rn((double)rn, z, acc);
        }
    }
    st4(x, xv);
    if (update_r) st4(rr, rv);
    return acc;
}

/* ── IRLS reweight (A13): w = w0 / sqrt(e^2 + delta^2) ───────────────────── */
template <typename V>
__device__ void phase_rw(const TileDesc &T, int li, const SolverPlanes &P, float delta)
{
    ItemXY q = item_xy(T, li);
    if (q.r >= T.nr || q.c0 >= T.nc) return;
    const V *x = (const V *)P.x + T.pix;
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
        double xa = (double)ldc(x + pi);
        float pa = __ldg(T.ph + gi);
        if (r < nr - 1) {
            float w0 = __ldg(P.w0d + T.pix + pi);
            if (w0 > 0.0f) {
                float g = lap_wrap_pi(__ldg(T.ph + gi + pp) - pa);
                double e = ((double)ldc(x + pi + pitch) - xa) - (double)g;
                wdo[j] = (float)((double)w0 / __dsqrt_rn(__fma_rn(e, e, dd)));
            }
        }
        if (c < nc - 1) {
            float w0 = __ldg(P.w0r + T.pix + pi);
            if (w0 > 0.0f) {
                float g = lap_wrap_pi(__ldg(T.ph + gi + 1) - pa);
                double e = ((double)ldc(x + pi + 1) - xa) - (double)g;
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
    const V *x = (const V *)P.x + T.pix;
    double off = (double)__ldg(T.ph) - (double)ldc(x);
    size_t prow = (size_t)q.r * T.pitch;
    float uo[4] = {0.f, 0.f, 0.f, 0.f}, co[4] = {0.f, 0.f, 0.f, 0.f};
    int ko[4] = {0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < kItemVx; ++j) {
        int c = q.c0 + j;
        if (c >= T.nc) continue;
        float ph = __ldg(T.ph + (size_t)q.r * T.ph_pitch + c);
        double u = (double)ldc(x + prow + c) + off;
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

__device__ __forceinline__ void finish_iter(TileState &S, double rzn, int max_iter, SolverCtl *ctl)
{
    S.iter += 1;
    if (rzn < S.thr || S.iter >= max_iter) {
        S.active = 0;
        atomicSub(&ctl->n_active, 1);
    } else {
        S.beta = rzn / S.rz;
        S.rz = rzn;
    }
}

template <typename V>
__global__ void __launch_bounds__(kItemThreads) k_solve(const TileDesc *__restrict__ tiles,
                                                        const int *__restrict__ item_tile,
                                                        int nitems, SolverPlanes P,
                                                        TileState *st, double *part,
                                                        SolverCtl *ctl, SolveParams sp,
                                                        long long timeout_ns)
{
    __shared__ V smP[kHaloH * kHaloW];
    __shared__ double sw[32];
    __shared__ int s_last;
    const bool mixed = sizeof(V) == 4;
    V *pb[2] = {(V *)P.p0, (V *)P.p1};
    double tot = 0.0;

    for (int outer = 0; outer <= sp.n_irls; ++outer) {
        /* assemble b, diag; r = b - A x; rz0 */
        for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
            int t = item_tile[item];
            const TileDesc &T = tiles[t];
            double acc = phase_init<V>(T, item - T.item0, P, outer == 0, true);
            if (item_reduce(acc, T, t, item, part, st, sw, &s_last, &tot) && threadIdx.x == 0) {
                TileState &S = st[t];
                S.rz = tot;
                S.rz0 = tot;
                S.thr = (double)sp.tol * (double)sp.tol * tot;
                S.iter = 0;
                S.beta = 0.0;
                S.active = tot > 0.0 ? 1 : 0;
                if (S.active) atomicAdd(&ctl->n_active, 1);
            }
        }
        if (!grid_sync(ctl, timeout_ns)) return;

        int it = 0;
        while (*(volatile int *)&ctl->snap > 0 && it < sp.max_iter) {
            const V *pold = pb[it & 1];
            V *pnew = pb[(it + 1) & 1];
            for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
                int t = item_tile[item];
                if (!*(volatile int *)&st[t].active) continue;
                const TileDesc &T = tiles[t];
                double beta = *(volatile double *)&st[t].beta;
                double acc = phase_a<V>(T, item - T.item0, P, pold, pnew, it == 0, beta, smP);
                if (item_reduce(acc, T, t, item, part, st, sw, &s_last, &tot) && threadIdx.x == 0) {
                    TileState &S = st[t];
                    if (tot <= 0.0) {
                        S.active = 0;
                        atomicSub(&ctl->n_active, 1);
                    } else {
                        S.alpha = S.rz / tot;
                    }
                }
            }
            if (!grid_sync(ctl, timeout_ns)) return;
            const bool repl = mixed && sp.replace_every > 0 && ((it + 1) % sp.replace_every) == 0;
            for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
                int t = item_tile[item];
                if (!*(volatile int *)&st[t].active) continue;
                const TileDesc &T = tiles[t];
                double alpha = *(volatile double *)&st[t].alpha;
                double acc = phase_b<V>(T, item - T.item0, P, pnew, alpha, !repl);
                if (!repl && item_reduce(acc, T, t, item, part, st, sw, &s_last, &tot) &&
                    threadIdx.x == 0)
                    finish_iter(st[t], tot, sp.max_iter, ctl);
            }
            if (!grid_sync(ctl, timeout_ns)) return;
            if (repl) {
                for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
                    int t = item_tile[item];
                    if (!*(volatile int *)&st[t].active) continue;
                    const TileDesc &T = tiles[t];
                    double acc = phase_init<V>(T, item - T.item0, P, false, false);
                    if (item_reduce(acc, T, t, item, part, st, sw, &s_last, &tot) &&
                        threadIdx.x == 0)
                        finish_iter(st[t], tot, sp.max_iter, ctl);
                }
                if (!grid_sync(ctl, timeout_ns)) return;
            }
            ++it;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            if (sp.pass_iters) sp.pass_iters[outer] = it;
            ctl->total_iters += it;
            if (it > ctl->max_pass_iters) ctl->max_pass_iters = it;
        }
        if (outer < sp.n_irls) {
            float delta = sp.deltas[outer];
            for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
                int t = item_tile[item];
                const TileDesc &T = tiles[t];
                phase_rw<V>(T, item - T.item0, P, delta);
            }
            if (!grid_sync(ctl, timeout_ns)) return;
        }
    }
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        int t = item_tile[item];
        const TileDesc &T = tiles[t];
        phase_final<V>(T, item - T.item0, P);
    }
}

template <typename V>
static int launch_solve_t(const TileDesc *tiles, const int *item_tile, int nitems,
                          const SolverPlanes &P, TileState *st, double *part, SolverCtl *ctl,
                          const SolveParams &sp, long long timeout_ns, int device,
                          cudaStream_t s)
{
    int nsm = 0, per_sm = 0;
    CUPHU_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    CUPHU_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve<V>,
                                                                 kItemThreads, 0));
    if (per_sm < 1) return fail(CUPHU_ERR_CUDA, "solver kernel cannot be resident");
    int grid = std::min(nsm * per_sm, std::max(nitems, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kItemThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUPHU_TRY_CUDA(cudaLaunchKernelEx(&cfg, k_solve<V>, tiles, item_tile, nitems, P, st, part,
                                      ctl, sp, timeout_ns));
    return 0;
}

int launch_solve(bool fp64, const TileDesc *tiles, const int *item_tile, int nitems,
                 int ntiles, const SolverPlanes &P, TileState *st, double *part,
                 SolverCtl *ctl, const SolveParams &sp, int device, cudaStream_t s)
{
    (void)ntiles;
    long long timeout_ns = sp.timeout_ns;
    if (fp64)
        return launch_solve_t<double>(tiles, item_tile, nitems, P, st, part, ctl, sp,
                                      timeout_ns, device, s);
    return launch_solve_t<float>(tiles, item_tile, nitems, P, st, part, ctl, sp, timeout_ns,
                                 device, s);
}

}  // namespace cuphu
