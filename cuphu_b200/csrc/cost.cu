/*
 * cost.cu -- wrapped phase, statistical costs, residues.
 *
 *  k_phase       A1: igram (complex64) -> wrapped phase in [0,2pi)
 *  k_costs       A2+A3+A5/A6(+A7)(+A8): one fused pass per 2-D block of arcs:
 *                wrapped differences of a mirror-padded halo window are formed
 *                in shared memory, box-car averaged in the reference summation
 *                order (row pass over padded rows, then column pass), and
 *                quantised to the int16 SNAPHU cost structs; residues of the
 *                same block are emitted from the same staged phase.
 *  k_w0          A5/A6 sigsq -> Laplace data weight w0 = 1/sigsq per arc,
 *                written straight into the solver's pitched arc planes.  The
 *                Laplace path only consumes sigsq, which depends on
 *                coherence alone, so this kernel skips the phase-gradient work
 *                the reference performs and discards.
 *  k_residues    A8 standalone.
 *
 * Reference: cuphu_util.cu:27-287, cuphu_cost.cu:41-479,
 *            cuphu_solver.cpp:397-450, 1706-1712.
 */
#include "common.cuh"
#include "kernels.cuh"

#include <cmath>

namespace cuphu {

CostConsts make_cost_consts(const CuPhuParams &p)
{
    /* host arithmetic of upload_smooth_constants (cuphu_cost.cu:41-59); this
     * translation unit is compiled with -ffp-contract=off on the host side */
    CostConsts k;
    k.rho0 = p.rhosconst1 / p.ncorrlooks + p.rhosconst2;
    k.thresh = p.defothreshfactor * k.rho0;
    k.rhopow = 2.0 * p.cstd1 + p.cstd2 * std::log(p.ncorrlooks) + p.cstd3 * p.ncorrlooks;
    k.sigsqrhoconst = 2.0 / 12.0;
    k.sigsqcorr = p.sigsqcorr;
    k.nsc = p.nshortcycle;
    k.nsc2 = p.nshortcycle * p.nshortcycle;
    k.costscale = p.costscale;
    k.defomax = p.defomax;
    k.sigsqshortmin = (int)p.sigsqshortmin;
    k.rhopow_f = (float)k.rhopow;
    k.screen = 1e-5 * (1.0 + std::fabs(k.rhopow));
    k.screen_f = (float)(k.screen + 2e-6);
    k.sig_f = (float)k.sigsqrhoconst;
    k.corr_f = (float)k.sigsqcorr;
    k.scale_f = (float)(k.nsc2 / k.costscale);
    /* dzmax = clamp(rn(nsc*defomax), 1, 32767) (cuphu_cost.cu:250-251) is a
     * per-launch constant; the FP64 product is exact as on the device */
    double dz = std::nearbyint(k.nsc * k.defomax);
    int dzi = (dz != dz) ? 0 : (dz >= 2147483647.0 ? 2147483647 : (dz <= -2147483648.0 ? (int)-2147483647 - 1 : (int)dz));
    k.dzmax = std::max(1, std::min(dzi, 32767));
    return k;
}

/* ── A1 ──────────────────────────────────────────────────────────────────
 * The reference takes atan2f on the host (glibc) and re-wraps on the device.
 * Here the angle is atan2 in FP64 rounded once to float (the correctly
 * rounded float angle except in double-rounding ties), then shifted and
 * re-wrapped with the reference's float operations.  glibc 2.39 atan2f is not
 * correctly rounded, so about one pixel in seven differs from the host value
 * by one ulp; callers needing the host phase bit for bit pass phase_in. */
__global__ void __launch_bounds__(256) k_phase(const float2 *__restrict__ ig,
                                               float *__restrict__ ph, long long n)
{
    long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float2 v = ig[i];
        if (!(isfinite(v.x) && isfinite(v.y))) { v.x = 0.0f; v.y = 0.0f; }
        float phi = (float)atan2((double)v.y, (double)v.x);
        if (phi < 0.0f) phi = __fadd_rn(phi, kTwoPiF);
        ph[i] = rewrap_2pi(phi);
    }
}

/* split real/imaginary planes (the C drop-in cuphu_unwrap signature) */
__global__ void __launch_bounds__(256) k_phase_split(const float *__restrict__ re,
                                                     const float *__restrict__ im,
                                                     float *__restrict__ ph, long long n)
{
    long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float x = re[i], y = im[i];
        if (!(isfinite(x) && isfinite(y))) { x = 0.0f; y = 0.0f; }
        float phi = (float)atan2((double)y, (double)x);
        if (phi < 0.0f) phi = __fadd_rn(phi, kTwoPiF);
        ph[i] = rewrap_2pi(phi);
    }
}

/* ── per-arc quantised cost, cuphu_cost.cu:98-132 (smooth), 225-265 (defo) */
struct ArcCost {
    short off, sigsq, dzmax, laycost;
};

/* hardware 2^x (MUFU EX2, 2 ulp) */
__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

/* (int)sigsq_f of the reference (cuphu_cost.cu:109-117) for a coherence rho
 * already thresholded.  The FP64 pow dominates the kernel's cost, and only
 * the truncated value matters, so it is screened first with an FP32 pow
 * estimate through the reference's FP64 formula; whenever the interval of
 * +-1e-5 (1 + |rhopow|) relative around it (40x the estimate's error bound)
 * contains no integer the truncated result is certain.  Everything else (intervals that straddle an integer,
 * bases outside (0,1], non-positive weights) takes the exact FP64 path, so
 * the result is bit-identical to the reference arithmetic. */
__device__ __forceinline__ int trunc_sigsq(double rho, short w, const CostConsts &k)
{
    double b = 1.0 - rho;
    if (w > 0 && b > 0.0 && b <= 1.0) {
        /* MUFU log2/exp2 (|error of log2| <= 2^-22 abs on [0.5,2], 2 ulp
         * elsewhere; exp2 2 ulp) and FP32 arithmetic (< 6 ulp): the relative
         * error of v stays below 3e-7 (1 + |rhopow|) + 1e-6; the screen keeps
         * a >= 10x margin */
        float pw = ex2_approx(k.rhopow_f * __log2f((float)b));
        float v = __fmaf_rn(k.sig_f, pw, k.corr_f) * k.scale_f;
        if (w != 1) v = __fdiv_rn(v, (float)w);
        float m = __fmaf_rn(k.screen_f, v, 1e-6f);
        float lo = floorf(v - m);
        if (lo == floorf(v + m) && lo >= 0.0f && v + m < 1.0e7f) return (int)lo;
    }
    double sigsqrho = __dmul_rn(__fma_rn(k.sigsqrhoconst, pow(b, k.rhopow), k.sigsqcorr), k.nsc2);
    return (int)(sigsqrho / (k.costscale * (double)w));
}

__device__ __forceinline__ int sigsq_of(double ca, double cb, short w, const CostConsts &k)
{
    double rho = 0.5 * (ca + cb);
    if (rho < k.thresh) rho = 0.0;
    int s = trunc_sigsq(rho, w, k);
    if (s < k.sigsqshortmin) s = k.sigsqshortmin;
    return s;
}

/* (int)sqrt((double)n) of the reference: floor(sqrt(n)) for n >= 0 (a
 * correctly rounded FP64 sqrt never crosses an integer for n < 2^52), and
 * NaN -> 0 for a negative (wrapped) product.  FP32 estimate, exact fix-up. */
__device__ __forceinline__ int isqrt_floor(int n)
{
    if (n <= 0) return 0;
    int s = (int)sqrtf((float)n);
    while ((long long)s * s > n) --s;
    while ((long long)(s + 1) * (s + 1) <= n) ++s;
    return s;
}

template <bool DEFO>
__device__ __forceinline__ ArcCost arc_cost(double ca, double cb, float dpsi, float avg, short w,
                                            const CostConsts &k)
{
    ArcCost o;
    if (w == 0) {
        o.off = kLargeShort / 2; o.sigsq = kLargeShort;
        o.dzmax = kLargeShort; o.laycost = 0;
        return o;
    }
    double rho = 0.5 * (ca + cb);
    if (rho < k.thresh) rho = 0.0;
    double dp = (double)dpsi, av = (double)avg;
    double offset = __dmul_rn(k.nsc, __dsub_rn(dp, rho > 0 ? av : __dmul_rn(0.5, av)));
    int sigsq_i = trunc_sigsq(rho, w, k);
    if (sigsq_i < k.sigsqshortmin) sigsq_i = k.sigsqshortmin;
    int off_i;
    int dzmax = 0, laycost = 0;
    if (DEFO) {
        dzmax = k.dzmax;
        laycost = isqrt_floor(dzmax * sigsq_i);   /* (int)sqrt((double)n), n < 0 -> 0 */
        laycost = min(laycost, (int)SHRT_MAX);
        off_i = __double2int_rn(offset);
    } else {
        off_i = (int)offset;
    }
    off_i = max(off_i, (int)SHRT_MIN);
    off_i = min(off_i, (int)SHRT_MAX);
    sigsq_i = min(sigsq_i, (int)SHRT_MAX);
    o.off = (short)off_i; o.sigsq = (short)sigsq_i;
    o.dzmax = (short)dzmax; o.laycost = (short)laycost;
    return o;
}

/* ── fused cost kernel ─────────────────────────────────────────────────────
 * Block = 256 threads producing a kCostBy x kCostBx block of arcs of one
 * family.  family 0 = row arcs (r,c)->(r+1,c), azimuth diffs, array
 * (nrow-1) x ncol, window (kpar/2 rows, kperp/2 cols); family 1 = col arcs
 * (r,c)->(r,c+1), range diffs, nrow x (ncol-1), window (kperp/2, kpar/2).
 * Interior blocks stage the phase window in shared memory with coalesced
 * loads and form the differences from it; blocks whose window crosses the
 * array edge read the mirror-reflected phase directly.  KR/KC > 0 fix the
 * half windows at compile time (the default 7x7 window); 0 = runtime. */
constexpr int kCostBx = 64;
constexpr int kCostBy = 32;

template <bool DEFO, int KR0, int KC0>
__global__ void __launch_bounds__(256) k_costs(const float *__restrict__ ph,
                                               const float *__restrict__ corr,
                                               const short *__restrict__ weights, int nrow,
                                               int ncol, int kperp, int kpar, CostConsts k,
                                               void *__restrict__ costs_out,
                                               signed char *__restrict__ res_out, int nbx0,
                                               int nby0, int nbx1)
{
    extern __shared__ float sm[];
    int b = blockIdx.x;
    int fam, by, bx;
    if (b < nbx0 * nby0) { fam = 0; by = b / nbx0; bx = b % nbx0; }
    else { b -= nbx0 * nby0; fam = 1; by = b / nbx1; bx = b % nbx1; }

    const int dr = fam == 0 ? nrow - 1 : nrow;      /* diff array rows */
    const int dc = fam == 0 ? ncol : ncol - 1;      /* diff array cols */
    /* with a compile-time square window both families share kr == kc */
    const int kr = KR0 > 0 ? KR0 : (fam == 0 ? kpar / 2 : kperp / 2);
    const int kc = KC0 > 0 ? KC0 : (fam == 0 ? kperp / 2 : kpar / 2);
    const int wr = 2 * kr + 1, wc = 2 * kc + 1;
    const int pr = kCostBy + 2 * kr, pc = kCostBx + 2 * kc;
    float *D = sm;                 /* pr x pc padded diffs          */
    float *T = sm + pr * pc;       /* pr x kCostBx row-pass results */
    float *PH = T + pr * kCostBx;  /* phase window (interior blocks) */
    const int r0 = by * kCostBy, c0 = bx * kCostBx;
    const bool interior = r0 - kr >= 0 && r0 + kCostBy + kr <= dr && c0 - kc >= 0 &&
                          c0 + kCostBx + kc <= dc;
    if (interior) {
        /* phase window: family 0 needs pr+1 rows x pc cols, family 1 pr x pc+1 */
        const int hr = pr + (fam == 0 ? 1 : 0), hc = pc + (fam == 1 ? 1 : 0);
        const int pr0 = r0 - kr, pc0 = c0 - kc;
        for (int i = threadIdx.x; i < hr * hc; i += blockDim.x) {
            int ii = i / hc, jj = i - ii * hc;
            PH[i] = ph[(size_t)(pr0 + ii) * ncol + pc0 + jj];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < pr * pc; i += blockDim.x) {
            int ii = i / pc, jj = i - ii * pc;
            float d;
            if (fam == 0) d = __fdiv_rn(PH[ii * hc + jj] - PH[(ii + 1) * hc + jj], kTwoPiF);
            else d = __fdiv_rn(PH[ii * hc + jj + 1] - PH[ii * hc + jj], kTwoPiF);
            D[i] = wrap_cycles(d);
        }
    } else {
        for (int i = threadIdx.x; i < pr * pc; i += blockDim.x) {
            int ii = i / pc, jj = i - ii * pc;
            int sr = reflect_index(r0 + ii - kr, dr);
            int sc = reflect_index(c0 + jj - kc, dc);
            float d;
            if (fam == 0)
                d = __fdiv_rn(ph[(size_t)sr * ncol + sc] - ph[(size_t)(sr + 1) * ncol + sc], kTwoPiF);
            else
                d = __fdiv_rn(ph[(size_t)sr * ncol + sc + 1] - ph[(size_t)sr * ncol + sc], kTwoPiF);
            D[i] = wrap_cycles(d);
        }
    }
    __syncthreads();
    /* row pass: sum k = 0..wc-1 ascending, then divide (cuphu_util.cu:116-121) */
    const float fwc = (float)wc, fwr = (float)wr;
    for (int i = threadIdx.x; i < pr * kCostBx; i += blockDim.x) {
        int ii = i / kCostBx, jj = i % kCostBx;
        const float *row = D + ii * pc + jj;
        float s = 0.0f;
        for (int q = 0; q < wc; ++q) s = __fadd_rn(s, row[q]);
        T[i] = __fdiv_rn(s, fwc);
    }
    __syncthreads();
    size_t nra = (size_t)(nrow - 1) * ncol;
    for (int i = threadIdx.x; i < kCostBy * kCostBx; i += blockDim.x) {
        int ii = i / kCostBx, jj = i % kCostBx;
        int ar = r0 + ii, ac = c0 + jj;
        if (ar >= dr || ac >= dc) continue;
        /* column pass (cuphu_util.cu:143-147) */
        float s = 0.0f;
        for (int q = 0; q < wr; ++q) s = __fadd_rn(s, T[(ii + q) * kCostBx + jj]);
        float avg = __fdiv_rn(s, fwr);
        float dpsi = D[(ii + kr) * pc + jj + kc];
        size_t a;
        float ca, cb;
        if (fam == 0) {
            a = (size_t)ar * ncol + ac;
            ca = sane(corr[(size_t)ar * ncol + ac]);
            cb = sane(corr[(size_t)(ar + 1) * ncol + ac]);
        } else {
            a = nra + (size_t)ar * (ncol - 1) + ac;
            ca = sane(corr[(size_t)ar * ncol + ac]);
            cb = sane(corr[(size_t)ar * ncol + ac + 1]);
        }
        short w = weights ? weights[a] : (short)1;
        ArcCost o = arc_cost<DEFO>((double)ca, (double)cb, dpsi, avg, w, k);
        if (DEFO) {
            short4 v = make_short4(o.off, o.sigsq, o.dzmax, o.laycost);
            reinterpret_cast<short4 *>(costs_out)[a] = v;
        } else {
            short2 v = make_short2(o.off, o.sigsq);
            reinterpret_cast<short2 *>(costs_out)[a] = v;
        }
        /* residue of plaquette (ar, ac) from the col-arc family blocks */
        if (res_out && fam == 1 && ar < nrow - 1 && ac < ncol - 1) {
            const float *p0 = ph + (size_t)ar * ncol + ac;
            const float *p1 = p0 + ncol;
            float rng0 = wrap_cycles(__fdiv_rn(p0[1] - p0[0], kTwoPiF));
            float rng1 = wrap_cycles(__fdiv_rn(p1[1] - p1[0], kTwoPiF));
            float az0 = wrap_cycles(__fdiv_rn(p0[0] - p1[0], kTwoPiF));
            float az1 = wrap_cycles(__fdiv_rn(p0[1] - p1[1], kTwoPiF));
            float rs = __fadd_rn(__fsub_rn(__fsub_rn(rng0, az1), rng1), az0);
            res_out[(size_t)ar * (ncol - 1) + ac] = (signed char)rintf(rs);
        }
    }
}

/* ── A8 standalone ──────────────────────────────────────────────────────── */
__global__ void __launch_bounds__(256) k_residues(const float *__restrict__ ph, int nrow,
                                                  int ncol, signed char *__restrict__ out)
{
    long long n = (long long)(nrow - 1) * (ncol - 1);
    long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int r = (int)(i / (ncol - 1)), c = (int)(i % (ncol - 1));
        const float *p0 = ph + (size_t)r * ncol + c;
        const float *p1 = p0 + ncol;
        float rng0 = wrap_cycles(__fdiv_rn(p0[1] - p0[0], kTwoPiF));
        float rng1 = wrap_cycles(__fdiv_rn(p1[1] - p1[0], kTwoPiF));
        float az0 = wrap_cycles(__fdiv_rn(p0[0] - p1[0], kTwoPiF));
        float az1 = wrap_cycles(__fdiv_rn(p0[1] - p1[1], kTwoPiF));
        float rs = __fadd_rn(__fsub_rn(__fsub_rn(rng0, az1), rng1), az0);
        out[i] = (signed char)rintf(rs);
    }
}

/* ── w0 planes for the solver (tile batched) ───────────────────────────────
 * One thread per tile pixel handles its down arc and its right arc:
 * w0 = 1/sigsq (float) unless sigsq <= 0 or >= 32000 (cuphu_laplace.cu:65-69);
 * arcs touching a mask-0 pixel get the masked-arc sigsq 32000 -> w0 = 0
 * (cuphu_cost.cu:98-103, cuphu_solver.cpp:404-426). Writes w0 and the
 * initial IRLS weight w = w0. */
__global__ void __launch_bounds__(256) k_w0(const TileDesc *__restrict__ tiles,
                                            const int *__restrict__ item_tile, int nitems,
                                            const CostConsts *__restrict__ scene_k,
                                            SolverPlanes P)
{
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        int t = item_tile[item];
        const TileDesc &T = tiles[t];
        int li = item - T.item0;
        int iby = li / T.nbx, ibx = li % T.nbx;
        int ty = threadIdx.x / kItemTx, tx = threadIdx.x % kItemTx;
        int r = iby * kItemBy + ty;
        if (r >= T.nr) continue;
        CostConsts k = scene_k[T.scene];
        for (int j = 0; j < kItemVx; ++j) {
            int c = ibx * kItemBx + tx * kItemVx + j;
            if (c >= T.nc) continue;
            size_t gi = (size_t)r * T.ph_pitch + c;
            size_t pi = T.pix + (size_t)r * T.pitch + c;
            float wdn = 0.0f, wrt = 0.0f;
            const unsigned char *m = T.mask;
            float ca = sane(T.corr[gi]);
            if (r < T.nr - 1) {
                short w = (m && !(m[gi] && m[gi + T.ph_pitch])) ? 0 : 1;
                int s = w ? sigsq_of((double)ca, (double)sane(T.corr[gi + T.ph_pitch]), w, k)
                          : kLargeShort;
                s = min(s, (int)SHRT_MAX);
                short ss = (short)s;
                wdn = (ss <= 0 || ss >= kLargeShort) ? 0.0f : __frcp_rn((float)ss);
            }
            if (c < T.nc - 1) {
                short w = (m && !(m[gi] && m[gi + 1])) ? 0 : 1;
                int s = w ? sigsq_of((double)ca, (double)sane(T.corr[gi + 1]), w, k)
                          : kLargeShort;
                s = min(s, (int)SHRT_MAX);
                short ss = (short)s;
                wrt = (ss <= 0 || ss >= kLargeShort) ? 0.0f : __frcp_rn((float)ss);
            }
            P.w0d[pi] = wdn; P.w0r[pi] = wrt;
            P.wd[pi] = wdn;  P.wr[pi] = wrt;
        }
    }
}

/* w0 planes from a cost array (launcher-level Laplace entry point) */
__global__ void __launch_bounds__(256) k_w0_from_costs(const short *__restrict__ costs,
                                                       int stride, int nrow, int ncol,
                                                       int pitch, SolverPlanes P)
{
    long long n = (long long)nrow * ncol;
    size_t nra = (size_t)(nrow - 1) * ncol;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int r = (int)(i / ncol), c = (int)(i % ncol);
        size_t pi = (size_t)r * pitch + c;
        float wdn = 0.0f, wrt = 0.0f;
        if (r < nrow - 1) {
            short s = costs[((size_t)r * ncol + c) * stride + 1];
            wdn = (s <= 0 || s >= kLargeShort) ? 0.0f : __frcp_rn((float)s);
        }
        if (c < ncol - 1) {
            short s = costs[(nra + (size_t)r * (ncol - 1) + c) * stride + 1];
            wrt = (s <= 0 || s >= kLargeShort) ? 0.0f : __frcp_rn((float)s);
        }
        P.w0d[pi] = wdn; P.w0r[pi] = wrt;
        P.wd[pi] = wdn;  P.wr[pi] = wrt;
    }
}

/* ── launchers ─────────────────────────────────────────────────────────── */
int launch_phase(const float2 *ig, float *ph, long long n, cudaStream_t s)
{
    if (n <= 0) return 0;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_phase<<<blocks, 256, 0, s>>>(ig, ph, n);
    return cuda_fail(cudaGetLastError(), "k_phase");
}

int launch_phase_split(const float *re, const float *im, float *ph, long long n, cudaStream_t s)
{
    if (n <= 0) return 0;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_phase_split<<<blocks, 256, 0, s>>>(re, im, ph, n);
    return cuda_fail(cudaGetLastError(), "k_phase_split");
}

template <bool DEFO, int KR, int KC>
static void launch_costs_t(int nblocks, size_t shm, cudaStream_t s, const float *ph,
                           const float *corr, const short *weights, int nrow, int ncol, int kperp,
                           int kpar, const CostConsts &k, void *costs, signed char *res, int nbx0,
                           int nby0, int nbx1)
{
    if (shm > 48 * 1024)
        cudaFuncSetAttribute(k_costs<DEFO, KR, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)shm);
    k_costs<DEFO, KR, KC><<<nblocks, 256, shm, s>>>(ph, corr, weights, nrow, ncol, kperp, kpar, k,
                                                    costs, res, nbx0, nby0, nbx1);
}

int launch_costs(const float *ph, const float *corr, const short *weights, int nrow, int ncol,
                 int mode, const CuPhuParams &p, void *costs, signed char *res, cudaStream_t s)
{
    if (nrow < 1 || ncol < 1) return 0;
    int kperp = p.kperpdpsi, kpar = p.kpardpsi;
    if (kperp < 1 || kpar < 1 || kperp > 257 || kpar > 257)
        return fail(CUPHU_ERR_INVALID, "phase gradient window must be in [1, 257]");
    CostConsts k = make_cost_consts(p);
    int nby0 = nrow > 1 ? (nrow - 1 + kCostBy - 1) / kCostBy : 0;
    int nbx0 = nrow > 1 ? (ncol + kCostBx - 1) / kCostBx : 0;
    int nby1 = ncol > 1 ? (nrow + kCostBy - 1) / kCostBy : 0;
    int nbx1 = ncol > 1 ? (ncol - 1 + kCostBx - 1) / kCostBx : 0;
    int nblocks = nbx0 * nby0 + nbx1 * nby1;
    if (nblocks == 0) return 0;
    int kmax = std::max(kperp / 2, kpar / 2);
    size_t pr = kCostBy + 2 * kmax, pcw = kCostBx + 2 * kmax;
    size_t shm = (pr * pcw + pr * kCostBx + (pr + 1) * (pcw + 1)) * sizeof(float);
    const bool w7 = kperp / 2 == 3 && kpar / 2 == 3;
    if (mode == CUPHU_COST_SMOOTH) {
        if (w7) launch_costs_t<false, 3, 3>(nblocks, shm, s, ph, corr, weights, nrow, ncol, kperp, kpar, k, costs, res, nbx0, nby0, nbx1);
        else launch_costs_t<false, 0, 0>(nblocks, shm, s, ph, corr, weights, nrow, ncol, kperp, kpar, k, costs, res, nbx0, nby0, nbx1);
    } else {
        if (w7) launch_costs_t<true, 3, 3>(nblocks, shm, s, ph, corr, weights, nrow, ncol, kperp, kpar, k, costs, res, nbx0, nby0, nbx1);
        else launch_costs_t<true, 0, 0>(nblocks, shm, s, ph, corr, weights, nrow, ncol, kperp, kpar, k, costs, res, nbx0, nby0, nbx1);
    }
    return cuda_fail(cudaGetLastError(), "k_costs");
}

int launch_residues(const float *ph, int nrow, int ncol, signed char *res, cudaStream_t s)
{
    long long n = (long long)(nrow - 1) * (ncol - 1);
    if (n <= 0) return 0;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_residues<<<blocks, 256, 0, s>>>(ph, nrow, ncol, res);
    return cuda_fail(cudaGetLastError(), "k_residues");
}

int launch_w0(const TileDesc *tiles, const int *item_tile, int nitems, const CostConsts *sk,
              const SolverPlanes &P, cudaStream_t s)
{
    if (nitems <= 0) return 0;
    int blocks = std::min(nitems, 148 * 16);
    k_w0<<<blocks, kItemThreads, 0, s>>>(tiles, item_tile, nitems, sk, P);
    return cuda_fail(cudaGetLastError(), "k_w0");
}

int launch_w0_from_costs(const short *costs, int stride, int nrow, int ncol, int pitch,
                         const SolverPlanes &P, cudaStream_t s)
{
    long long n = (long long)nrow * ncol;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_w0_from_costs<<<blocks, 256, 0, s>>>(costs, stride, nrow, ncol, pitch, P);
    return cuda_fail(cudaGetLastError(), "k_w0_from_costs");
}

}  // namespace cuphu
