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

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>

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

    /* FP32 fast path (k_costs7): every quantity it rounds is bracketed by a
     * margin above its FP32 error bound; see arc_fast2 */
    k.fast = 0;
    k.nsc_f = (float)k.nsc;
    k.thr_lo = std::nextafter((float)(k.thresh * (1.0 - std::ldexp(1.0, -20))), 0.0f);
    k.thr_hi = std::nextafter((float)(k.thresh * (1.0 + std::ldexp(1.0, -20))), 3.0e38f);
    k.a_f = (float)(k.sigsqrhoconst * k.nsc2 / k.costscale);
    k.c_f = (float)(k.sigsqcorr * k.nsc2 / k.costscale);
    const double m_off = std::fabs(k.nsc) * std::ldexp(1.0, -22) + std::ldexp(1.0, -30);
    k.off_hm = std::nextafter((float)(0.5 - m_off), 0.0f);
    k.half_m = std::nextafter((float)(0.5 - 1e-6), 0.0f);
    /* the reference's FP64 arithmetic at rho = 0 (pow(1, rhopow) = 1) */
    double t0 = std::fma(k.sigsqrhoconst, 1.0, k.sigsqcorr);
    t0 = t0 * k.nsc2;
    t0 = t0 / (k.costscale * 1.0);
    k.s_rho0 = (t0 >= 0.0 && t0 < 1.0e6) ? (int)t0 : -1;
    const bool ok = k.nsc > 0.0 && k.nsc <= 4096.0 && (double)k.nsc_f == k.nsc &&
                    std::isfinite(k.costscale) && k.costscale > 0.0 &&
                    std::isfinite(k.sigsqrhoconst) && k.sigsqrhoconst >= 0.0 &&
                    std::isfinite(k.sigsqcorr) && k.sigsqcorr >= 0.0 &&
                    std::isfinite(k.rhopow) && k.rhopow > 0.0 && k.rhopow < 64.0 &&
                    std::isfinite(k.thresh) && k.thresh > 0.0 && k.thresh < 1.0 &&
                    std::isfinite(k.a_f) && std::isfinite(k.c_f) && k.s_rho0 >= 0 &&
                    /* v = a b^rhopow + c < 1e6 for every b in [0, 1] */
                    ((double)k.a_f * 1.001 + (double)k.c_f) * 1.001 < 1.0e6 &&
                    std::isfinite(k.nsc2);
    k.fast = ok ? 1 : 0;
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

/* ── division by the path's two constants ─────────────────────────────────
 * x / c correctly rounded for c = 2 pi (wrapped differences) and c = 7 (the
 * default box-car length), with zc = RN(1/c): q0 = RN(x zc), r = x - q0 c
 * (exact through the FMA), q = RN(q0 + r zc) -- the correction step of
 * P. Markstein, "Computation of elementary functions on the IBM RISC
 * System/6000 processor", IBM J. Res. Develop. 34(1), 1990.  An exhaustive
 * comparison with IEEE division over every float of the ranges used
 * (tests/test_const_division.py) finds it exact for 2^-104 <= |x| <= 6.6
 * when c = 2 pi, and for every |x| <= 3.6 except -0 when c = 7.  Phase
 * differences outside that range take the IEEE division; box-car sums are
 * bounded by 3.5 and never -0 (they accumulate from +0). */
constexpr float kRcpTwoPiRN = 0x1.45f306p-3f;   /* RN(1 / (float)2pi) */
constexpr float kRcp7RN = 0x1.24924ap-3f;       /* RN(1 / 7) */

__device__ __forceinline__ float div_2pi(float x)
{
    const float a = fabsf(x);
    if (!(a >= 0x1p-104f && a <= 6.6f)) return __fdiv_rn(x, kTwoPiF);
    const float q0 = __fmul_rn(x, kRcpTwoPiRN);
    const float r = __fmaf_rn(-q0, kTwoPiF, x);
    return __fmaf_rn(r, kRcpTwoPiRN, q0);
}

__device__ __forceinline__ float div_7(float x)
{
    const float q0 = __fmul_rn(x, kRcp7RN);
    const float r = __fmaf_rn(-q0, 7.0f, x);
    return __fmaf_rn(r, kRcp7RN, q0);
}

/* (int)sigsq_f of the reference (cuphu_cost.cu:109-117) for a coherence rho
 * already thresholded.  The FP64 pow dominates the kernel's cost, and only
 * the truncated value matters, so it is screened first with an FP32 pow
 * estimate through the reference's FP64 formula; whenever the interval of
 * +-1e-5 (1 + |rhopow|) relative around it (40x the estimate's error bound)
 * contains no integer the truncated result is certain.  Everything else (intervals that straddle an integer,
 * bases outside (0,1], non-positive weights) takes the exact FP64 path, so
 * the result is bit-identical to the reference arithmetic. */
/* the reference's FP64 arithmetic (cuphu_cost.cu:109-117); out of line, the
 * screen above sends it about one arc in a hundred */
__device__ __noinline__ int trunc_sigsq_exact(double b, short w, double sigsqrhoconst,
                                              double rhopow, double sigsqcorr, double nsc2,
                                              double costscale)
{
    double sigsqrho = __dmul_rn(__fma_rn(sigsqrhoconst, pow(b, rhopow), sigsqcorr), nsc2);
    return (int)(sigsqrho / (costscale * (double)w));
}

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
    /* scalars by value: the constants' struct is never address-taken, so the
     * kernels read it from the parameter bank directly */
    return trunc_sigsq_exact(b, w, k.sigsqrhoconst, k.rhopow, k.sigsqcorr, k.nsc2, k.costscale);
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

/* ── fused cost kernel, default 7 x 7 window ───────────────────────────────
 * k_costs computes the same costs for any window; this kernel is the
 * kperp/2 == kpar/2 == 3 case laid out for the instruction budget:
 *  - one family per instantiation, 64 x 64 arcs per block;
 *  - columns j and j+32 of the phase window, the differences and the row
 *    sums are stored as float2 pairs, so every stencil step -- difference,
 *    division by 2 pi, re-wrap, 7-term sums, division by 7 -- runs as paired
 *    FP32 instructions (__fadd2_rn, __ffma2_rn, __fmul2_rn: IEEE
 *    round-to-nearest per lane, the reference's per-element arithmetic);
 *  - the per-arc cost is evaluated in FP32 with error margins (arc_fast2);
 *    the few arcs whose integer results a margin cannot decide are queued in
 *    shared memory, then in a launch-wide queue that k_costs7_drain
 *    finishes with arc_cost's FP64 reference arithmetic (a block whose
 *    arcs do not fit the queue finishes them itself).
 * Summation order and rounding of the box-car follow cuphu_util.cu:104-181:
 * s = 0, s += d[k] for k = 0..6, then s / 7. */
constexpr int kC7B = 64;        /* arcs per block edge */
constexpr int kC7W = kC7B + 6;  /* padded difference window edge */
constexpr int kC7H = 32;        /* pairing distance: (column j, column j + 32) */
constexpr int kC7PP = 40;       /* float2 pitch of the paired planes */
constexpr int kC7Q = 256;       /* deferred arcs per block */
constexpr int kC7Tab = 1024;    /* laycost table entries */

struct C7Deferred {
    float ca, cb, dp, av;
    int rc, w;
};
/* TMA staging (when the planes allow it): the phase window as one box of
 * columns c0-4 .. c0+71 (x 16-byte aligned) and rows r0-3 .. r0+67, and the
 * coherence window of columns c0 .. c0+67, rows r0 .. r0+64 */
constexpr int kC7WinW = 76, kC7WinH = 71;
constexpr int kC7CorW = 68, kC7CorH = 65;
struct C7Smem {
    union {
        float2 php[(kC7W + 1) * kC7PP];   /* phase pairs (load path), then the row sums */
        float win[kC7WinH * kC7WinW];     /* phase window (TMA path) */
    };
    float2 dpp[kC7W * kC7PP];             /* difference pairs */
    alignas(128) float cor[kC7CorH * kC7CorW];   /* coherence window (TMA path) */
    C7Deferred q[kC7Q];
    alignas(8) short lay[kC7Tab];
    unsigned long long bar;
    int qn;
    unsigned gbase;
};
static_assert(sizeof(float) * kC7WinH * kC7WinW <= sizeof(float2) * (kC7W + 1) * kC7PP,
              "phase window must fit the pair buffer");
static_assert(kC7WinW * 4 % 16 == 0 && kC7CorW * 4 % 16 == 0, "TMA boxes: 16-byte rows");

__device__ __forceinline__ unsigned c7_smem(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void c7_tma_2d(void *dst, const CUtensorMap *map, int x, int y,
                                          unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(c7_smem(dst)),
        "l"(map), "r"(x), "r"(y), "r"(c7_smem(bar))
        : "memory");
}
/* bounded wait for the block's TMA boxes (parity 0: one use per block); a
 * thread whose boxes have not landed may be suspended for up to 20 us per
 * test (the suspend-time hint), so waiting warps leave the issue slots to
 * the other blocks' computing warps */
__device__ __forceinline__ void c7_wait(unsigned long long *bar)
{
    for (int i = 0; i < (1 << 20); ++i) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0, %2;\n"
            " selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(c7_smem(bar)), "r"(20000u)
            : "memory");
        if (ok) return;
    }
}
/* launch-wide queue of deferred arcs, finished by k_costs7_drain */
struct C7Global {
    float ca, cb, dp, av;
    unsigned long long a;
    int w, pad;
};
constexpr unsigned kC7NoSlot = 0xffffffffu;

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
/* a - b per lane, one rounding */
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    return __ffma2_rn(b, f2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ float2 div_2pi2(float2 x)
{
    const float ax = fabsf(x.x), ay = fabsf(x.y);
    if (ax >= 0x1p-104f && ax <= 6.6f && ay >= 0x1p-104f && ay <= 6.6f) {
        const float2 z = f2(kRcpTwoPiRN, kRcpTwoPiRN);
        const float2 q0 = __fmul2_rn(x, z);
        const float2 r = __ffma2_rn(q0, f2(-kTwoPiF, -kTwoPiF), x);
        return __ffma2_rn(r, z, q0);
    }
    return f2(div_2pi(x.x), div_2pi(x.y));
}
__device__ __forceinline__ float2 div_72(float2 x)
{
    const float2 z = f2(kRcp7RN, kRcp7RN);
    const float2 q0 = __fmul2_rn(x, z);
    const float2 r = __ffma2_rn(q0, f2(-7.0f, -7.0f), x);
    return __ffma2_rn(r, z, q0);
}
/* wrap_cycles per lane: d - floorf(d + 0.5f) */
__device__ __forceinline__ float2 wrap2(float2 d)
{
    const float2 t = __fadd2_rn(d, f2(0.5f, 0.5f));
    return __ffma2_rn(f2(floorf(t.x), floorf(t.y)), f2(-1.0f, -1.0f), d);
}
/* (0 + v[o] + ... + v[o+6]) / 7 per lane */
__device__ __forceinline__ float2 boxcar7(const float2 *v)
{
    float2 s = __fadd2_rn(f2(0.0f, 0.0f), v[0]);
#pragma unroll
    for (int t = 1; t < 7; ++t) s = __fadd2_rn(s, v[t]);
    return div_72(s);
}

__device__ __forceinline__ float lg2_ftz(float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_ftz(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

/* coherence as the FP32 fast path reads it: values in [0, 1] unchanged,
 * non-finite values as 0 (sane), and every other value -- finite outside
 * [0, 1], or -0 -- as NaN.  A NaN fails the threshold test of arc_lane, so
 * the arc goes to the exact arithmetic, which reloads the stored value. */
__device__ __forceinline__ float cor_fast(float c)
{
    const unsigned u = __float_as_uint(c);
    if (u <= 0x3f800000u) return c;
    return (u & 0x7fffffffu) >= 0x7f800000u ? 0.0f : __uint_as_float(0x7fc00000u);
}

/* arc_lane / arc_fast2: FP32 evaluation of arc_cost for weight 1 and
 * coherences in [0, 1] (cor_fast).  Each rounded decision is taken only when
 * the FP32 value is farther from the decision boundary than the bound on its
 * distance to the reference's FP64 value, so the integers equal the
 * reference's; otherwise the lane reports false.
 *  rho:    rho_f = RN(ca + cb)/2 is within 2^-23 relative of the reference's
 *          (ca + cb)/2, so rho_f >= thresh (1 + 2^-20) and rho_f <=
 *          thresh (1 - 2^-20) decide rho < thresh.
 *  offset: X = RN(RN(dp - sel) nsc) is within nsc 2^-23 of the reference's
 *          FP64 value, and |X| <= nsc <= 4096.  DEFO rounds to nearest: the
 *          boundaries are the half-integers.  SMOOTH truncates: X - sign(X)/2
 *          (exact for |X| >= 1/4, and rounding to 0 below) moves the
 *          boundaries, the integers, to half-integers.  Either way XM =
 *          RN(X' + 1.5 2^23) holds the nearest integer of X' in its low bits,
 *          and |X' - (XM - 1.5 2^23)| <= 1/2 - m_off, m_off = nsc 2^-22 +
 *          2^-30, keeps X' away from the boundaries.
 *  sigsq:  b = ((1 - ca) + (1 - cb))/2 is within 2^-22 relative of the
 *          reference's 1 - rho and b <= 1; for b >= 2^-8 the MUFU log2/exp2
 *          estimate of b^rhopow and the FMA stay within 2e-6 rhopow + 5e-7
 *          relative, so v = a b^rhopow + c is bracketed by the screen m =
 *          (1e-5 (1 + rhopow) + 2e-6) v + 1e-6 with at least a 5x margin;
 *          w = v - 1/2 rounded to the nearest integer gives floor(v), and
 *          |w - round(w)| <= 1/2 - m keeps v that far from the integers.
 *          v >= 0 and v < 1e6 hold for every b in [0, 1] (host-checked).
 *  rho = 0 uses the exact host value of the reference's formula at b = 1.
 * arc_lane takes one lane's decisions from the values arc_fast2 computed. */
template <bool DEFO>
__device__ __forceinline__ bool arc_lane(bool pos, float rho, float XM, float f, float b, float vm,
                                         float g, float mh, const CostConsts &k, const short *lay,
                                         int ntab, ArcCost &o)
{
    bool ok = pos | (rho <= k.thr_lo);
    ok &= fabsf(f) <= k.off_hm;
    ok &= !pos | ((b >= 0x1p-8f) & (fabsf(g) <= mh));
    int sg = pos ? __float_as_int(vm) - 0x4B400000 : k.s_rho0;
    sg = max(sg, k.sigsqshortmin);
    if (DEFO) {
        /* the table holds every value of the fast path; the test only
         * guards lanes that fail anyway */
        ok &= (unsigned)sg < (unsigned)ntab;
        o.dzmax = (short)k.dzmax;
        o.laycost = lay[min((unsigned)sg, (unsigned)(ntab - 1))];
    } else {
        o.dzmax = 0;
        o.laycost = 0;
        sg = min(sg, (int)SHRT_MAX);
    }
    o.off = (short)(__float_as_int(XM) - 0x4B400000);
    o.sigsq = (short)sg;
    return ok;
}

/* the two columns of a pair: the arithmetic on both lanes at once (same
 * roundings as the scalar forms), the decisions per lane.  Every candidate
 * is computed and each margin test folds into one predicate (a NaN anywhere
 * fails its test). */
template <bool DEFO>
__device__ __forceinline__ void arc_fast2(float2 ca, float2 cb, float2 dp, float2 av,
                                          const CostConsts &k, const short *lay, int ntab,
                                          ArcCost &o0, ArcCost &o1, bool &ok0, bool &ok1)
{
    const float2 half = f2(0.5f, 0.5f), one = f2(1.0f, 1.0f);
    const float2 mg = f2(12582912.0f, 12582912.0f);
    const float2 rho = __fmul2_rn(half, __fadd2_rn(ca, cb));
    const bool pos0 = rho.x >= k.thr_hi, pos1 = rho.y >= k.thr_hi;
    const float2 hav = __fmul2_rn(half, av);
    const float2 sel = f2(pos0 ? av.x : hav.x, pos1 ? av.y : hav.y);
    float2 X = __fmul2_rn(sub2(dp, sel), f2(k.nsc_f, k.nsc_f));
    if (!DEFO) X = sub2(X, f2(copysignf(0.5f, X.x), copysignf(0.5f, X.y)));
    const float2 XM = __fadd2_rn(X, mg);
    const float2 f = sub2(X, sub2(XM, mg));
    const float2 b = __fmul2_rn(half, __fadd2_rn(sub2(one, ca), sub2(one, cb)));
    const float2 t = __fmul2_rn(f2(k.rhopow_f, k.rhopow_f), f2(lg2_ftz(b.x), lg2_ftz(b.y)));
    const float2 v = __ffma2_rn(f2(k.a_f, k.a_f), f2(ex2_ftz(t.x), ex2_ftz(t.y)), f2(k.c_f, k.c_f));
    const float2 w = sub2(v, half);
    const float2 vm = __fadd2_rn(w, mg);
    const float2 g = sub2(w, sub2(vm, mg));
    const float2 mh = __ffma2_rn(f2(-k.screen_f, -k.screen_f), v, f2(k.half_m, k.half_m));
    ok0 = arc_lane<DEFO>(pos0, rho.x, XM.x, f.x, b.x, vm.x, g.x, mh.x, k, lay, ntab, o0);
    ok1 = arc_lane<DEFO>(pos1, rho.y, XM.y, f.y, b.y, vm.y, g.y, mh.y, k, lay, ntab, o1);
}

template <bool DEFO>
__device__ __forceinline__ void store_arc(void *costs, size_t a, const ArcCost &o)
{
    if (DEFO)
        reinterpret_cast<short4 *>(costs)[a] = make_short4(o.off, o.sigsq, o.dzmax, o.laycost);
    else
        reinterpret_cast<short2 *>(costs)[a] = make_short2(o.off, o.sigsq);
}

template <bool DEFO, int FAM, int MINB, bool TMA>
__global__ void __launch_bounds__(256, MINB) k_costs7(const float *__restrict__ ph,
                                                   const float *__restrict__ corr,
                                                   const short *__restrict__ weights, int nrow,
                                                   int ncol, const CostConsts k,
                                                   void *__restrict__ costs_out, int nbx,
                                                   C7Global *__restrict__ gq, unsigned *gqn,
                                                   unsigned gqcap,
                                                   const short *__restrict__ laytab,
                                                   const __grid_constant__ CUtensorMap tm_ph,
                                                   const __grid_constant__ CUtensorMap tm_cor)
{
    /* TMA: the windows arrive as TMA boxes (else the threads load them) */
    constexpr bool tma = TMA;
    extern __shared__ __align__(16) char c7raw[];
    C7Smem &S = *reinterpret_cast<C7Smem *>(
        ((uintptr_t)c7raw + 127) & ~(uintptr_t)127);
    const int by = blockIdx.x / nbx, bx = blockIdx.x - (blockIdx.x / nbx) * nbx;
    const int dr = FAM == 0 ? nrow - 1 : nrow;
    const int dc = FAM == 0 ? ncol : ncol - 1;
    const int r0 = by * kC7B, c0 = bx * kC7B;
    const int tid = threadIdx.x;
    if (tid == 0) S.qn = 0;
    /* laycost of every sigsq the fast path can produce: the launch's table
     * (k_c7_laytab), four entries per thread, or computed here when the
     * launch has no scratch for it */
    const int ntab = DEFO ? min(max(k.s_rho0, k.sigsqshortmin) + 1, kC7Tab) : 0;
    if (DEFO) {
        if (laytab) {
            static_assert(kC7Tab == 4 * 256, "one short4 of the table per thread");
            reinterpret_cast<short4 *>(S.lay)[tid] = __ldg(reinterpret_cast<const short4 *>(laytab) + tid);
        } else {
            for (int v = tid; v < ntab; v += blockDim.x)
                S.lay[v] = (short)min(isqrt_floor(k.dzmax * v), (int)SHRT_MAX);
        }
    }

    constexpr int NR = kC7W + (FAM == 0 ? 1 : 0);             /* phase rows */
    constexpr int NP = kC7W - kC7H + (FAM == 1 ? 1 : 0);      /* phase pairs per row */
    constexpr int ND = kC7W - kC7H;                            /* difference pairs per row */
    const bool interior = r0 >= 3 && r0 + kC7B + 3 <= dr && c0 >= 3 && c0 + kC7B + 3 <= dc;
    if (tma) {
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(c7_smem(&S.bar))
                         : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            const unsigned tx = (unsigned)(kC7CorH * kC7CorW * 4) +
                                (interior ? (unsigned)(kC7WinH * kC7WinW * 4) : 0u);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                             c7_smem(&S.bar)),
                         "r"(tx)
                         : "memory");
            c7_tma_2d(S.cor, &tm_cor, c0, r0, &S.bar);
            if (interior) c7_tma_2d(S.win, &tm_ph, c0 - 4, r0 - 3, &S.bar);
        }
        __syncthreads();
        c7_wait(&S.bar);
    }
    if (interior && tma) {
        /* differences from the row-major window (column c0-3+j is win[.][j+1]):
         * thread (i0, j) takes rows i0, i0 + RS, ... of pair column j, so the
         * addresses advance by constants */
        constexpr int RS = 256 / ND;
        if (tid < RS * ND) {
            const int i0 = tid / ND, j = tid - i0 * ND;
            const float *w0 = S.win + i0 * kC7WinW + j + 1;
            float2 *dst = S.dpp + i0 * kC7PP + j;
            for (int i = i0; i < kC7W; i += RS, w0 += RS * kC7WinW, dst += RS * kC7PP) {
                const float2 x =
                    FAM == 0 ? sub2(f2(w0[0], w0[kC7H]), f2(w0[kC7WinW], w0[kC7WinW + kC7H]))
                             : sub2(f2(w0[1], w0[kC7H + 1]), f2(w0[0], w0[kC7H]));
                *dst = wrap2(div_2pi2(x));
            }
        }
    } else if (interior) {
        /* all of a thread's window loads in flight before the first store */
        const float *src = ph + (size_t)(r0 - 3) * ncol + (c0 - 3);
        constexpr int NU = (NR * NP + 255) / 256;
        float2 pv[NU];
#pragma unroll
        for (int t = 0; t < NU; ++t) {
            const int u = tid + t * 256;
            if (u < NR * NP) {
                const int i = u / NP, j = u - (u / NP) * NP;
                const float *row = src + (size_t)i * ncol;
                pv[t] = f2(__ldg(row + j), __ldg(row + j + kC7H));
            }
        }
#pragma unroll
        for (int t = 0; t < NU; ++t) {
            const int u = tid + t * 256;
            if (u < NR * NP) {
                const int i = u / NP, j = u - (u / NP) * NP;
                S.php[i * kC7PP + j] = pv[t];
            }
        }
        __syncthreads();
        for (int u = tid; u < kC7W * ND; u += blockDim.x) {
            const int i = u / ND, j = u - (u / ND) * ND;
            const float2 x = FAM == 0 ? sub2(S.php[i * kC7PP + j], S.php[(i + 1) * kC7PP + j])
                                      : sub2(S.php[i * kC7PP + j + 1], S.php[i * kC7PP + j]);
            S.dpp[i * kC7PP + j] = wrap2(div_2pi2(x));
        }
    } else {
        /* window crosses the array edge: mirror-reflected differences */
        for (int u = tid; u < kC7W * ND; u += blockDim.x) {
            const int i = u / ND, j = u - (u / ND) * ND;
            const int sr = reflect_index(r0 + i - 3, dr);
            float v[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int sc = reflect_index(c0 + j + h * kC7H - 3, dc);
                const float *p = ph + (size_t)sr * ncol + sc;
                v[h] = wrap_cycles(FAM == 0 ? div_2pi(__fsub_rn(p[0], p[ncol]))
                                            : div_2pi(__fsub_rn(p[1], p[0])));
            }
            S.dpp[i * kC7PP + j] = f2(v[0], v[1]);
        }
    }
    __syncthreads();
    /* row pass: row sums of the pairs, two pairs per thread; the sums
     * overwrite the phase pairs ([kC7W][kC7H] pairs, pitch kC7H) */
    float2 *tp = S.php;
    for (int u = tid; u < kC7W * (kC7H / 2); u += blockDim.x) {
        const int i = u >> 4, m = (u & 15) * 2;
        const float4 *d4 = reinterpret_cast<const float4 *>(S.dpp + i * kC7PP + m);
        float2 v[8];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float4 q = d4[t];
            v[2 * t] = f2(q.x, q.y);
            v[2 * t + 1] = f2(q.z, q.w);
        }
        const float2 o0 = boxcar7(v), o1 = boxcar7(v + 1);
        *reinterpret_cast<float4 *>(tp + i * kC7H + m) = make_float4(o0.x, o0.y, o1.x, o1.y);
    }
    __syncthreads();
    /* column pass and arc costs: thread = column pair j, an 8-row strip
     * walked in two halves of 4 rows */
    const int j = tid & 31, rs0 = (tid >> 5) * 8;
    const size_t nra = (size_t)(nrow - 1) * ncol;
    const bool fast = k.fast != 0;
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
    const int rs = rs0 + half * 4;
    if (r0 + rs >= dr) break;
    /* a rolling window of the row sums and of the coherence: each row of
     * the strip loads one new row sum and its coherence (fewer live
     * registers than loading the whole strip up front) */
    auto cor_at = [&](int q, int h, int dcol) -> float {
        const int ac = c0 + j + h * kC7H, rr = r0 + rs + q;
        float v = 0.0f;
        if (tma) {
            /* staged window: row rs+q, column j+32h (+1); zero outside the array */
            v = S.cor[(rs + q) * kC7CorW + j + h * kC7H + dcol];
        } else if (ac < dc && rr < nrow) {
            v = __ldg(corr + (size_t)rr * ncol + ac + dcol);
        }
        return cor_fast(v);
    };
    float2 w[7];
#pragma unroll
    for (int q = 0; q < 6; ++q) w[q] = tp[(rs + q) * kC7H + j];
    float2 cnext = FAM == 0 ? f2(cor_at(0, 0, 0), cor_at(0, 1, 0)) : f2(0.0f, 0.0f);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int ar = r0 + rs + m;
        if (ar >= dr) break;
        w[6] = tp[(rs + m + 6) * kC7H + j];
        const float2 avg = boxcar7(w);
#pragma unroll
        for (int q = 0; q < 6; ++q) w[q] = w[q + 1];
        const float2 dps = S.dpp[(rs + m + 3) * kC7PP + j + 3];
        float2 ca2, cb2;
        if (FAM == 0) {
            ca2 = cnext;
            cb2 = f2(cor_at(m + 1, 0, 0), cor_at(m + 1, 1, 0));
            cnext = cb2;
        } else {
            ca2 = f2(cor_at(m, 0, 0), cor_at(m, 1, 0));
            cb2 = f2(cor_at(m, 0, 1), cor_at(m, 1, 1));
        }
        ArcCost of[2];
        bool okf[2] = {false, false};
        if (fast) arc_fast2<DEFO>(ca2, cb2, dps, avg, k, S.lay, ntab, of[0], of[1], okf[0], okf[1]);
        /* arc index of the strip's column pair in this row (column j, j + 32) */
        const size_t a0 = (FAM == 0 ? (size_t)ar * ncol : nra + (size_t)ar * (ncol - 1)) +
                          (size_t)(c0 + j);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int ac = c0 + j + h * kC7H;
            if (ac >= dc) continue;
            const float dpv = h ? dps.y : dps.x, avv = h ? avg.y : avg.x;
            const size_t a = a0 + (size_t)(h * kC7H);
            /* an arc the fast path could not decide: queued for the exact
             * arithmetic with the stored coherence (cor_fast changed values
             * it rejects) */
            auto defer = [&](short wt) {
                const float *cp = corr + (size_t)ar * ncol + ac;
                const float ca = sane(__ldg(cp)), cb = sane(__ldg(cp + (FAM == 0 ? ncol : 1)));
                const int slot = atomicAdd(&S.qn, 1);
                if (slot < kC7Q) {
                    S.q[slot] = C7Deferred{ca, cb, dpv, avv, (ar - r0) * kC7B + (ac - c0), (int)wt};
                } else {
                    store_arc<DEFO>(costs_out, a,
                                    arc_cost<DEFO>((double)ca, (double)cb, dpv, avv, wt, k));
                }
            };
            if (!weights) {
                /* every weight 1 */
                if (okf[h]) store_arc<DEFO>(costs_out, a, of[h]);
                else defer((short)1);
            } else {
                const short wt = weights[a];
                if (wt == 0) {
                    ArcCost o;
                    o.off = kLargeShort / 2; o.sigsq = kLargeShort;
                    o.dzmax = kLargeShort; o.laycost = 0;
                    store_arc<DEFO>(costs_out, a, o);
                } else if (wt == 1 && okf[h]) {
                    store_arc<DEFO>(costs_out, a, of[h]);
                } else {
                    defer(wt);
                }
            }
        }
    }
    }
    __syncthreads();
    /* deferred arcs: handed to the launch-wide queue (finished by
     * k_costs7_drain with full warps) when it has room, else the
     * reference's FP64 arithmetic here */
    const int nq = min(S.qn, kC7Q);
    if (tid == 0) S.gbase = (gq && nq > 0) ? atomicAdd(gqn, (unsigned)nq) : kC7NoSlot;
    __syncthreads();
    /* slots below the capacity are the queue's; a block that reaches past
     * it finishes the rest itself, so the first min(count, capacity) slots
     * are always valid */
    const unsigned gb = S.gbase;
    for (int i = tid; i < nq; i += blockDim.x) {
        const C7Deferred e = S.q[i];
        const int ar = r0 + e.rc / kC7B, ac = c0 + e.rc % kC7B;
        const size_t a = FAM == 0 ? (size_t)ar * ncol + ac : nra + (size_t)ar * (ncol - 1) + ac;
        if (gb != kC7NoSlot && gb < gqcap && (unsigned)i < gqcap - gb)
            gq[gb + i] = C7Global{e.ca, e.cb, e.dp, e.av, (unsigned long long)a, e.w, 0};
        else
            store_arc<DEFO>(costs_out, a,
                            arc_cost<DEFO>((double)e.ca, (double)e.cb, e.dp, e.av, (short)e.w, k));
    }
}

/* the laycost table of a launch: entry v = (int)sqrt(dzmax v) of the
 * reference (cuphu_cost.cu:225-265), clamped to SHRT_MAX, for every sigsq
 * the fast path can produce (entries past that are zero and never read) */
__global__ void __launch_bounds__(256) k_c7_laytab(short *__restrict__ tab, const CostConsts k)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= kC7Tab) return;
    const int ntab = min(max(k.s_rho0, k.sigsqshortmin) + 1, kC7Tab);
    tab[v] = v < ntab ? (short)min(isqrt_floor(k.dzmax * v), (int)SHRT_MAX) : (short)0;
}

template <bool DEFO>
__global__ void __launch_bounds__(256) k_costs7_drain(const C7Global *__restrict__ gq,
                                                      const unsigned *__restrict__ gqn,
                                                      unsigned gqcap, const CostConsts k,
                                                      void *__restrict__ costs_out)
{
    const unsigned n = min(*gqn, gqcap);
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const C7Global e = gq[i];
        store_arc<DEFO>(costs_out, (size_t)e.a,
                        arc_cost<DEFO>((double)e.ca, (double)e.cb, e.dp, e.av, (short)e.w, k));
    }
}

static PFN_cuTensorMapEncodeTiled_v12000 c7_encoder()
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

/* TMA map of an nrow x ncol float plane with the given box; false when the
 * plane's base or row pitch is not 16-byte aligned (the load path is used) */
static bool c7_map(CUtensorMap &m, const float *base, int nrow, int ncol, int bx, int by)
{
    if (((uintptr_t)base & 15) || (ncol & 3)) return false;
    auto enc = c7_encoder();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)ncol, (cuuint64_t)nrow};
    cuuint64_t strides[1] = {(cuuint64_t)ncol * 4};
    cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
    cuuint32_t es[2] = {1, 1};
    return enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides,
               box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool DEFO, int FAM, int MINB>
static int launch_costs7_v(const float *ph, const float *corr, const short *weights, int nrow,
                           int ncol, const CostConsts &k, void *costs, C7Global *gq,
                           unsigned *gqn, unsigned gqcap, const short *laytab, cudaStream_t s)
{
    const int dr = FAM == 0 ? nrow - 1 : nrow, dc = FAM == 0 ? ncol : ncol - 1;
    if (dr < 1 || dc < 1) return 0;
    const int nby = (dr + kC7B - 1) / kC7B, nbx = (dc + kC7B - 1) / kC7B;
    const size_t shm = sizeof(C7Smem) + 128;
    CUtensorMap tm_ph, tm_cor;
    std::memset(&tm_ph, 0, sizeof(tm_ph));
    std::memset(&tm_cor, 0, sizeof(tm_cor));
    const int tma = (c7_map(tm_ph, ph, nrow, ncol, kC7WinW, kC7WinH) &&
                     c7_map(tm_cor, corr, nrow, ncol, kC7CorW, kC7CorH)) ? 1 : 0;
    auto kern = tma ? k_costs7<DEFO, FAM, MINB, true> : k_costs7<DEFO, FAM, MINB, false>;
    CUPHU_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)shm));
    kern<<<nby * nbx, 256, shm, s>>>(ph, corr, weights, nrow, ncol, k, costs, nbx, gq, gqn, gqcap,
                                     laytab, tm_ph, tm_cor);
    return cuda_fail(cudaGetLastError(), "k_costs7");
}

/* occupancy variant from the autotuner (default: 3 blocks per SM) */
template <bool DEFO, int FAM>
static int launch_costs7_t(const float *ph, const float *corr, const short *weights, int nrow,
                           int ncol, const CostConsts &k, void *costs, C7Global *gq,
                           unsigned *gqn, unsigned gqcap, const short *laytab, cudaStream_t s)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const long long arcs = 2LL * nrow * ncol;
    if (tune_get(dev, 0, arcs) == 1)
        return launch_costs7_v<DEFO, FAM, 4>(ph, corr, weights, nrow, ncol, k, costs, gq, gqn,
                                             gqcap, laytab, s);
    return launch_costs7_v<DEFO, FAM, 3>(ph, corr, weights, nrow, ncol, k, costs, gq, gqn, gqcap,
                                         laytab, s);
}

/* both arc families, then the queued arcs; the queue (about one arc in 128
 * of room) is stream-ordered scratch, and blocks that find it full finish
 * their deferred arcs themselves */
template <bool DEFO>
static int launch_costs7_all(const float *ph, const float *corr, const short *weights, int nrow,
                             int ncol, const CostConsts &k, void *costs, cudaStream_t s)
{
    const unsigned long long narcs =
        (unsigned long long)(nrow - 1) * ncol + (unsigned long long)nrow * (ncol - 1);
    const unsigned cap = (unsigned)std::min<unsigned long long>(narcs / 128 + 4096, 1u << 24);
    /* scratch: the queue counter, the laycost table (DEFO), the queue */
    constexpr size_t kTabOff = 256, kQueueOff = kTabOff + kC7Tab * sizeof(short);
    static_assert(kQueueOff % 256 == 0, "queue offset");
    void *buf = nullptr;
    C7Global *gq = nullptr;
    unsigned *gqn = nullptr;
    short *laytab = nullptr;
    if (cudaMallocAsync(&buf, (size_t)cap * sizeof(C7Global) + kQueueOff, s) == cudaSuccess) {
        gqn = reinterpret_cast<unsigned *>(buf);
        gq = reinterpret_cast<C7Global *>(static_cast<char *>(buf) + kQueueOff);
        CUPHU_TRY_CUDA(cudaMemsetAsync(gqn, 0, sizeof(unsigned), s));
        if (DEFO) {
            laytab = reinterpret_cast<short *>(static_cast<char *>(buf) + kTabOff);
            k_c7_laytab<<<kC7Tab / 256, 256, 0, s>>>(laytab, k);
            CUPHU_TRY_CUDA(cudaGetLastError());
        }
    } else {
        cudaGetLastError();
    }
    int rc = launch_costs7_t<DEFO, 0>(ph, corr, weights, nrow, ncol, k, costs, gq, gqn, cap, laytab,
                                      s);
    if (!rc)
        rc = launch_costs7_t<DEFO, 1>(ph, corr, weights, nrow, ncol, k, costs, gq, gqn, cap,
                                      laytab, s);
    if (!rc && gq) {
        k_costs7_drain<DEFO><<<148 * 4, 256, 0, s>>>(gq, gqn, cap, k, costs);
        rc = cuda_fail(cudaGetLastError(), "k_costs7_drain");
    }
    if (buf) cudaFreeAsync(buf, s);
    return rc;
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
    if (w7) {
        int rc = mode == CUPHU_COST_SMOOTH
                     ? launch_costs7_all<false>(ph, corr, weights, nrow, ncol, k, costs, s)
                     : launch_costs7_all<true>(ph, corr, weights, nrow, ncol, k, costs, s);
        if (!rc && res) rc = launch_residues(ph, nrow, ncol, res, s);
        return rc;
    }
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
