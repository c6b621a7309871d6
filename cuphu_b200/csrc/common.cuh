/*
 * common.cuh -- shared constants, numeric helpers and error plumbing for the
 * sm_100a kernels of the cuPHU unwrapping path.
 *
 * Numeric helpers restate the reference's float conventions exactly; where
 * nvcc contracts a multiply-add in the reference kernel the fused form is
 * written out explicitly here, so the result does not depend on compiler
 * contraction decisions.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/cuphu_b200.h"

namespace cuphu {

/* 2*CUDART_PI_F (cuphu_util.cu:23, cuphu_phase.cu:24) == LAPLACE_TWOPI
 * (cuphu_laplace.cu:59) as float: 0x40C90FDB */
constexpr float kTwoPiF = 6.28318548202514648f;
constexpr float kInvTwoPiF = 0.15915494309189534561f;  /* cuphu_laplace.cu:60 */
constexpr float kPiF = 3.14159274101257324f;           /* (float)CUDART_PI_F   */
constexpr float kLapEpsF = 1e-12f;                      /* cuphu_laplace.cu:61 */
constexpr int kLargeShort = 32000;                      /* LARGESHORT          */
constexpr double kTwoPiD = 6.283185307179586;           /* 2.0*M_PI            */

/* canonical solver work item: kItemTx threads x kItemVx pixels per row,
 * kItemBy rows; the FP64 oracle reduces in exactly this geometry */
constexpr int kItemTx = 16;
constexpr int kItemVx = 4;
constexpr int kItemBy = 16;
constexpr int kItemBx = kItemTx * kItemVx;
constexpr int kItemThreads = kItemTx * kItemBy;

/* cuphu_util.cu:27-30 */
__device__ __forceinline__ float wrap_cycles(float d) { return d - floorf(d + 0.5f); }

/* device re-wrap to [0,2pi): cuphu_util.cu:33-36 */
__device__ __forceinline__ float rewrap_2pi(float p)
{
    return __fmaf_rn(-kTwoPiF, floorf(__fdiv_rn(p, kTwoPiF)), p);
}

/* cuphu_laplace.cu:71-73 */
__device__ __forceinline__ float lap_wrap_pi(float x)
{
    return __fmaf_rn(-kTwoPiF, rintf(__fmul_rn(x, kInvTwoPiF)), x);
}

/* cuphu_phase.cu:27-29 */
__device__ __forceinline__ float wrap_angle(float x)
{
    return __fmaf_rn(-kTwoPiF, rintf(__fdiv_rn(x, kTwoPiF)), x);
}

/* mirror index with repeated reflection (equals cuphu_util.cu:172-177
 * whenever the half window is smaller than the extent) */
__device__ __forceinline__ int reflect_index(int i, int n)
{
    if (n <= 1) return 0;
    int period = 2 * (n - 1);
    int j = i % period;
    if (j < 0) j += period;
    if (j > n - 1) j = period - j;
    return j;
}

/* non-finite coherence reads as 0, as cuphu.unwrap sanitises it (_unwrap.py:521-522) */
__device__ __forceinline__ float sane(float v) { return isfinite(v) ? v : 0.0f; }

/* ── statistical-cost constants, host-computed like upload_smooth_constants
 *    (cuphu_cost.cu:41-59) and passed by value ───────────────────────────── */
struct CostConsts {
    double rho0, thresh, rhopow, sigsqrhoconst, sigsqcorr, nsc, nsc2, costscale, defomax;
    int sigsqshortmin;
    float rhopow_f;   /* screening exponent of the FP32 pow estimate */
    double screen;    /* relative half-width of the screening interval */
    float screen_f, sig_f, corr_f, scale_f;   /* FP32 screening constants */
    int dzmax;        /* DEFO discontinuity shelf in short-cycle steps */
    /* FP32 fast path of the default-window cost kernel (k_costs7); fast = 0
     * when its error bounds do not hold for these parameters */
    int fast;
    float nsc_f;          /* nshortcycle (exact in float) */
    float thr_lo, thr_hi; /* coherence threshold bracket, 2^-20 relative */
    float a_f, c_f;       /* v = a_f b^rhopow + c_f (weight 1) */
    float off_hm;         /* 1/2 - offset rounding margin (rounded down) */
    float half_m;         /* 1/2 - 1e-6 (rounded down): sigsq margin base */
    int s_rho0;           /* truncated sigsq of a zero-coherence arc, weight 1 */
};

CostConsts make_cost_consts(const CuPhuParams &p);

/* ── error plumbing ─────────────────────────────────────────────────────── */
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define CUPHU_TRY_CUDA(expr)                                             \
    do {                                                                 \
        cudaError_t _e = (expr);                                         \
        if (_e != cudaSuccess) return ::cuphu::cuda_fail(_e, #expr);     \
    } while (0)

}  // namespace cuphu
