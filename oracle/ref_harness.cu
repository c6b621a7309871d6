/*
 * ref_harness.cu -- host-pointer wrappers around the reference cuPHU kernel
 * launchers, compiled together with the reference's own hot-path sources
 * (cuphu_util.cu, cuphu_cost.cu, cuphu_laplace.cu, cuphu_phase.cu,
 * cuphu_conncomp.cu, cuphu_incrcost.cu) into oracle/_ref/libcuphu_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY: the reference kernels are the GPU-side parity
 * oracle ("the existing cuPHU kernels") and the GPU timing bar.  The product
 * library never links this.  Every wrapper returns 0 on success and -1 if
 * the reference code threw (its CUDA_CHECK throws std::runtime_error).
 */
#include "cuphu.h"
extern "C" {
#include "snaphu.h"
}
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

extern "C" void cuphu_wrap_phase(float *, int, cudaStream_t);
extern "C" void cuphu_build_smooth_costs_gpu(const float *, const float *, const short *,
                                             const short *, int, int, const CuPhuParams *,
                                             int, int, smoothcostT **, cudaStream_t);
extern "C" void cuphu_build_defo_costs_gpu(const float *, const float *, const short *,
                                           const short *, int, int, const CuPhuParams *,
                                           int, int, costT **, cudaStream_t);
extern "C" void cuphu_laplace_unwrap_gpu(const smoothcostT *, const float *, int, int, double,
                                         int, float, int, float *, cudaStream_t);
extern "C" bool cuphu_incrcost_early_exit(const smoothcostT *, const short *, int, long, int,
                                          short *, short *, int *);

static CuPhuParams make(double ncorrlooks, double defothreshfactor, double rhosconst1,
                        double rhosconst2, double cstd1, double cstd2, double cstd3,
                        double sigsqcorr, double costscale, double nshortcycle,
                        long sigsqshortmin, double defomax, double minfrac,
                        long maxncomps, long cthr)
{
    CuPhuParams p;
    std::memset(&p, 0, sizeof(p));
    p.nlooks = p.ncorrlooks = ncorrlooks;
    p.defothreshfactor = defothreshfactor;
    p.rhosconst1 = rhosconst1;
    p.rhosconst2 = rhosconst2;
    p.cstd1 = cstd1; p.cstd2 = cstd2; p.cstd3 = cstd3;
    p.sigsqcorr = sigsqcorr;
    p.costscale = costscale;
    p.nshortcycle = nshortcycle;
    p.sigsqshortmin = sigsqshortmin;
    p.defomax = defomax;
    p.minconncompfrac = minfrac;
    p.maxncomps = maxncomps;
    p.conncompthresh = cthr;
    return p;
}

template <typename T>
static T *dev_copy(const T *h, size_t n)
{
    T *d = nullptr;
    if (cudaMalloc(&d, (n ? n : 1) * sizeof(T)) != cudaSuccess) throw std::exception();
    if (h && n) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

extern "C" {

/* costs: mode 0 smooth (4 B/arc), else defo (8 B/arc); out holds the flat
 * row-arcs-then-col-arcs array.  weights may be NULL (flat layout). */
int ref_build_costs(const float *phase, const float *corr, const short *weights, int nrow,
                    int ncol, int mode, const double *pd, const long *pl, int kperp,
                    int kpar, void *out, float *ms_out, int reps)
{
    try {
        size_t npix = (size_t)nrow * ncol;
        size_t nra = (size_t)(nrow - 1) * ncol, nca = (size_t)nrow * (ncol - 1);
        CuPhuParams p = make(pd[0], pd[1], pd[2], pd[3], pd[4], pd[5], pd[6], pd[7], pd[8],
                             pd[9], pl[0], pd[10], 0.01, 32, 300);
        float *dph = dev_copy(phase, npix), *dco = dev_copy(corr, npix);
        short *dw = weights ? dev_copy(weights, nra + nca) : nullptr;
        cuphu_wrap_phase(dph, (int)npix, 0);
        size_t es = mode ? sizeof(costT) : sizeof(smoothcostT);
        void *dc = nullptr;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0); cudaEventCreate(&e1);
        if (reps < 1) reps = 1;
        float best = 1e30f;
        for (int rep = 0; rep < reps; ++rep) {
            if (dc) cudaFree(dc);
            dc = nullptr;
            cudaDeviceSynchronize();
            cudaEventRecord(e0, 0);
            if (mode == 0) {
                smoothcostT *c = nullptr;
                cuphu_build_smooth_costs_gpu(dph, dco, dw, dw ? dw + nra : nullptr, nrow, ncol,
                                             &p, kperp, kpar, &c, 0);
                dc = c;
            } else {
                costT *c = nullptr;
                cuphu_build_defo_costs_gpu(dph, dco, dw, dw ? dw + nra : nullptr, nrow, ncol,
                                           &p, kperp, kpar, &c, 0);
                dc = c;
            }
            cudaEventRecord(e1, 0);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) best = ms;
        }
        if (ms_out) *ms_out = best;
        cudaMemcpy(out, dc, (nra + nca) * es, cudaMemcpyDeviceToHost);
        cudaFree(dc); cudaFree(dph); cudaFree(dco);
        if (dw) cudaFree(dw);
        cudaEventDestroy(e0); cudaEventDestroy(e1);
        return cudaGetLastError() == cudaSuccess ? 0 : -1;
    } catch (...) {
        return -1;
    }
}

/* the reference FP32 Laplace solve on smooth costs (4 B/arc), u out (host) */
int ref_laplace(const void *costs, const float *phase, int nrow, int ncol, int max_iter,
                float tol, float *unw, float *ms_out)
{
    try {
        size_t npix = (size_t)nrow * ncol;
        size_t narcs = (size_t)(nrow - 1) * ncol + (size_t)nrow * (ncol - 1);
        smoothcostT *dc = dev_copy((const smoothcostT *)costs, narcs);
        float *dph = dev_copy(phase, npix);
        float *du = dev_copy<float>(nullptr, npix);
        cudaStream_t s;
        cudaStreamCreate(&s);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0); cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
        cuphu_laplace_unwrap_gpu(dc, dph, nrow, ncol, 200.0, max_iter, tol, 0, du, s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms_out) *ms_out = ms;
        cudaMemcpy(unw, du, npix * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(dc); cudaFree(dph); cudaFree(du);
        cudaEventDestroy(e0); cudaEventDestroy(e1);
        cudaStreamDestroy(s);
        return cudaGetLastError() == cudaSuccess ? 0 : -1;
    } catch (...) {
        return -1;
    }
}

int ref_conncomp(const float *unw, const float *corr, const unsigned char *mask, int nrow,
                 int ncol, const short *pos, const short *neg, double minfrac,
                 long maxncomps, long cthr, unsigned *labels)
{
    try {
        size_t npix = (size_t)nrow * ncol;
        size_t narcs = (size_t)(nrow - 1) * ncol + (size_t)nrow * (ncol - 1);
        CuPhuParams p = make(1, 1.25, 1.3, 0.14, 0.4, 0.35, 0.06, 0.05, 100, 200, 1, 1.2,
                             minfrac, maxncomps, cthr);
        float *du = dev_copy(unw, npix), *dco = dev_copy(corr, npix);
        unsigned char *dm = mask ? dev_copy(mask, npix) : nullptr;
        short *dp = pos ? dev_copy(pos, narcs) : nullptr;
        short *dn = neg ? dev_copy(neg, narcs) : nullptr;
        uint32_t *dl = dev_copy<uint32_t>(nullptr, npix);
        cuphu_conncomp_gpu(du, dco, dm, nrow, ncol, dp, dn, &p, 0, dl);
        cudaMemcpy(labels, dl, npix * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        cudaFree(du); cudaFree(dco); cudaFree(dl);
        if (dm) cudaFree(dm);
        if (dp) cudaFree(dp);
        if (dn) cudaFree(dn);
        return cudaGetLastError() == cudaSuccess ? 0 : -1;
    } catch (...) {
        return -1;
    }
}

int ref_integrate(const float *phase, const short *hflows, const short *vflows, int nrow,
                  int ncol, float *unw)
{
    try {
        size_t npix = (size_t)nrow * ncol;
        float *dph = dev_copy(phase, npix);
        short *dh = dev_copy(hflows, (size_t)(nrow - 1) * ncol);
        short *dv = dev_copy(vflows, (size_t)nrow * (ncol - 1));
        float *du = dev_copy<float>(nullptr, npix);
        cuphu_integrate_phase_gpu(dph, dh, dv, nrow, ncol, 0, du);
        cudaMemcpy(unw, du, npix * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(dph); cudaFree(dh); cudaFree(dv); cudaFree(du);
        return cudaGetLastError() == cudaSuccess ? 0 : -1;
    } catch (...) {
        return -1;
    }
}

int ref_incrcost(const void *costs, const short *flows, int narcs, long nsc, int nflow,
                 short *pos, short *neg)
{
    try {
        smoothcostT *dc = dev_copy((const smoothcostT *)costs, (size_t)narcs);
        short *df = dev_copy(flows, (size_t)narcs);
        short *dp = dev_copy<short>(nullptr, (size_t)narcs);
        short *dn = dev_copy<short>(nullptr, (size_t)narcs);
        int *ds = dev_copy<int>(nullptr, 2);
        bool ex = cuphu_incrcost_early_exit(dc, df, narcs, nsc, nflow, dp, dn, ds);
        cudaMemcpy(pos, dp, narcs * sizeof(short), cudaMemcpyDeviceToHost);
        cudaMemcpy(neg, dn, narcs * sizeof(short), cudaMemcpyDeviceToHost);
        cudaFree(dc); cudaFree(df); cudaFree(dp); cudaFree(dn); cudaFree(ds);
        return ex ? 1 : 0;
    } catch (...) {
        return -1;
    }
}

} /* extern "C" */
