/*
 * host_phase.cu -- the wrapped phase of a host interferogram computed as the
 * reference computes it, and uploaded to the GPU.
 *
 * The reference derives the phase on the host (cuphu_solver.cpp:1706-1712,
 * and the same loop in cuphu_build_costs_gpu, :2120-2126): the C library's
 * float atan2(im, re), plus 2 pi when negative, then re-wraps it on the
 * device as p - 2 pi floor(p / 2 pi) (cuphu_util.cu:32-46, a fused
 * multiply-add after nvcc contraction).  The C library's float atan2 is not
 * correctly rounded -- it differs from the correctly rounded angle in the
 * last bit for about one sample in six -- so no device atan2 reproduces it.
 * The host-buffer entry points therefore take the phase the same way here,
 * which makes every downstream result (costs, residues, cycle maps, labels)
 * identical to the reference's on the same interferogram.
 *
 * Mechanism: a pool of host threads computes the phase chunk by chunk into
 * a pinned staging buffer (one per device, grow-only); the calling thread
 * enqueues each chunk's upload as soon as the chunk is complete, so the
 * upload of chunk k overlaps the computation of the later chunks.  Only
 * 4 bytes per pixel cross PCIe instead of the interferogram's 8.
 */
#include "kernels.cuh"

#include <atomic>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace cuphu {

namespace {

struct PhaseStaging {
    std::mutex mu;
    float *buf = nullptr;    /* pinned */
    size_t cap = 0;          /* floats */
    cudaEvent_t done = nullptr;
};

PhaseStaging g_stage[64];

constexpr size_t kChunk = (size_t)1 << 20;   /* pixels per upload */

/* one sample: non-finite samples read as 0 (cuphu.unwrap replaces them,
 * _unwrap.py:515-520); host float atan2, shift, device re-wrap */
inline float ref_phase(float re, float im)
{
    if (!(std::isfinite(re) && std::isfinite(im))) {
        re = 0.0f;
        im = 0.0f;
    }
    float phi = std::atan2(im, re);
    if (phi < 0.0f) phi += 6.28318530717958648f;
    return std::fmaf(-kTwoPiF, std::floor(phi / kTwoPiF), phi);
}

void phase_range(const float *c64, const float *re, const float *im, float *out, size_t a,
                 size_t b)
{
    if (c64) {
        for (size_t k = a; k < b; ++k) out[k] = ref_phase(c64[2 * k], c64[2 * k + 1]);
    } else {
        for (size_t k = a; k < b; ++k) out[k] = ref_phase(re[k], im[k]);
    }
}

int host_threads()
{
    if (const char *e = std::getenv("CUPHU_HOST_THREADS")) {
        int v = std::atoi(e);
        if (v >= 1) return std::min(v, 256);
    }
    unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hc, 64u));
}

}  // namespace

void compute_host_phase(const float *c64, const float *re, const float *im, size_t n, float *out)
{
    const size_t nch = (n + kChunk - 1) / kChunk;
    const int nth = (int)std::min<size_t>((size_t)host_threads(), nch);
    if (nth <= 1) {
        phase_range(c64, re, im, out, 0, n);
        return;
    }
    std::atomic<size_t> next(0);
    std::vector<std::thread> pool;
    pool.reserve(nth);
    for (int t = 0; t < nth; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                size_t c = next.fetch_add(1, std::memory_order_relaxed);
                if (c >= nch) return;
                phase_range(c64, re, im, out, c * kChunk, std::min(n, (c + 1) * kChunk));
            }
        });
    for (auto &th : pool) th.join();
}

int upload_host_phase(const float *c64, const float *re, const float *im, size_t n, float *d_ph,
                      int dev, cudaStream_t s)
{
    if (n == 0) return 0;
    if (dev < 0 || dev >= 64) return fail(CUPHU_ERR_INVALID, "device index out of range");
    PhaseStaging &P = g_stage[dev];
    std::lock_guard<std::mutex> lk(P.mu);
    if (!P.done) {
        cudaEvent_t ev = nullptr;
        CUPHU_TRY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        P.done = ev;
    } else {
        /* the previous call's uploads read the staging buffer */
        CUPHU_TRY_CUDA(cudaEventSynchronize(P.done));
    }
    if (n > P.cap) {
        if (P.buf) cudaFreeHost(P.buf);
        P.buf = nullptr;
        P.cap = 0;
        float *b = nullptr;
        if (cudaHostAlloc((void **)&b, n * sizeof(float), cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return fail(CUPHU_ERR_ALLOC, "pinned phase staging allocation failed");
        }
        P.buf = b;
        P.cap = n;
    }
    const size_t nch = (n + kChunk - 1) / kChunk;
    const int nth = (int)std::min<size_t>((size_t)host_threads(), nch);
    int rc = 0;
    if (nth <= 1) {
        phase_range(c64, re, im, P.buf, 0, n);
        rc = cuda_fail(cudaMemcpyAsync(d_ph, P.buf, n * sizeof(float), cudaMemcpyHostToDevice, s),
                       "H2D phase");
    } else {
        std::unique_ptr<std::atomic<int>[]> ready(new std::atomic<int>[nch]);
        for (size_t c = 0; c < nch; ++c) ready[c].store(0, std::memory_order_relaxed);
        std::atomic<size_t> next(0);
        std::vector<std::thread> pool;
        pool.reserve(nth);
        for (int t = 0; t < nth; ++t)
            pool.emplace_back([&]() {
                for (;;) {
                    size_t c = next.fetch_add(1, std::memory_order_relaxed);
                    if (c >= nch) return;
                    size_t a = c * kChunk, b = std::min(n, a + kChunk);
                    phase_range(c64, re, im, P.buf, a, b);
                    ready[c].store(1, std::memory_order_release);
                }
            });
        for (size_t c = 0; c < nch; ++c) {
            while (!ready[c].load(std::memory_order_acquire)) std::this_thread::yield();
            if (rc) continue;
            size_t a = c * kChunk, len = std::min(n, a + kChunk) - a;
            rc = cuda_fail(cudaMemcpyAsync(d_ph + a, P.buf + a, len * sizeof(float),
                                           cudaMemcpyHostToDevice, s),
                           "H2D phase");
        }
        for (auto &th : pool) th.join();
    }
    cudaError_t e = cudaEventRecord(P.done, s);
    if (!rc) rc = cuda_fail(e, "phase upload event");
    return rc;
}

}  // namespace cuphu
