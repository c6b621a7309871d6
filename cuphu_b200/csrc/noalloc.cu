/*
 * noalloc.cu -- phase integration for callers that cannot allocate device
 * memory.
 *
 * cuphu_integrate_phase_gpu takes its per-row scratch (one float of column-0
 * cumulative phase per row) from cudaMallocAsync.  Some callers cannot make
 * that call: a host framework whose caching allocator already holds the
 * device's free memory (a second allocator would fail or fragment it), a
 * real-time processor that forbids allocation once it is running, or a
 * plugin host that owns every device allocation itself.  For them
 * cuphu_integrate_phase_noalloc runs the same two kernels with the scratch
 * taken from a fixed array compiled into this library, so the call allocates
 * nothing: no cudaMalloc, cudaMallocAsync, cudaFree, or allocating library
 * routine.
 *
 * The array holds CUPHU_NOALLOC_MAX_ROWS floats (256 KiB).  Every GPU that
 * loads the library holds it until the process exits.  Scenes with more rows
 * are rejected with CUPHU_ERR_INVALID.
 *
 * In host code the array's name is only a host-side stand-in for the device
 * symbol.  Its device address is looked up once per device, with that device
 * current, by cudaGetSymbolAddress, the first time the entry point runs on
 * that device.  Make that first call before any stream capture begins.  The
 * address is kept for the life of the process: it does not survive a
 * cudaDeviceReset, after which the library's module is loaded anew.
 *
 * Every call on a device shares the one array, and the array keeps the last
 * call's contents.  No element has to start at zero: k_int_rowoff writes rows
 * 0..nrow-1 before k_int_rows reads them, both on the caller's stream.  Two
 * calls that overlap on the GPU (different streams of one device, with no
 * ordering between them) race on the array, so the caller must order them.
 */
#include <mutex>

#include "kernels.cuh"

namespace cuphu {
namespace {

static __device__ __align__(256) float g_rowoff_scratch[CUPHU_NOALLOC_MAX_ROWS];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
float *g_scratch_addr[kMaxDevices] = {};

/* device address of g_rowoff_scratch on device dev (the current device) */
int scratch_address(int dev, float **out)
{
    if (dev < 0 || dev >= kMaxDevices)
        return fail(CUPHU_ERR_UNSUPPORTED, "cuphu_integrate_phase_noalloc: device ordinal " +
                                               std::to_string(dev) + " above the supported 63");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_rowoff_scratch);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaGetSymbolAddress(g_rowoff_scratch)");
        if (!p) return fail(CUPHU_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
        g_scratch_addr[dev] = static_cast<float *>(p);
    }
    *out = g_scratch_addr[dev];
    return 0;
}

}  // namespace
}  // namespace cuphu

using namespace cuphu;

extern "C" int cuphu_integrate_phase_noalloc(const float *wrapped_phase, const short *hflows,
                                             const short *vflows, int nrow, int ncol,
                                             float *unw_out, void *stream)
{
    if (nrow > CUPHU_NOALLOC_MAX_ROWS)
        return fail(CUPHU_ERR_INVALID,
                    "cuphu_integrate_phase_noalloc: nrow=" + std::to_string(nrow) +
                        " exceeds the no-allocation limit of " +
                        std::to_string(CUPHU_NOALLOC_MAX_ROWS) +
                        " rows; use cuphu_integrate_phase_gpu for larger scenes");
    if (!wrapped_phase || !hflows || !vflows || !unw_out || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "cuphu_integrate_phase_noalloc: bad arguments");
    int dev = 0;
    CUPHU_TRY_CUDA(cudaGetDevice(&dev));
    float *rowoff = nullptr;
    int rc = scratch_address(dev, &rowoff);
    if (rc) return rc;
    return launch_integrate(wrapped_phase, hflows, vflows, nrow, ncol, rowoff, unw_out,
                            static_cast<cudaStream_t>(stream));
}
