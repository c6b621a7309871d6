/*
 * scene_stream.cu -- a scene fed to the GPU band by band.
 *
 * The reference reads its inputs whole: cuphu.unwrap() calls np.asarray on
 * the interferogram and the coherence (_unwrap.py:515-523), so a scene held
 * in an HDF5 or GeoTIFF dataset is read completely before any transfer
 * begins.  A stream handle takes row bands instead: for each band the
 * caller's thread computes the reference's host phase (host_phase.cu) and
 * copies coherence and masks into one of two pinned staging slots, and the
 * band's uploads are enqueued on the handle's stream.  While a band is in
 * flight the caller reads the next band from its dataset into the other
 * slot, so storage reads, the phase computation and PCIe transfers overlap.
 * Once every row has arrived, cuphu_stream_unwrap runs the device pipeline
 * on the resident scene and cuphu_stream_get_rows returns the outputs in
 * bands.
 */
#include "kernels.cuh"

#include <cstring>
#include <vector>

namespace cuphu {
namespace {

struct Slot {
    float *ph = nullptr, *corr = nullptr;
    unsigned char *mask = nullptr, *omask = nullptr;
    size_t cap = 0;                 /* pixels */
    cudaEvent_t done = nullptr;
};

struct SceneStream {
    int dev = 0, nrow = 0, ncol = 0, flags = 0;
    cudaStream_t s = nullptr;
    float *d_ph = nullptr, *d_corr = nullptr, *d_unw = nullptr;
    unsigned char *d_mask = nullptr, *d_omask = nullptr;
    uint32_t *d_cc = nullptr;
    Slot slot[2];
    int next = 0;
    long long rows_in = 0;          /* rows received (each row once) */
    std::vector<unsigned char> seen;
    bool solved = false;
};

void free_slot(Slot &z)
{
    if (z.done) cudaEventSynchronize(z.done);
    if (z.ph) cudaFreeHost(z.ph);
    if (z.corr) cudaFreeHost(z.corr);
    if (z.mask) cudaFreeHost(z.mask);
    if (z.omask) cudaFreeHost(z.omask);
    if (z.done) cudaEventDestroy(z.done);
    z = Slot();
}

void destroy(SceneStream *h)
{
    if (!h) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(h->dev);
    if (h->s) cudaStreamSynchronize(h->s);
    for (auto &z : h->slot) free_slot(z);
    for (void *p : {(void *)h->d_ph, (void *)h->d_corr, (void *)h->d_unw, (void *)h->d_mask,
                    (void *)h->d_omask, (void *)h->d_cc})
        if (p) cudaFree(p);
    if (h->s) cudaStreamDestroy(h->s);
    cudaGetLastError();
    cudaSetDevice(cur);
    delete h;
}

int grow_slot(Slot &z, size_t px, int flags)
{
    if (z.done) CUPHU_TRY_CUDA(cudaEventSynchronize(z.done));
    else CUPHU_TRY_CUDA(cudaEventCreateWithFlags(&z.done, cudaEventDisableTiming));
    if (px <= z.cap) return 0;
    cudaEvent_t ev = z.done;
    z.done = nullptr;
    free_slot(z);
    z.done = ev;
    bool ok = cudaHostAlloc((void **)&z.ph, px * 4, cudaHostAllocDefault) == cudaSuccess &&
              cudaHostAlloc((void **)&z.corr, px * 4, cudaHostAllocDefault) == cudaSuccess;
    if (ok && (flags & CUPHU_STREAM_MASK))
        ok = cudaHostAlloc((void **)&z.mask, px, cudaHostAllocDefault) == cudaSuccess;
    if (ok && (flags & CUPHU_STREAM_ORIG_MASK))
        ok = cudaHostAlloc((void **)&z.omask, px, cudaHostAllocDefault) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return fail(CUPHU_ERR_ALLOC, "pinned band staging allocation failed");
    }
    z.cap = px;
    return 0;
}

}  // namespace
}  // namespace cuphu

using namespace cuphu;

extern "C" {

int cuphu_stream_create(int nrow, int ncol, int flags, int gpu_id, void **handle)
{
    if (!handle) return fail(CUPHU_ERR_INVALID, "handle must not be NULL");
    *handle = nullptr;
    if (nrow < 1 || ncol < 1) return fail(CUPHU_ERR_INVALID, "nrow and ncol must be >= 1");
    if (flags & ~(CUPHU_STREAM_MASK | CUPHU_STREAM_ORIG_MASK))
        return fail(CUPHU_ERR_INVALID, "unknown stream flags");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    auto *h = new SceneStream();
    h->dev = gpu_id;
    h->nrow = nrow;
    h->ncol = ncol;
    h->flags = flags;
    h->seen.assign((size_t)nrow, 0);
    const size_t n = (size_t)nrow * ncol;
    bool ok = cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&h->d_ph, n * 4) == cudaSuccess &&
              cudaMalloc(&h->d_corr, n * 4) == cudaSuccess &&
              cudaMalloc(&h->d_unw, n * 4) == cudaSuccess &&
              cudaMalloc(&h->d_cc, n * 4) == cudaSuccess;
    if (ok && (flags & CUPHU_STREAM_MASK)) ok = cudaMalloc(&h->d_mask, n) == cudaSuccess;
    if (ok && (flags & CUPHU_STREAM_ORIG_MASK)) ok = cudaMalloc(&h->d_omask, n) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        destroy(h);
        return fail(CUPHU_ERR_ALLOC, "device allocation of the streamed scene failed");
    }
    *handle = h;
    return 0;
}

int cuphu_stream_put_rows(void *handle, int row0, int nrows, const float *igram_c64,
                          const float *corr, const unsigned char *mask,
                          const unsigned char *orig_mask)
{
    auto *h = static_cast<SceneStream *>(handle);
    if (!h) return fail(CUPHU_ERR_INVALID, "not a stream handle");
    if (row0 < 0 || nrows < 1 || row0 + nrows > h->nrow)
        return fail(CUPHU_ERR_INVALID, "rows outside the scene");
    if (!igram_c64 || !corr) return fail(CUPHU_ERR_INVALID, "igram and corr must not be NULL");
    if (((h->flags & CUPHU_STREAM_MASK) != 0) != (mask != nullptr) ||
        ((h->flags & CUPHU_STREAM_ORIG_MASK) != 0) != (orig_mask != nullptr))
        return fail(CUPHU_ERR_INVALID, "masks must match the flags the stream was created with");
    CUPHU_TRY_CUDA(cudaSetDevice(h->dev));
    Slot &z = h->slot[h->next];
    const size_t px = (size_t)nrows * h->ncol, off = (size_t)row0 * h->ncol;
    int rc = grow_slot(z, px, h->flags);   /* waits for the slot's previous band */
    if (rc) return rc;
    compute_host_phase(igram_c64, nullptr, nullptr, px, z.ph);
    std::memcpy(z.corr, corr, px * 4);
    if (mask) std::memcpy(z.mask, mask, px);
    if (orig_mask) std::memcpy(z.omask, orig_mask, px);
    CUPHU_TRY_CUDA(cudaMemcpyAsync(h->d_ph + off, z.ph, px * 4, cudaMemcpyHostToDevice, h->s));
    CUPHU_TRY_CUDA(cudaMemcpyAsync(h->d_corr + off, z.corr, px * 4, cudaMemcpyHostToDevice, h->s));
    if (mask)
        CUPHU_TRY_CUDA(cudaMemcpyAsync(h->d_mask + off, z.mask, px, cudaMemcpyHostToDevice, h->s));
    if (orig_mask)
        CUPHU_TRY_CUDA(cudaMemcpyAsync(h->d_omask + off, z.omask, px, cudaMemcpyHostToDevice, h->s));
    CUPHU_TRY_CUDA(cudaEventRecord(z.done, h->s));
    h->next ^= 1;
    for (int r = row0; r < row0 + nrows; ++r)
        if (!h->seen[r]) {
            h->seen[r] = 1;
            ++h->rows_in;
        }
    h->solved = false;
    return 0;
}

int cuphu_stream_unwrap(void *handle, CuPhuCostMode cost_mode, const CuPhuParams *params,
                        const CuPhuTileParams *tile, const CuPhuSolveOptions *opts,
                        CuPhuSolveStats *stats)
{
    auto *h = static_cast<SceneStream *>(handle);
    if (!h) return fail(CUPHU_ERR_INVALID, "not a stream handle");
    if (h->rows_in != h->nrow) return fail(CUPHU_ERR_INVALID, "not every row of the scene was put");
    CUPHU_TRY_CUDA(cudaSetDevice(h->dev));
    int rc = cuphu_unwrap_device(nullptr, h->d_ph, h->d_corr, h->d_mask, h->d_omask, h->nrow,
                                 h->ncol, cost_mode, params, tile, opts, h->d_unw, h->d_cc,
                                 nullptr, stats, h->s);
    if (rc) return rc;
    CUPHU_TRY_CUDA(cudaStreamSynchronize(h->s));
    rc = cuphu_last_status(h->dev);
    if (!rc) h->solved = true;
    return rc;
}

int cuphu_stream_get_rows(void *handle, int row0, int nrows, float *unw_out,
                          uint32_t *conncomp_out)
{
    auto *h = static_cast<SceneStream *>(handle);
    if (!h) return fail(CUPHU_ERR_INVALID, "not a stream handle");
    if (!h->solved) return fail(CUPHU_ERR_INVALID, "the streamed scene has not been unwrapped");
    if (row0 < 0 || nrows < 1 || row0 + nrows > h->nrow)
        return fail(CUPHU_ERR_INVALID, "rows outside the scene");
    CUPHU_TRY_CUDA(cudaSetDevice(h->dev));
    const size_t px = (size_t)nrows * h->ncol, off = (size_t)row0 * h->ncol;
    if (unw_out)
        CUPHU_TRY_CUDA(cudaMemcpyAsync(unw_out, h->d_unw + off, px * 4, cudaMemcpyDeviceToHost,
                                       h->s));
    if (conncomp_out)
        CUPHU_TRY_CUDA(cudaMemcpyAsync(conncomp_out, h->d_cc + off, px * 4,
                                       cudaMemcpyDeviceToHost, h->s));
    CUPHU_TRY_CUDA(cudaStreamSynchronize(h->s));
    return 0;
}

int cuphu_stream_destroy(void *handle)
{
    destroy(static_cast<SceneStream *>(handle));
    return 0;
}

}  // extern "C"
