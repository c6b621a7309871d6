/*
 * api.cu -- C ABI of libcuphu_b200 and the host orchestrator.
 *
 * Replaces cuphu_unwrap / solve_tile / cuphu_build_costs_gpu
 * (cuphu_solver.cpp:370-510, 1675-2171) for the Laplace path.  Differences
 * in mechanism (not in results):
 *  - one stream per call, no host threads: all tiles of all scenes are
 *    planned on the host and solved by one persistent launch;
 *  - no host round trips inside the pipeline: phase, weights, solve,
 *    labelling, stitching and merge are device kernels, the host copies the
 *    inputs in and the outputs out once;
 *  - a grow-only per-device workspace replaces the reference's per-call
 *    cudaMalloc/cudaFree; calls on one device are serialised by a mutex and
 *    ordered on the GPU by an event, so asynchronous device-pointer calls on
 *    different streams never share scratch concurrently;
 *  - errors are returned as status codes (cuphu_last_error() has the text),
 *    never thrown across the ABI.
 */
#include "kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

namespace cuphu {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return 0;
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    /* the error is reported now: clear the thread's last-error state so a
     * later call's cudaGetLastError check does not report it again */
    cudaGetLastError();
    return CUPHU_ERR_CUDA;
}

/* an asynchronous copy whose immediate error (a bad pointer or size)
 * becomes the call's status instead of passing unnoticed */
static int copy_async(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind,
                      cudaStream_t s, const char *what)
{
    return cuda_fail(cudaMemcpyAsync(dst, src, bytes, kind, s), what);
}

/* ── per-device workspace ──────────────────────────────────────────────── */
struct Workspace {
    std::mutex mu;
    char *dev = nullptr;
    size_t dev_size = 0;
    char *host = nullptr;   /* pinned staging for descriptors */
    size_t host_size = 0;
    cudaEvent_t done = nullptr;
    cudaStream_t stream = nullptr;
    int *status = nullptr;  /* pinned: device status of the last job */
};

static Workspace g_ws[64];

static int ws_prepare(Workspace *W, size_t dbytes, size_t hbytes, cudaStream_t s)
{
    /* each member is set only once its creation succeeded, so a failed first
     * call leaves nothing half-made for the next one */
    if (!W->status) {
        int *st = nullptr;
        CUPHU_TRY_CUDA(cudaHostAlloc((void **)&st, sizeof(int), cudaHostAllocDefault));
        *st = 0;
        W->status = st;
    }
    if (!W->done) {
        cudaEvent_t ev = nullptr;
        CUPHU_TRY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        W->done = ev;
        CUPHU_TRY_CUDA(cudaEventRecord(W->done, s));
    }
    if (dbytes > W->dev_size) {
        CUPHU_TRY_CUDA(cudaDeviceSynchronize());
        if (W->dev) cudaFree(W->dev);
        W->dev = nullptr;
        W->dev_size = 0;
        size_t want = dbytes + dbytes / 8 + (1u << 20);
        if (cudaMalloc(&W->dev, want) != cudaSuccess) {
            cudaGetLastError();
            if (cudaMalloc(&W->dev, dbytes) != cudaSuccess) {
                cudaGetLastError();
                return fail(CUPHU_ERR_ALLOC, "device workspace allocation failed (" +
                                                 std::to_string(dbytes >> 20) + " MiB)");
            }
            want = dbytes;
        }
        W->dev_size = want;
    }
    if (hbytes > W->host_size) {
        CUPHU_TRY_CUDA(cudaEventSynchronize(W->done));
        if (W->host) cudaFreeHost(W->host);
        W->host = nullptr;
        W->host_size = 0;
        size_t want = hbytes + hbytes / 4 + 4096;
        if (cudaHostAlloc((void **)&W->host, want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return fail(CUPHU_ERR_ALLOC, "pinned staging allocation failed");
        }
        W->host_size = want;
    }
    /* previous user of the workspace (any stream) must be done on the GPU; the
     * pinned staging buffer is rewritten by the host, so wait on the host */
    CUPHU_TRY_CUDA(cudaEventSynchronize(W->done));
    return 0;
}

static int ws_acquire(int dev, size_t dbytes, size_t hbytes, cudaStream_t s, Workspace *&W)
{
    if (dev < 0 || dev >= 64) return fail(CUPHU_ERR_INVALID, "device index out of range");
    W = &g_ws[dev];
    return ws_prepare(W, dbytes, hbytes, s);
}

static void ws_free(Workspace &W)
{
    if (W.dev) cudaFree(W.dev);
    if (W.host) cudaFreeHost(W.host);
    if (W.status) cudaFreeHost(W.status);
    if (W.done) cudaEventDestroy(W.done);
    W.dev = nullptr; W.host = nullptr; W.status = nullptr; W.done = nullptr;
    W.dev_size = W.host_size = 0;
}

/* the timing events of one call, destroyed on every return path */
struct Timers {
    cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
    explicit Timers(int n)
    {
        for (int i = 0; i < n && i < 4; ++i)
            if (cudaEventCreate(&e[i]) != cudaSuccess) {
                e[i] = nullptr;
                cudaGetLastError();
            }
    }
    ~Timers()
    {
        for (cudaEvent_t x : e)
            if (x) cudaEventDestroy(x);
    }
    Timers(const Timers &) = delete;
    Timers &operator=(const Timers &) = delete;
};

/* a captured batch pipeline: its own workspace (the descriptors and device
 * pointers are baked into the graph) and the instantiated graph */
struct GraphJob {
    Workspace ws;
    cudaGraphExec_t exec = nullptr;
    int dev = 0;
};

struct Bump {
    char *base;
    size_t off = 0;
    explicit Bump(char *b) : base(b) {}
    template <typename T> T *take(size_t n)
    {
        off = (off + 255) & ~(size_t)255;
        T *p = reinterpret_cast<T *>(base + off);
        off += n * sizeof(T);
        return p;
    }
};

/* ── planning ──────────────────────────────────────────────────────────── */
struct SceneIn {
    const float2 *ig = nullptr;
    const float *re = nullptr, *im = nullptr;
    const float *ph_in = nullptr;
    const float *corr = nullptr;
    const unsigned char *mask = nullptr, *conf = nullptr;
    int nrow = 0, ncol = 0, ntr = 1, ntc = 1, rovl = 0, covl = 0;
    double nlooks = 1.0;
    float *unw = nullptr;
    uint32_t *cc = nullptr;
    int ref_row = -1, ref_col = -1;
    /* optional post-passes on the stitched scene (multi-tile scenes only,
     * as in the reference's tiled path, cuphu_solver.cpp:2036-2095) */
    int feedback = 0, feather = 200, spikes = 0;
    /* labels of the whole stitched scene instead of per-tile label spaces */
    int merge_cc = 0;
};

static bool merges_labels(const SceneIn &in)
{
    return in.merge_cc && in.cc && (in.ntr > 1 || in.ntc > 1);
}

static bool has_postpass(const SceneIn &in)
{
    return (in.ntr > 1 || in.ntc > 1) && (in.feedback || in.spikes);
}

static void tile_bounds(int n, int nt, int ovl, int t, int &first, int &len)
{
    int f = (int)((long long)t * (n - ovl) / nt);
    int last = (t == nt - 1) ? n : (int)((long long)(t + 1) * (n - ovl) / nt) + ovl;
    first = f;
    len = last - f;
}

struct Plan {
    std::vector<TileDesc> tiles;
    std::vector<int> item_tile, row_tile, maps;
    std::vector<ScenePlan> scenes;
    std::vector<PairDesc> pairs;
    std::vector<CostConsts> consts;
    std::vector<size_t> map_off;
    long long nplane = 0;
    int nitems = 0, total_rows = 0, pitch = 4;
};

static int plan_job(const std::vector<SceneIn> &S, const CuPhuParams &prm, Plan &pl)
{
    for (size_t s = 0; s < S.size(); ++s) {
        const SceneIn &in = S[s];
        if (in.nrow < 1 || in.ncol < 1) return fail(CUPHU_ERR_INVALID, "scene shape must be >= 1x1");
        if (in.ntr < 1 || in.ntc < 1 || in.ntr > in.nrow || in.ntc > in.ncol)
            return fail(CUPHU_ERR_INVALID, "tile counts must be in [1, extent]");
        if (in.rovl < 0 || in.covl < 0) return fail(CUPHU_ERR_INVALID, "tile overlap must be >= 0");
        bool single = in.ntr == 1 && in.ntc == 1;
        ScenePlan sp = {};
        sp.unw_out = in.unw;
        sp.cc_out = in.cc;
        sp.nrow = in.nrow;
        sp.ncol = in.ncol;
        sp.ntr = in.ntr;
        sp.ntc = in.ntc;
        sp.rovl = in.rovl;
        sp.covl = in.covl;
        sp.tile0 = (int)pl.tiles.size();
        sp.pair0 = (int)pl.pairs.size();
        /* with post-passes the reference-pixel shift follows them */
        sp.ref_row = has_postpass(in) ? -1 : in.ref_row;
        sp.ref_col = has_postpass(in) ? -1 : in.ref_col;
        sp.maxncomps = (int)std::min<long>(prm.maxncomps, 0x7fffffffL);
        sp.minfrac = prm.minconncompfrac;
        sp.single = single ? 1 : 0;
        CuPhuParams p2 = prm;
        p2.nlooks = p2.ncorrlooks = in.nlooks;
        pl.consts.push_back(make_cost_consts(p2));
        for (int tr = 0; tr < in.ntr; ++tr)
            for (int tc = 0; tc < in.ntc; ++tc) {
                TileDesc T = {};
                if (single) { T.r0 = 0; T.nr = in.nrow; T.c0 = 0; T.nc = in.ncol; }
                else {
                    tile_bounds(in.nrow, in.ntr, in.rovl, tr, T.r0, T.nr);
                    tile_bounds(in.ncol, in.ntc, in.covl, tc, T.c0, T.nc);
                }
                if (T.nr < 1 || T.nc < 1 || T.r0 < 0 || T.c0 < 0 || T.r0 + T.nr > in.nrow ||
                    T.c0 + T.nc > in.ncol)
                    return fail(CUPHU_ERR_INVALID, "tile geometry degenerates (overlap too large)");
                T.scene = (int)s;
                T.tr = tr;
                T.tc = tc;
                T.ph_pitch = in.ncol;
                T.pitch = (T.nc + 3) & ~3;   /* replaced by the common pitch below */
                T.nbx = (T.nc + kItemBx - 1) / kItemBx;
                int nby = (T.nr + kItemBy - 1) / kItemBy;
                T.nitems = T.nbx * nby;
                T.item0 = pl.nitems;
                pl.nitems += T.nitems;
                T.row0 = pl.total_rows;
                pl.total_rows += T.nr;
                int tidx = (int)pl.tiles.size();
                for (int i = 0; i < T.nitems; ++i) pl.item_tile.push_back(tidx);
                for (int i = 0; i < T.nr; ++i) pl.row_tile.push_back(tidx);
                pl.tiles.push_back(T);
            }
        if (!single && (in.rovl > 0 || in.covl > 0)) {
            for (int tr = 0; tr < in.ntr; ++tr)
                for (int tc = 0; tc + 1 < in.ntc; ++tc)
                    pl.pairs.push_back({sp.tile0 + tr * in.ntc + tc, sp.tile0 + tr * in.ntc + tc + 1, 0,
                                        in.covl});
            for (int tr = 0; tr + 1 < in.ntr; ++tr)
                for (int tc = 0; tc < in.ntc; ++tc)
                    pl.pairs.push_back({sp.tile0 + tr * in.ntc + tc, sp.tile0 + (tr + 1) * in.ntc + tc, 1,
                                        in.rovl});
        }
        /* merge maps: the last tile (in row-major order) whose kept interval
         * covers a row/column wins, as the reference's sequential merge does */
        pl.map_off.push_back(pl.maps.size());
        std::vector<int> rm(in.nrow, 0), cm(in.ncol, 0);
        if (!single) {
            for (int tr = 0; tr < in.ntr; ++tr) {
                int f, n;
                tile_bounds(in.nrow, in.ntr, in.rovl, tr, f, n);
                int a = tr == 0 ? 0 : in.rovl / 2, b = tr == in.ntr - 1 ? n : n - in.rovl / 2;
                for (int r = f + a; r < f + b; ++r) rm[r] = tr;
            }
            for (int tc = 0; tc < in.ntc; ++tc) {
                int f, n;
                tile_bounds(in.ncol, in.ntc, in.covl, tc, f, n);
                int a = tc == 0 ? 0 : in.covl / 2, b = tc == in.ntc - 1 ? n : n - in.covl / 2;
                for (int c = f + a; c < f + b; ++c) cm[c] = tc;
            }
        }
        pl.maps.insert(pl.maps.end(), rm.begin(), rm.end());
        pl.maps.insert(pl.maps.end(), cm.begin(), cm.end());
        pl.scenes.push_back(sp);
    }
    /* common pitch: tiles are stacked row-wise into one 2-D array per plane */
    int P = 4;
    for (auto &T : pl.tiles) P = std::max(P, T.pitch);
    pl.pitch = P;
    for (auto &T : pl.tiles) {
        T.pitch = P;
        T.pix = (long long)T.row0 * P;
    }
    pl.nplane = (long long)pl.total_rows * P;
    return 0;
}

struct JobOpts {
    bool fp64 = false;
    bool want_cc = true;
    bool want_cyc = false;
    CuPhuSolveOptions so;
    const short *costs = nullptr;   /* launcher-level entry: w0 from a cost array */
    int cost_stride = 2;
    int32_t *cycles_out = nullptr;
    float *cont_out = nullptr;      /* anchored continuous solution (single tile) */
    /* WLS mode (single tile): caller's per-arc weights and targets or
     * right-hand side, optional FP64 warm start, raw FP64 solution out */
    GraphJob *graph = nullptr;      /* capture mode: leave the capture open on s */
    bool wls = false;
    const float *wls_gd = nullptr, *wls_gr = nullptr, *wls_rhs = nullptr;
    const float *wls_wd = nullptr, *wls_wr = nullptr;
    const double *wls_u0 = nullptr;
    double *wls_u = nullptr;
};

/* WLS mode of run_job: copy the caller's planes into the tile layout, one
 * solve without reweighting, raw FP64 solution out. */
static int wls_job(const Plan &pl, SolverPlanes &P, const JobOpts &jo, cudaStream_t s,
                   TileDesc *d_tiles, int *d_item, int ntiles, TileState *d_st, double *d_part,
                   SolverCtl *d_ctl, float *d_deltas, int *d_pass, int dev, Workspace *W,
                   CuPhuSolveStats *stats)
{
    const TileDesc &T = pl.tiles[0];
    const size_t sp_b = (size_t)T.pitch * 4, sc_b = (size_t)T.nc * 4;
    auto put = [&](float *dst, const float *src) -> cudaError_t {
        return cudaMemcpy2DAsync(dst, sp_b, src, sc_b, sc_b, T.nr, cudaMemcpyDeviceToDevice, s);
    };
    const size_t np = (size_t)pl.nplane;
    /* weights: zero the padding, then the caller's planes (also as w0) */
    CUPHU_TRY_CUDA(cudaMemsetAsync(P.wd, 0, np * 4, s));
    CUPHU_TRY_CUDA(cudaMemsetAsync(P.wr, 0, np * 4, s));
    CUPHU_TRY_CUDA(put(P.wd, jo.wls_wd));
    CUPHU_TRY_CUDA(put(P.wr, jo.wls_wr));
    CUPHU_TRY_CUDA(put(P.w0d, jo.wls_wd));
    CUPHU_TRY_CUDA(put(P.w0r, jo.wls_wr));
    if (P.gd) CUPHU_TRY_CUDA(put((float *)P.gd, jo.wls_gd));
    if (P.gr) CUPHU_TRY_CUDA(put((float *)P.gr, jo.wls_gr));
    if (P.rhs) CUPHU_TRY_CUDA(put((float *)P.rhs, jo.wls_rhs));
    if (jo.wls_u0) {
        CUPHU_TRY_CUDA(cudaMemcpy2DAsync(P.x, (size_t)T.pitch * 8, jo.wls_u0, (size_t)T.nc * 8,
                                         (size_t)T.nc * 8, T.nr, cudaMemcpyDeviceToDevice, s));
        if (P.dx) CUPHU_TRY_CUDA(cudaMemsetAsync(P.dx, 0, np * 4, s));
    }
    const CuPhuSolveOptions &o = jo.so;
    SolveParams sp;
    sp.n_irls = 0;
    sp.max_iter = o.max_iter;
    sp.replace_every = jo.fp64 ? 0 : o.replace_every;
    sp.tol = o.tol;
    sp.deltas = d_deltas;
    sp.pass_iters = d_pass;
    sp.timeout_ns = (long long)std::max(1, o.timeout_ms) * 1000000LL;
    sp.wls = 1;
    sp.warm = jo.wls_u0 ? 1 : 0;
    Timers tm(stats ? 2 : 0);
    cudaEvent_t e1 = tm.e[0], e2 = tm.e[1];
    if (stats) cudaEventRecord(e1, s);
    int rc = launch_solve(jo.fp64, d_tiles, d_item, pl.nitems, ntiles, P, pl.pitch, pl.total_rows,
                          d_st, d_part, d_ctl, sp, dev, s);
    if (rc) return rc;
    CUPHU_TRY_CUDA(cudaMemcpy2DAsync(jo.wls_u, (size_t)T.nc * 8, P.x, (size_t)T.pitch * 8,
                                     (size_t)T.nc * 8, T.nr, cudaMemcpyDeviceToDevice, s));
    CUPHU_TRY_CUDA(cudaMemcpyAsync(W->status, &d_ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUPHU_TRY_CUDA(cudaEventRecord(W->done, s));
    if (stats) {
        cudaEventRecord(e2, s);
        CUPHU_TRY_CUDA(cudaEventSynchronize(e2));
        SolverCtl ctl;
        CUPHU_TRY_CUDA(cudaMemcpy(&ctl, d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
        float ms = 0;
        cudaEventElapsedTime(&ms, e1, e2);
        stats->ntiles = ntiles;
        stats->total_iters = ctl.total_iters;
        stats->max_iters_pass = ctl.max_pass_iters;
        stats->solve_ms = ms;
        stats->total_ms = ms;
        stats->px_iters = (double)ctl.px_iters;
        if (ctl.err) return fail(CUPHU_ERR_TIMEOUT, "solver grid barrier timed out");
    }
    return 0;
}

/* Enqueue the whole unwrapping pipeline for a list of scenes on stream s. */
static int run_job(std::vector<SceneIn> &S, const CuPhuParams &prm, const JobOpts &jo,
                   cudaStream_t s, CuPhuSolveStats *stats)
{
    int dev = 0;
    CUPHU_TRY_CUDA(cudaGetDevice(&dev));
    Plan pl;
    int rc = plan_job(S, prm, pl);
    if (rc) return rc;
    const CuPhuSolveOptions &o = jo.so;
    if (o.n_irls < 0 || o.n_irls > 4096) return fail(CUPHU_ERR_INVALID, "n_irls out of range");
    if (o.max_iter < 0) return fail(CUPHU_ERR_INVALID, "max_iter must be >= 0");
    const int ntiles = (int)pl.tiles.size(), nsc = (int)S.size(), npairs = (int)pl.pairs.size();
    const size_t vs = jo.fp64 ? sizeof(double) : sizeof(float);
    const size_t np = (size_t)pl.nplane;

    /* device layout */
    size_t post_bytes = 0;
    for (auto &in : S)
        if (has_postpass(in)) post_bytes = std::max(post_bytes, postpass_scratch_bytes(in.nrow, in.ncol));
    char *d_post = nullptr;
    SceneOut *d_shift = nullptr;
    /* scene-level labelling of merged scenes: one descriptor each (uploaded
     * with the tile descriptors) and one set of pitched planes */
    int n_merge = 0;
    size_t cc_bytes = 0;
    for (auto &in : S)
        if (merges_labels(in)) {
            ++n_merge;
            const size_t pitch = ((size_t)in.ncol + 3) & ~(size_t)3;
            const size_t items = (size_t)((in.ncol + kItemBx - 1) / kItemBx) *
                                 ((in.nrow + kItemBy - 1) / kItemBy);
            cc_bytes = std::max(cc_bytes, (size_t)in.nrow * pitch * 12 + items * 4 +
                                              (size_t)in.nrow * 8 + 4096);
        }
    TileDesc *d_cctd = nullptr;
    char *d_ccbuf = nullptr;
    size_t need_phase = 0;
    for (auto &in : S)
        if (!in.ph_in) need_phase += (size_t)in.nrow * in.ncol;
    auto layout = [&](Bump &b, SolverPlanes &P, float *&phase, TileDesc *&d_tiles, int *&d_item,
                      ScenePlan *&d_sc, PairDesc *&d_pairs, int *&d_maps, int *&d_rowcnt,
                      int *&d_nlab, double *&d_pairk, double *&d_tilek, unsigned *&d_coff,
                      SceneOut *&d_sout, CostConsts *&d_k, TileState *&d_st, double *&d_part,
                      SolverCtl *&d_ctl, float *&d_deltas, int *&d_pass) {
        phase = b.take<float>(need_phase);
        P.w0d = b.take<float>(np);
        P.w0r = b.take<float>(np);
        P.wd = b.take<float>(np);
        P.wr = b.take<float>(np);
        P.x = b.take<double>(np);
        P.dx = jo.fp64 ? nullptr : b.take<float>(np);
        P.bvec = jo.fp64 ? nullptr : b.take<double>(np);
        P.r = b.take<char>(np * vs);
        P.p0 = b.take<char>(np * vs);
        P.p1 = b.take<char>(np * vs);
        P.q = b.take<char>(np * vs);
        P.diag = b.take<char>(np * vs);
        P.z = b.take<char>(np * vs);
        P.q1 = jo.fp64 ? nullptr : b.take<float>(np);
        P.unw = b.take<float>(np);
        P.cyc = jo.want_cyc ? b.take<int32_t>(np) : nullptr;
        P.cont = jo.cont_out ? b.take<float>(np) : nullptr;
        P.cc = b.take<uint32_t>(np);
        P.aux = b.take<uint32_t>(np);
        if (jo.wls) {
            P.gd = jo.wls_gd ? b.take<float>(np) : nullptr;
            P.gr = jo.wls_gr ? b.take<float>(np) : nullptr;
            P.rhs = jo.wls_rhs ? b.take<float>(np) : nullptr;
        }
        d_tiles = b.take<TileDesc>(ntiles);
        d_item = b.take<int>(pl.nitems);
        d_sc = b.take<ScenePlan>(nsc);
        d_pairs = b.take<PairDesc>(std::max(npairs, 1));
        d_maps = b.take<int>(pl.maps.size());
        d_rowcnt = b.take<int>(2 * (size_t)pl.total_rows);
        d_nlab = b.take<int>(ntiles);
        d_pairk = b.take<double>(npairs + ntiles + 1);
        d_tilek = b.take<double>(ntiles);
        d_coff = b.take<unsigned>(ntiles);
        d_sout = b.take<SceneOut>(nsc);
        d_k = b.take<CostConsts>(nsc);
        d_cctd = b.take<TileDesc>(std::max(n_merge, 1));
        d_st = b.take<TileState>(2 * (size_t)ntiles);
        /* item partials x2, published tile totals x2 (kNComp components
         * each), tile item tickets */
        d_part = b.take<double>(2 * (size_t)kNComp * pl.nitems + (2 * (size_t)kNComp + 1) * ntiles);
        d_ctl = b.take<SolverCtl>(1);
        d_deltas = b.take<float>(o.n_irls + 1);
        d_pass = b.take<int>(o.n_irls + 1);
        d_post = post_bytes ? b.take<char>(post_bytes) : nullptr;
        d_shift = b.take<SceneOut>(nsc);
        d_ccbuf = cc_bytes ? b.take<char>(cc_bytes) : nullptr;
    };
    SolverPlanes P = {};
    float *phase = nullptr, *d_deltas = nullptr;
    TileDesc *d_tiles = nullptr;
    int *d_item = nullptr, *d_maps = nullptr, *d_rowcnt = nullptr, *d_nlab = nullptr, *d_pass = nullptr;
    ScenePlan *d_sc = nullptr;
    PairDesc *d_pairs = nullptr;
    double *d_pairk = nullptr, *d_tilek = nullptr, *d_part = nullptr;
    unsigned *d_coff = nullptr;
    SceneOut *d_sout = nullptr;
    CostConsts *d_k = nullptr;
    TileState *d_st = nullptr;
    SolverCtl *d_ctl = nullptr;
    Bump probe(nullptr);
    layout(probe, P, phase, d_tiles, d_item, d_sc, d_pairs, d_maps, d_rowcnt, d_nlab, d_pairk,
           d_tilek, d_coff, d_sout, d_k, d_st, d_part, d_ctl, d_deltas, d_pass);
    size_t dbytes = probe.off + 256;
    /* host staging: descriptors packed in the same order as the device copy */
    size_t desc_begin = (size_t)((char *)d_tiles - (char *)nullptr);
    size_t desc_end = (size_t)((char *)d_st - (char *)nullptr);
    size_t hbytes = desc_end - desc_begin + 256;

    std::unique_lock<std::mutex> lock;
    Workspace *W = nullptr;
    if (jo.graph) {
        if (stats) return fail(CUPHU_ERR_INVALID, "statistics are not available in a graph");
        W = &jo.graph->ws;
        rc = ws_prepare(W, dbytes, hbytes, s);
    } else {
        if (dev < 0 || dev >= 64) return fail(CUPHU_ERR_UNSUPPORTED, "device ordinal above 63");
        lock = std::unique_lock<std::mutex>(g_ws[dev].mu);
        rc = ws_acquire(dev, dbytes, hbytes, s, W);
    }
    if (rc) return rc;
    Bump b(W->dev);
    layout(b, P, phase, d_tiles, d_item, d_sc, d_pairs, d_maps, d_rowcnt, d_nlab, d_pairk, d_tilek,
           d_coff, d_sout, d_k, d_st, d_part, d_ctl, d_deltas, d_pass);

    /* finalise descriptors with device addresses */
    size_t poff = 0;
    std::vector<const float *> scene_ph(nsc);
    for (int i = 0; i < nsc; ++i) {
        if (S[i].ph_in) scene_ph[i] = S[i].ph_in;
        else {
            scene_ph[i] = phase + poff;
            poff += (size_t)S[i].nrow * S[i].ncol;
        }
        pl.scenes[i].ph = scene_ph[i];
        pl.scenes[i].rowmap = d_maps + pl.map_off[i];
        pl.scenes[i].colmap = d_maps + pl.map_off[i] + S[i].nrow;
    }
    for (auto &T : pl.tiles) {
        const SceneIn &in = S[T.scene];
        size_t o0 = (size_t)T.r0 * in.ncol + T.c0;
        T.ph = scene_ph[T.scene] + o0;
        T.corr = in.corr + o0;
        T.mask = in.mask ? in.mask + o0 : nullptr;
        T.conf = in.conf ? in.conf + o0 : (in.mask ? in.mask + o0 : nullptr);
    }
    char *h = W->host;
    auto put = [&](void *dptr, const void *src, size_t n) {
        size_t off = (size_t)((char *)dptr - (char *)d_tiles);
        if (n) std::memcpy(h + off, src, n);
    };
    put(d_tiles, pl.tiles.data(), ntiles * sizeof(TileDesc));
    put(d_item, pl.item_tile.data(), pl.nitems * sizeof(int));
    put(d_sc, pl.scenes.data(), nsc * sizeof(ScenePlan));
    put(d_pairs, pl.pairs.data(), npairs * sizeof(PairDesc));
    put(d_maps, pl.maps.data(), pl.maps.size() * sizeof(int));
    put(d_rowcnt + pl.total_rows, pl.row_tile.data(), pl.total_rows * sizeof(int));
    put(d_k, pl.consts.data(), nsc * sizeof(CostConsts));
    std::vector<TileDesc> cctd;
    for (auto &in : S)
        if (merges_labels(in)) {
            TileDesc T = {};
            T.ph = in.unw;
            T.corr = in.corr;
            T.mask = in.mask;
            T.ph_pitch = in.ncol;
            T.nr = in.nrow;
            T.nc = in.ncol;
            T.pitch = (in.ncol + 3) & ~3;
            T.nbx = (in.ncol + kItemBx - 1) / kItemBx;
            T.nitems = T.nbx * ((in.nrow + kItemBy - 1) / kItemBy);
            cctd.push_back(T);
        }
    put(d_cctd, cctd.data(), cctd.size() * sizeof(TileDesc));

    Timers tm(stats ? 4 : 0);
    cudaEvent_t e0 = tm.e[0], e1 = tm.e[1], e2 = tm.e[2], e3 = tm.e[3];
    if (stats) cudaEventRecord(e0, s);
    /* IRLS schedule, host powf exactly as cuphu_laplace.cu:517-518 */
    std::vector<float> deltas(o.n_irls + 1, 0.0f);
    for (int k = 0; k < o.n_irls; ++k)
        deltas[k] = std::max(o.irls_delta_min, o.irls_delta_max * powf(0.5f, (float)k));
    if (jo.graph) {
        /* the graph replays everything after the descriptors: upload them
         * now, then capture the rest */
        CUPHU_TRY_CUDA(cudaMemcpy(d_tiles, h, (char *)d_st - (char *)d_tiles,
                                  cudaMemcpyHostToDevice));
        CUPHU_TRY_CUDA(cudaMemcpy(d_deltas, deltas.data(), deltas.size() * sizeof(float),
                                  cudaMemcpyHostToDevice));
        CUPHU_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    } else {
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_tiles, h, (char *)d_st - (char *)d_tiles,
                                       cudaMemcpyHostToDevice, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(d_deltas, deltas.data(), deltas.size() * sizeof(float),
                                       cudaMemcpyHostToDevice, s));
    }
    CUPHU_TRY_CUDA(cudaMemsetAsync(d_st, 0, 2 * ntiles * sizeof(TileState), s));
    CUPHU_TRY_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(SolverCtl), s));
    CUPHU_TRY_CUDA(cudaMemsetAsync(d_part + 2 * (size_t)kNComp * pl.nitems +
                                       2 * (size_t)kNComp * ntiles,
                                   0, (size_t)ntiles * sizeof(double), s));

    if (jo.wls) return wls_job(pl, P, jo, s, d_tiles, d_item, ntiles, d_st, d_part, d_ctl,
                               d_deltas, d_pass, dev, W, stats);
    for (int i = 0; i < nsc; ++i) {
        if (S[i].ph_in) continue;
        long long n = (long long)S[i].nrow * S[i].ncol;
        rc = S[i].ig ? launch_phase(S[i].ig, (float *)scene_ph[i], n, s)
                     : launch_phase_split(S[i].re, S[i].im, (float *)scene_ph[i], n, s);
        if (rc) return rc;
    }
    if (jo.costs) {
        const TileDesc &T = pl.tiles[0];
        rc = launch_w0_from_costs(jo.costs, jo.cost_stride, T.nr, T.nc, T.pitch, P, s);
    } else {
        rc = launch_w0(d_tiles, d_item, pl.nitems, d_k, P, s);
    }
    if (rc) return rc;
    SolveParams sp;
    sp.n_irls = o.n_irls;
    sp.max_iter = o.max_iter;
    sp.replace_every = jo.fp64 ? 0 : o.replace_every;
    sp.tol = o.tol;
    sp.deltas = d_deltas;
    sp.pass_iters = d_pass;
    sp.timeout_ns = (long long)std::max(1, o.timeout_ms) * 1000000LL;
    if (stats) cudaEventRecord(e1, s);
    rc = launch_solve(jo.fp64, d_tiles, d_item, pl.nitems, ntiles, P, pl.pitch, pl.total_rows, d_st,
                      d_part, d_ctl, sp, dev, s);
    if (rc) return rc;
    if (stats) cudaEventRecord(e2, s);
    if (jo.want_cc) {
        CcArgs ca;
        ca.poscost = nullptr;
        ca.negcost = nullptr;
        ca.corr_thresh = 0.05f;
        ca.conncompthresh = prm.conncompthresh;
        ca.minfrac = prm.minconncompfrac;
        ca.maxncomps = (int)std::min<long>(prm.maxncomps, 0x7fffffffL);
        rc = launch_conncomp(d_tiles, ntiles, pl.total_rows, d_item, pl.nitems, P, ca, d_rowcnt,
                             d_nlab, s);
        if (rc) return rc;
    } else {
        CUPHU_TRY_CUDA(cudaMemsetAsync(d_nlab, 0, ntiles * sizeof(int), s));
    }
    rc = launch_stitch(d_sc, nsc, d_tiles, d_pairs, npairs, P, d_nlab, d_pairk, d_tilek, d_coff,
                       d_sout, s);
    if (rc) return rc;
    rc = launch_merge(d_sc, pl.scenes.data(), nsc, d_tiles, P, d_tilek, d_coff, d_sout, s);
    if (rc) return rc;
    /* post-passes on the stitched scenes, in the reference's order, then the
     * reference-pixel shift they deferred */
    for (int i = 0; i < nsc; ++i) {
        const SceneIn &in = S[i];
        if (!has_postpass(in)) continue;
        if (in.feedback)
            rc = launch_neighbor_feedback(in.unw, in.mask, in.nrow, in.ncol, in.ntr, in.ntc,
                                          in.rovl, in.covl, in.feather, d_post, s);
        if (!rc && in.spikes) rc = launch_fix_cycle_spikes(in.unw, in.mask, in.nrow, in.ncol, d_post, s);
        if (!rc) rc = launch_ref_shift(in.unw, scene_ph[i], in.nrow, in.ncol, in.ref_row, in.ref_col,
                                       d_shift + i, s);
        if (rc) return rc;
    }
    /* labels over the whole stitched scene (the same criteria as the
     * per-tile labelling, cuphu_conncomp.cu:290-428): components that cross
     * tile seams get one label */
    for (int i = 0, j = 0; i < nsc; ++i) {
        const SceneIn &in = S[i];
        if (!merges_labels(in)) continue;
        const TileDesc &T = cctd[j];
        const size_t np_s = (size_t)in.nrow * T.pitch;
        Bump cb(d_ccbuf);
        SolverPlanes Q = {};
        Q.unw = cb.take<float>(np_s);
        Q.cc = cb.take<uint32_t>(np_s);
        Q.aux = cb.take<uint32_t>(np_s);
        int *c_item = cb.take<int>(T.nitems);
        int *c_row = cb.take<int>(2 * (size_t)in.nrow);
        int *c_nlab = cb.take<int>(1);
        CUPHU_TRY_CUDA(cudaMemsetAsync(c_item, 0, (size_t)T.nitems * 4, s));
        CUPHU_TRY_CUDA(cudaMemsetAsync(c_row + in.nrow, 0, (size_t)in.nrow * 4, s));
        CUPHU_TRY_CUDA(cudaMemcpy2DAsync(Q.unw, (size_t)T.pitch * 4, in.unw, (size_t)in.ncol * 4,
                                         (size_t)in.ncol * 4, in.nrow, cudaMemcpyDeviceToDevice, s));
        CcArgs ca;
        ca.poscost = nullptr;
        ca.negcost = nullptr;
        ca.corr_thresh = 0.05f;
        ca.conncompthresh = prm.conncompthresh;
        ca.minfrac = prm.minconncompfrac;
        ca.maxncomps = (int)std::min<long>(prm.maxncomps, 0x7fffffffL);
        rc = launch_conncomp(d_cctd + j, 1, in.nrow, c_item, T.nitems, Q, ca, c_row, c_nlab, s);
        if (rc) return rc;
        CUPHU_TRY_CUDA(cudaMemcpy2DAsync(in.cc, (size_t)in.ncol * 4, Q.cc, (size_t)T.pitch * 4,
                                         (size_t)in.ncol * 4, in.nrow, cudaMemcpyDeviceToDevice, s));
        ++j;
    }
    if (jo.cycles_out && nsc == 1 && ntiles == 1 && P.cyc) {
        const TileDesc &T = pl.tiles[0];
        CUPHU_TRY_CUDA(cudaMemcpy2DAsync(jo.cycles_out, (size_t)T.nc * 4, P.cyc, (size_t)T.pitch * 4,
                                         (size_t)T.nc * 4, T.nr, cudaMemcpyDeviceToDevice, s));
    }
    if (jo.cont_out && nsc == 1 && ntiles == 1 && P.cont) {
        const TileDesc &T = pl.tiles[0];
        CUPHU_TRY_CUDA(cudaMemcpy2DAsync(jo.cont_out, (size_t)T.nc * 4, P.cont, (size_t)T.pitch * 4,
                                         (size_t)T.nc * 4, T.nr, cudaMemcpyDeviceToDevice, s));
    }
    if (jo.graph) return 0;   /* the caller ends the capture */
    CUPHU_TRY_CUDA(cudaMemcpyAsync(W->status, &d_ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUPHU_TRY_CUDA(cudaEventRecord(W->done, s));
    if (stats) {
        cudaEventRecord(e3, s);
        CUPHU_TRY_CUDA(cudaEventSynchronize(e3));
        SolverCtl ctl;
        CUPHU_TRY_CUDA(cudaMemcpy(&ctl, d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
        float ms_solve = 0, ms_total = 0;
        cudaEventElapsedTime(&ms_solve, e1, e2);
        cudaEventElapsedTime(&ms_total, e0, e3);
        stats->ntiles = ntiles;
        stats->total_iters = ctl.total_iters;
        stats->max_iters_pass = ctl.max_pass_iters;
        stats->solve_ms = ms_solve;
        stats->total_ms = ms_total;
        stats->px_iters = (double)ctl.px_iters;
        if (ctl.err) return fail(CUPHU_ERR_TIMEOUT, "solver grid barrier timed out");
    }
    return cuda_fail(cudaGetLastError(), "unwrap pipeline");
}

/* default solver options, honouring the reference's environment overrides */
static void default_solve_options(CuPhuSolveOptions *o)
{
    o->precision = CUPHU_PREC_MIXED;
    o->n_irls = 16;
    o->irls_delta_max = 0.5f;
    o->irls_delta_min = 0.01f;
    o->max_iter = 1000;
    o->tol = 1e-3f;
    o->replace_every = 50;
    o->ref_row = -1;
    o->ref_col = -1;
    o->timeout_ms = 5000;
    o->device_phase = 0;
    o->merge_conncomp = 0;
    if (const char *e = std::getenv("CUPHU_N_IRLS")) o->n_irls = std::atoi(e);
    if (const char *e = std::getenv("CUPHU_IRLS_DELTA_MAX")) o->irls_delta_max = (float)std::atof(e);
    if (const char *e = std::getenv("CUPHU_IRLS_DELTA_MIN")) o->irls_delta_min = (float)std::atof(e);
    if (const char *e = std::getenv("CUPHU_LAPLACE_MAX_ITER")) o->max_iter = std::atoi(e);
    if (const char *e = std::getenv("CUPHU_LAPLACE_TOL")) o->tol = (float)std::atof(e);
}

static int check_common(CuPhuCostMode cost, const CuPhuParams *p)
{
    if (!p) return fail(CUPHU_ERR_INVALID, "params must not be NULL");
    if (cost != CUPHU_COST_SMOOTH && cost != CUPHU_COST_DEFO && cost != CUPHU_COST_TOPO)
        return fail(CUPHU_ERR_INVALID, "cost must be 'smooth', 'defo', or 'topo'");
    if (!(p->ncorrlooks >= 1.0)) return fail(CUPHU_ERR_INVALID, "nlooks must be >= 1");
    return 0;
}

static int check_tile_flags(const CuPhuTileParams *t)
{
    if (!t) return 0;
    if (t->single_tile_reoptimize)
        return fail(CUPHU_ERR_UNSUPPORTED,
                    "single_tile_reoptimize needs SNAPHU's CPU TreeSolve, which is outside this build");
    if (t->laplace_neighbor_feedback && t->laplace_neighbor_feedback_feather < 0)
        return fail(CUPHU_ERR_INVALID, "laplace_neighbor_feedback_feather must be >= 0");
    return 0;
}

static int check_bridge(const CuPhuBridgeParams *bp)
{
    if (!bp) return fail(CUPHU_ERR_INVALID, "bridge params must not be NULL");
    if (bp->radius < 0 || bp->erosion_size < 0 || bp->max_boundary_samples < 1 ||
        (int)bp->ramp_type < 0 || (int)bp->ramp_type > 6)
        return fail(CUPHU_ERR_INVALID, "bad bridge params");
    return 0;
}

/* status of the last pipeline on a device, after its work completed */
static int device_status(int dev)
{
    if (dev < 0 || dev >= 64) return 0;
    Workspace &W = g_ws[dev];
    if (!W.done) return 0;
    CUPHU_TRY_CUDA(cudaEventSynchronize(W.done));
    if (W.status && *W.status)
        return fail(CUPHU_ERR_TIMEOUT, "solver grid barrier timed out (device status set)");
    return 0;
}

/* the library's own stream on device dev, created once (threads that call
 * the host-buffer entry points at the same time share it); the legacy
 * default stream if it cannot be created */
static std::mutex g_stream_mu;
static cudaStream_t lib_stream(int dev)
{
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_stream_mu);
    Workspace &W = g_ws[dev];
    if (!W.stream) {
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess)
            W.stream = st;
        else
            cudaGetLastError();
    }
    return W.stream;
}

template <typename T>
static T *dev_alloc_async(size_t n, cudaStream_t s)
{
    T *p = nullptr;
    if (cudaMallocAsync((void **)&p, (n ? n : 1) * sizeof(T), s) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

}  // namespace cuphu

using namespace cuphu;

extern "C" {

const char *cuphu_last_error(void) { return g_err.c_str(); }

/* SNAPHU's documented defaults (snaphu.conf); the reference takes them from
 * the DEF_* macros of snaphu.h (cuphu_solver.cpp:148-216), absent here. */
void cuphu_default_params(CuPhuParams *p)
{
    std::memset(p, 0, sizeof(*p));
    p->rhosconst1 = 1.3;
    p->rhosconst2 = 0.14;
    p->cstd1 = 0.4;
    p->cstd2 = 0.35;
    p->cstd3 = 0.06;
    p->defothreshfactor = 1.2;
    p->sigsqcorr = 0.05;
    p->nlooks = 23.8;
    p->ncorrlooks = 23.8;
    p->costscale = 100.0;
    p->nshortcycle = 200.0;
    p->sigsqshortmin = 1;
    p->kperpdpsi = 7;
    p->kpardpsi = 7;
    p->defomax = 1.2;
    p->p = -1.0;
    p->maxcost = 1000.0;
    p->minconncompfrac = 0.01;
    p->conncompthresh = 300;
    p->maxncomps = 32;
}

void cuphu_default_tile_params(CuPhuTileParams *tp)
{
    std::memset(tp, 0, sizeof(*tp));
    tp->ntilerow = 1;
    tp->ntilecol = 1;
    tp->tilecostthresh = 500;
    tp->minregionsize = 100;
    tp->nproc = 1;
    tp->ngpustreams = 2;
    tp->laplace_neighbor_feedback_feather = 200;
}

void cuphu_default_bridge_params(CuPhuBridgeParams *bp)
{
    std::memset(bp, 0, sizeof(*bp));
    bp->radius = 500;
    bp->min_num_pixel = 14;
    bp->erosion_size = 2;
    bp->max_boundary_samples = 4096;
    bp->ramp_type = CUPHU_RAMP_NONE;
    bp->ramp_max_num_sample = 1000000;
}

void cuphu_default_solve_options(CuPhuSolveOptions *o) { default_solve_options(o); }

int cuphu_unwrap_device(const float *igram_c64, const float *phase_in, const float *corr,
                        const unsigned char *mask, const unsigned char *orig_mask, int nrow,
                        int ncol, CuPhuCostMode cost_mode, const CuPhuParams *params,
                        const CuPhuTileParams *tile, const CuPhuSolveOptions *opts,
                        float *unw_out, uint32_t *conncomp_out, int32_t *cycles_out,
                        CuPhuSolveStats *stats, void *stream)
{
    int rc = check_common(cost_mode, params);
    if (rc) return rc;
    if ((rc = check_tile_flags(tile))) return rc;
    if ((!igram_c64 && !phase_in) || !corr || !unw_out)
        return fail(CUPHU_ERR_INVALID, "igram (or phase), corr and unw must not be NULL");
    CuPhuSolveOptions so;
    if (opts) so = *opts; else default_solve_options(&so);
    SceneIn in;
    in.ig = reinterpret_cast<const float2 *>(igram_c64);
    in.ph_in = igram_c64 ? nullptr : phase_in;
    in.corr = corr;
    in.mask = mask;
    in.conf = orig_mask;
    in.nrow = nrow;
    in.ncol = ncol;
    if (tile) {
        in.ntr = tile->ntilerow; in.ntc = tile->ntilecol;
        in.rovl = tile->rowovrlp; in.covl = tile->colovrlp;
        in.feedback = tile->laplace_neighbor_feedback ? 1 : 0;
        in.feather = tile->laplace_neighbor_feedback_feather;
        in.spikes = tile->fix_cycle_spikes ? 1 : 0;
    }
    in.nlooks = params->ncorrlooks;
    in.unw = unw_out;
    in.cc = conncomp_out;
    in.ref_row = so.ref_row;
    in.ref_col = so.ref_col;
    in.merge_cc = so.merge_conncomp ? 1 : 0;
    std::vector<SceneIn> S(1, in);
    JobOpts jo;
    jo.fp64 = so.precision == CUPHU_PREC_FP64;
    jo.so = so;
    jo.want_cc = conncomp_out != nullptr;
    jo.want_cyc = cycles_out != nullptr && in.ntr == 1 && in.ntc == 1;
    jo.cycles_out = cycles_out;
    return run_job(S, *params, jo, (cudaStream_t)stream, stats);
}

static int batch_scenes(const CuPhuScene *scenes, int nscenes, CuPhuCostMode cost_mode,
                        const CuPhuParams *params, const CuPhuSolveOptions *opts,
                        std::vector<SceneIn> &S, JobOpts &jo)
{
    int rc = check_common(cost_mode, params);
    if (rc) return rc;
    if (!scenes || nscenes < 1) return fail(CUPHU_ERR_INVALID, "no scenes");
    CuPhuSolveOptions so;
    if (opts) so = *opts; else default_solve_options(&so);
    S.assign(nscenes, SceneIn());
    for (int i = 0; i < nscenes; ++i) {
        const CuPhuScene &c = scenes[i];
        if ((!c.igram_c64 && !c.phase) || !c.corr || !c.unw_out)
            return fail(CUPHU_ERR_INVALID, "scene igram/phase, corr and unw must not be NULL");
        if (!(c.nlooks >= 1.0)) return fail(CUPHU_ERR_INVALID, "nlooks must be >= 1");
        SceneIn &in = S[i];
        in.ig = reinterpret_cast<const float2 *>(c.igram_c64);
        in.ph_in = c.igram_c64 ? nullptr : c.phase;
        in.corr = c.corr;
        in.mask = c.mask;
        in.conf = c.orig_mask;
        in.nrow = c.nrow; in.ncol = c.ncol;
        in.ntr = c.ntilerow; in.ntc = c.ntilecol;
        in.rovl = c.rowovrlp; in.covl = c.colovrlp;
        in.nlooks = c.nlooks;
        in.unw = c.unw_out;
        in.cc = c.conncomp_out;
        in.ref_row = so.ref_row;
        in.ref_col = so.ref_col;
    }
    jo.fp64 = so.precision == CUPHU_PREC_FP64;
    jo.so = so;
    bool cc = true;
    for (auto &in : S) cc = cc && in.cc;
    jo.want_cc = cc;
    return 0;
}

int cuphu_unwrap_batch_device(const CuPhuScene *scenes, int nscenes, CuPhuCostMode cost_mode,
                              const CuPhuParams *params, const CuPhuSolveOptions *opts,
                              CuPhuSolveStats *stats, void *stream)
{
    std::vector<SceneIn> S;
    JobOpts jo;
    int rc = batch_scenes(scenes, nscenes, cost_mode, params, opts, S, jo);
    if (rc) return rc;
    return run_job(S, *params, jo, (cudaStream_t)stream, stats);
}

int cuphu_batch_graph_create(const CuPhuScene *scenes, int nscenes, CuPhuCostMode cost_mode,
                             const CuPhuParams *params, const CuPhuSolveOptions *opts,
                             void **graph_out)
{
    if (!graph_out) return fail(CUPHU_ERR_INVALID, "graph_out must not be NULL");
    *graph_out = nullptr;
    std::vector<SceneIn> S;
    JobOpts jo;
    int rc = batch_scenes(scenes, nscenes, cost_mode, params, opts, S, jo);
    if (rc) return rc;
    auto *G = new GraphJob();
    CUPHU_TRY_CUDA(cudaGetDevice(&G->dev));
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        delete G;
        return fail(CUPHU_ERR_CUDA, "stream creation failed");
    }
    jo.graph = G;
    rc = run_job(S, *params, jo, s, nullptr);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    cudaGraph_t g = nullptr;
    if (cs != cudaStreamCaptureStatusNone) {
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture");
    }
    if (!rc) {
        cudaError_t e = cudaGraphInstantiate(&G->exec, g, 0);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphInstantiate");
    }
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(s);
    if (rc) {
        if (G->exec) cudaGraphExecDestroy(G->exec);
        ws_free(G->ws);
        delete G;
        return rc;
    }
    *graph_out = G;
    return 0;
}

int cuphu_batch_graph_launch(void *graph, void *stream)
{
    auto *G = static_cast<GraphJob *>(graph);
    if (!G || !G->exec) return fail(CUPHU_ERR_INVALID, "not a graph from cuphu_batch_graph_create");
    CUPHU_TRY_CUDA(cudaGraphLaunch(G->exec, (cudaStream_t)stream));
    return 0;
}

int cuphu_batch_graph_destroy(void *graph)
{
    auto *G = static_cast<GraphJob *>(graph);
    if (!G) return 0;
    CUPHU_TRY_CUDA(cudaDeviceSynchronize());
    if (G->exec) cudaGraphExecDestroy(G->exec);
    ws_free(G->ws);
    delete G;
    return 0;
}

int cuphu_autotune(const float *igram_c64, const float *corr, int nrow, int ncol,
                   CuPhuCostMode cost_mode, const CuPhuParams *params,
                   const CuPhuTileParams *tile, int gpu_id, int *choices)
{
    int rc = check_common(cost_mode, params);
    if (rc) return rc;
    if (!igram_c64 || !corr || nrow < 2 || ncol < 2)
        return fail(CUPHU_ERR_INVALID, "igram and corr of at least 2x2 pixels are required");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    cudaStream_t s = lib_stream(gpu_id);
    const size_t n = (size_t)nrow * ncol;
    const size_t narcs = (size_t)(nrow - 1) * ncol + (size_t)nrow * (ncol - 1);
    const int es = cost_mode == CUPHU_COST_SMOOTH ? 2 : 4;
    float *d_ig = dev_alloc_async<float>(2 * n, s), *d_corr = dev_alloc_async<float>(n, s);
    float *d_ph = dev_alloc_async<float>(n, s), *d_unw = dev_alloc_async<float>(n, s);
    short *d_cost = dev_alloc_async<short>(narcs * es, s);
    if (!d_ig || !d_corr || !d_ph || !d_unw || !d_cost) rc = fail(CUPHU_ERR_ALLOC, "device allocation failed");
    Timers tm(rc ? 0 : 2);
    cudaEvent_t e0 = tm.e[0], e1 = tm.e[1];
    int best_cost = 0, best_shape = 0;
    if (!rc) {
        rc = copy_async(d_ig, igram_c64, 8 * n, cudaMemcpyHostToDevice, s, "H2D igram");
        if (!rc) rc = copy_async(d_corr, corr, 4 * n, cudaMemcpyHostToDevice, s, "H2D corr");
        if (!rc) rc = launch_phase(reinterpret_cast<const float2 *>(d_ig), d_ph, (long long)n, s);
    }
    /* cost kernel: 3 or 4 blocks per SM (identical results) */
    float best_ms = 1e30f;
    for (int v = 0; v < 2 && !rc; ++v) {
        tune_force(0, v);
        for (int rep = 0; rep < 2 && !rc; ++rep) {
            cudaEventRecord(e0, s);
            for (int k = 0; k < 3 && !rc; ++k)
                rc = launch_costs(d_ph, d_corr, nullptr, nrow, ncol,
                                  cost_mode == CUPHU_COST_SMOOTH ? 0 : 1, *params, d_cost,
                                  nullptr, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best_cost = v; }
    }
    tune_force(0, -1);
    if (!rc) tune_set(gpu_id, 0, 2LL * nrow * ncol, best_cost);
    /* persistent solver: each launch shape (ring stages x blocks per SM) of
     * the default precision, 20 PCG iterations, no IRLS */
    best_ms = 1e30f;
    long long items = 0;
    CuPhuSolveOptions so0;
    default_solve_options(&so0);
    const bool fp64 = so0.precision == CUPHU_PREC_FP64;
    const int kind = fp64 ? 2 : 1;
    const int nshape = solve_shape_count(fp64);
    for (int v = 0; v < nshape && !rc; ++v) {
        tune_force(kind, v);
        CuPhuSolveOptions so = so0;
        so.max_iter = 20;
        so.n_irls = 0;
        so.ref_row = so.ref_col = -1;
        CuPhuSolveStats st = {};
        for (int rep = 0; rep < 2 && !rc; ++rep)
            rc = cuphu_unwrap_device(nullptr, d_ph, d_corr, nullptr, nullptr, nrow, ncol, cost_mode,
                                     params, tile, &so, d_unw, nullptr, nullptr, &st, s);
        items = tune_probe_items();
        if (!rc && st.solve_ms < best_ms) { best_ms = (float)st.solve_ms; best_shape = v; }
    }
    tune_force(kind, -1);
    if (!rc && items > 0) tune_set(gpu_id, kind, items, best_shape);
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_ig, s); cudaFreeAsync(d_corr, s); cudaFreeAsync(d_ph, s);
    cudaFreeAsync(d_unw, s); cudaFreeAsync(d_cost, s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cuphu_autotune");
    if (!rc && choices) { choices[0] = best_cost; choices[1] = best_shape; }
    return rc;
}

int cuphu_unwrap_ex(const float *igram_c64, const float *corr, const unsigned char *mask,
                    const unsigned char *orig_mask, int nrow, int ncol, CuPhuCostMode cost_mode,
                    const CuPhuParams *params, const CuPhuTileParams *tile,
                    const CuPhuSolveOptions *opts, int gpu_id, float *unw_out,
                    uint32_t *conncomp_out, CuPhuSolveStats *stats)
{
    if (!igram_c64 || !corr || !unw_out || !conncomp_out)
        return fail(CUPHU_ERR_INVALID, "igram, corr, unw and conncomp must not be NULL");
    if (nrow < 1 || ncol < 1) return fail(CUPHU_ERR_INVALID, "nrow and ncol must be >= 1");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    cudaStream_t s = lib_stream(gpu_id);
    size_t n = (size_t)nrow * ncol;
    /* the wrapped phase: the reference's host atan2 (default), or the
     * interferogram itself for the device's phase kernel */
    const bool dev_phase = opts && opts->device_phase;
    float *d_ig = dev_alloc_async<float>(dev_phase ? 2 * n : n, s), *d_corr = dev_alloc_async<float>(n, s);
    float *d_unw = dev_alloc_async<float>(n, s);
    uint32_t *d_cc = dev_alloc_async<uint32_t>(n, s);
    unsigned char *d_mask = mask ? dev_alloc_async<unsigned char>(n, s) : nullptr;
    unsigned char *d_om = orig_mask ? dev_alloc_async<unsigned char>(n, s) : nullptr;
    int rc = 0;
    if (!d_ig || !d_corr || !d_unw || !d_cc || (mask && !d_mask) || (orig_mask && !d_om))
        rc = fail(CUPHU_ERR_ALLOC, "device allocation failed");
    if (!rc) {
        rc = dev_phase ? copy_async(d_ig, igram_c64, 8 * n, cudaMemcpyHostToDevice, s, "H2D igram")
                       : upload_host_phase(igram_c64, nullptr, nullptr, n, d_ig, gpu_id, s);
        if (!rc) rc = copy_async(d_corr, corr, 4 * n, cudaMemcpyHostToDevice, s, "H2D corr");
        if (!rc && mask) rc = copy_async(d_mask, mask, n, cudaMemcpyHostToDevice, s, "H2D mask");
        if (!rc && orig_mask)
            rc = copy_async(d_om, orig_mask, n, cudaMemcpyHostToDevice, s, "H2D orig_mask");
    }
    if (!rc) {
        rc = cuphu_unwrap_device(dev_phase ? d_ig : nullptr, dev_phase ? nullptr : d_ig, d_corr,
                                 d_mask, d_om, nrow, ncol, cost_mode, params, tile, opts, d_unw,
                                 d_cc, nullptr, stats, s);
    }
    if (!rc) rc = copy_async(unw_out, d_unw, 4 * n, cudaMemcpyDeviceToHost, s, "D2H unw");
    if (!rc) rc = copy_async(conncomp_out, d_cc, 4 * n, cudaMemcpyDeviceToHost, s, "D2H conncomp");
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_ig, s); cudaFreeAsync(d_corr, s); cudaFreeAsync(d_unw, s); cudaFreeAsync(d_cc, s);
    if (d_mask) cudaFreeAsync(d_mask, s);
    if (d_om) cudaFreeAsync(d_om, s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cuphu_unwrap_ex");
    if (!rc) rc = device_status(gpu_id);
    return rc;
}

int cuphu_unwrap(const float *igram_r, const float *igram_i, const float *corr, const float *mag,
                 const unsigned char *mask, int nrow, int ncol, CuPhuCostMode cost_mode,
                 CuPhuInitMethod init_meth, const CuPhuParams *params,
                 const CuPhuTileParams *tile, const CuPhuBridgeParams *bridge,
                 const unsigned char *orig_mask, int gpu_id, CuPhuResult *result)
{
    (void)mag;
    if (!result) return fail(CUPHU_ERR_INVALID, "result must not be NULL");
    result->unw = nullptr;
    result->conncomp = nullptr;
    result->nrow = nrow;
    result->ncol = ncol;
    if (init_meth != CUPHU_INIT_LAPLACE)
        return fail(CUPHU_ERR_UNSUPPORTED,
                    "init 'mst'/'mcf' needs SNAPHU's CPU network-flow solver, which is outside this "
                    "build; use init 'laplace'");
    if (bridge && bridge->enabled) {
        int rb = check_bridge(bridge);
        if (rb) return rb;
    }
    if (!igram_r || !igram_i || !corr) return fail(CUPHU_ERR_INVALID, "igram and corr must not be NULL");
    if (nrow < 1 || ncol < 1) return fail(CUPHU_ERR_INVALID, "nrow and ncol must be >= 1");
    int rc = check_common(cost_mode, params);
    if (rc) return rc;
    if ((rc = check_tile_flags(tile))) return rc;
    size_t n = (size_t)nrow * ncol;
    result->unw = (float *)std::malloc(n * sizeof(float));
    result->conncomp = (uint32_t *)std::malloc(n * sizeof(uint32_t));
    if (!result->unw || !result->conncomp) {
        std::free(result->unw);
        std::free(result->conncomp);
        result->unw = nullptr;
        result->conncomp = nullptr;
        return fail(CUPHU_ERR_ALLOC, "host allocation failed");
    }
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    cudaStream_t s = lib_stream(gpu_id);
    float *d_corr = dev_alloc_async<float>(n, s), *d_unw = dev_alloc_async<float>(n, s);
    float *d_ph = dev_alloc_async<float>(n, s);
    uint32_t *d_cc = dev_alloc_async<uint32_t>(n, s);
    unsigned char *d_mask = mask ? dev_alloc_async<unsigned char>(n, s) : nullptr;
    unsigned char *d_om = orig_mask ? dev_alloc_async<unsigned char>(n, s) : nullptr;
    if (!d_corr || !d_unw || !d_ph || !d_cc || (mask && !d_mask) || (orig_mask && !d_om))
        rc = fail(CUPHU_ERR_ALLOC, "device allocation failed");
    if (!rc) {
        /* the phase as the reference takes it: host atan2 (cuphu_solver.cpp:1706-1712) */
        rc = upload_host_phase(nullptr, igram_r, igram_i, n, d_ph, gpu_id, s);
        if (!rc) rc = copy_async(d_corr, corr, 4 * n, cudaMemcpyHostToDevice, s, "H2D corr");
        if (!rc && mask) rc = copy_async(d_mask, mask, n, cudaMemcpyHostToDevice, s, "H2D mask");
        if (!rc && orig_mask)
            rc = copy_async(d_om, orig_mask, n, cudaMemcpyHostToDevice, s, "H2D orig_mask");
    }
    if (!rc) {
        CuPhuSolveOptions so;
        default_solve_options(&so);
        CuPhuParams p = *params;
        rc = cuphu_unwrap_device(nullptr, d_ph, d_corr, d_mask, d_om, nrow, ncol, cost_mode, &p,
                                 tile, &so, d_unw, d_cc, nullptr, nullptr, s);
        /* the reference's last stage: bridging over the solve mask
         * (cuphu_solver.cpp:1720-1722, 2097-2098) */
        if (!rc && bridge && bridge->enabled)
            rc = run_bridge(d_unw, d_cc, d_mask, nrow, ncol, *bridge, s);
    }
    if (!rc) rc = copy_async(result->unw, d_unw, 4 * n, cudaMemcpyDeviceToHost, s, "D2H unw");
    if (!rc)
        rc = copy_async(result->conncomp, d_cc, 4 * n, cudaMemcpyDeviceToHost, s, "D2H conncomp");
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_corr, s);
    cudaFreeAsync(d_unw, s); cudaFreeAsync(d_ph, s); cudaFreeAsync(d_cc, s);
    if (d_mask) cudaFreeAsync(d_mask, s);
    if (d_om) cudaFreeAsync(d_om, s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cuphu_unwrap");
    if (!rc) rc = device_status(gpu_id);
    return rc;
}

/* ── phase bridging (ref cuphu_solver.cpp:996-1352) ───────────────────── */
int cuphu_bridge_device(float *d_unw, uint32_t *d_conncomp, const unsigned char *d_mask, int nrow,
                        int ncol, const CuPhuBridgeParams *bp, void *stream)
{
    int rc = check_bridge(bp);
    if (rc) return rc;
    if (!d_unw || !d_conncomp || nrow < 1 || ncol < 1) return fail(CUPHU_ERR_INVALID, "bad arguments");
    return run_bridge(d_unw, d_conncomp, d_mask, nrow, ncol, *bp, (cudaStream_t)stream);
}

int cuphu_bridge_apply_test(float *unw, uint32_t *conncomp, int nrow, int ncol,
                            const CuPhuBridgeParams *bridge, const unsigned char *mask, int gpu_id)
{
    int rc = check_bridge(bridge);
    if (rc) return rc;
    if (!unw || !conncomp || nrow < 1 || ncol < 1) return fail(CUPHU_ERR_INVALID, "bad arguments");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    cudaStream_t s = lib_stream(gpu_id);
    const size_t n = (size_t)nrow * ncol;
    float *d_u = dev_alloc_async<float>(n, s);
    uint32_t *d_c = dev_alloc_async<uint32_t>(n, s);
    unsigned char *d_m = mask ? dev_alloc_async<unsigned char>(n, s) : nullptr;
    if (!d_u || !d_c || (mask && !d_m)) rc = fail(CUPHU_ERR_ALLOC, "device allocation failed");
    if (!rc) rc = copy_async(d_u, unw, 4 * n, cudaMemcpyHostToDevice, s, "H2D unw");
    if (!rc) rc = copy_async(d_c, conncomp, 4 * n, cudaMemcpyHostToDevice, s, "H2D conncomp");
    if (!rc && mask) rc = copy_async(d_m, mask, n, cudaMemcpyHostToDevice, s, "H2D mask");
    if (!rc) rc = run_bridge(d_u, d_c, d_m, nrow, ncol, *bridge, s);
    if (!rc) rc = copy_async(unw, d_u, 4 * n, cudaMemcpyDeviceToHost, s, "D2H unw");
    if (!rc) rc = copy_async(conncomp, d_c, 4 * n, cudaMemcpyDeviceToHost, s, "D2H conncomp");
    cudaError_t e = cudaStreamSynchronize(s);
    for (void *p : {(void *)d_u, (void *)d_c, (void *)d_m})
        if (p) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "bridging");
    return rc;
}

/* ── failure test of the bounded device waits ─────────────────────────── */
int cuphu_test_skip_barrier_once(int gpu_id, int block)
{
    if (gpu_id < 0 || gpu_id >= 64 || block < 0)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    solver_skip_barrier_once(gpu_id, block);
    return 0;
}

int cuphu_test_force_solve_shape(int shape)
{
    if (shape < -1 || shape >= std::max(solve_shape_count(false), solve_shape_count(true)))
        return fail(CUPHU_ERR_INVALID, "no such solver launch shape");
    tune_force(1, shape);
    tune_force(2, shape);
    return 0;
}

/* ── inputs of the CPU network-flow front end, computed on the GPU ─────── */
int cuphu_mst_costs_device(const void *d_smooth_costs, long long narcs, long nshortcycle,
                           long maxcost, short *d_out, void *stream)
{
    if (!d_smooth_costs || !d_out || narcs < 0 || nshortcycle < 1 || maxcost < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    return launch_mst_costs(static_cast<const short *>(d_smooth_costs), narcs, nshortcycle,
                            maxcost, d_out, (cudaStream_t)stream);
}

int cuphu_mcf_inputs(const float *igram_r, const float *igram_i, const float *corr,
                     const short *weights, int nrow, int ncol, CuPhuCostMode cost_mode,
                     const CuPhuParams *params, int gpu_id, short *costs_out,
                     short *mst_costs_out, signed char *residues_out)
{
    int rc = check_common(cost_mode, params);
    if (rc) return rc;
    if (!igram_r || !igram_i || !corr || !costs_out || nrow < 2 || ncol < 2)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    if (mst_costs_out && cost_mode != CUPHU_COST_SMOOTH)
        return fail(CUPHU_ERR_UNSUPPORTED,
                    "initial-flow weights of DEFO/TOPO costs need SNAPHU's CalcCostDefo, which "
                    "is outside this build");
    if (mst_costs_out && !(params->maxcost >= 1.0))
        return fail(CUPHU_ERR_INVALID, "params->maxcost must be >= 1");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    cudaStream_t s = lib_stream(gpu_id);
    const size_t n = (size_t)nrow * ncol;
    const size_t narcs = (size_t)(nrow - 1) * ncol + (size_t)nrow * (ncol - 1);
    const size_t es = cost_mode == CUPHU_COST_SMOOTH ? 4 : 8;
    const size_t nres = (size_t)(nrow - 1) * (ncol - 1);
    float *d_ph = dev_alloc_async<float>(n, s), *d_corr = dev_alloc_async<float>(n, s);
    short *d_w = weights ? dev_alloc_async<short>(narcs, s) : nullptr;
    char *d_c = dev_alloc_async<char>(narcs * es + 8, s);
    short *d_mst = mst_costs_out ? dev_alloc_async<short>(narcs, s) : nullptr;
    signed char *d_res = residues_out ? dev_alloc_async<signed char>(nres, s) : nullptr;
    if (!d_ph || !d_corr || !d_c || (weights && !d_w) || (mst_costs_out && !d_mst) ||
        (residues_out && !d_res))
        rc = fail(CUPHU_ERR_ALLOC, "device allocation failed");
    if (!rc) rc = upload_host_phase(nullptr, igram_r, igram_i, n, d_ph, gpu_id, s);
    if (!rc) rc = copy_async(d_corr, corr, 4 * n, cudaMemcpyHostToDevice, s, "H2D corr");
    if (!rc && weights)
        rc = copy_async(d_w, weights, 2 * narcs, cudaMemcpyHostToDevice, s, "H2D weights");
    if (!rc)
        rc = launch_costs(d_ph, d_corr, d_w, nrow, ncol, cost_mode == CUPHU_COST_SMOOTH ? 0 : 1,
                          *params, d_c, d_res, s);
    if (!rc && d_mst)
        rc = launch_mst_costs(reinterpret_cast<const short *>(d_c), (long long)narcs,
                              (long)params->nshortcycle, (long)params->maxcost, d_mst, s);
    if (!rc) rc = copy_async(costs_out, d_c, narcs * es, cudaMemcpyDeviceToHost, s, "D2H costs");
    if (!rc && d_mst)
        rc = copy_async(mst_costs_out, d_mst, narcs * 2, cudaMemcpyDeviceToHost, s, "D2H mst");
    if (!rc && d_res)
        rc = copy_async(residues_out, d_res, nres, cudaMemcpyDeviceToHost, s, "D2H residues");
    cudaError_t e = cudaStreamSynchronize(s);
    for (void *p : {(void *)d_ph, (void *)d_corr, (void *)d_w, (void *)d_c, (void *)d_mst,
                    (void *)d_res})
        if (p) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cuphu_mcf_inputs");
    return rc;
}

/* ── post-passes on a stitched scene ─────────────────────────────────── */
static int postpass_device(int which, float *unw, const unsigned char *mask, int nrow, int ncol,
                           int ntr, int ntc, int rovl, int covl, int feather, cudaStream_t s)
{
    if (!unw || nrow < 1 || ncol < 1) return fail(CUPHU_ERR_INVALID, "bad arguments");
    if (which == 1 && (ntr < 1 || ntc < 1 || rovl < 0 || covl < 0))
        return fail(CUPHU_ERR_INVALID, "tile counts must be >= 1 and overlaps >= 0");
    char *scratch = dev_alloc_async<char>(postpass_scratch_bytes(nrow, ncol), s);
    if (!scratch) return fail(CUPHU_ERR_ALLOC, "device allocation failed");
    int rc = which == 0 ? launch_fix_cycle_spikes(unw, mask, nrow, ncol, scratch, s)
                        : launch_neighbor_feedback(unw, mask, nrow, ncol, ntr, ntc, rovl, covl,
                                                   feather, scratch, s);
    cudaFreeAsync(scratch, s);
    return rc;
}

static int postpass_host(int which, float *unw, const unsigned char *mask, int nrow, int ncol,
                         int ntr, int ntc, int rovl, int covl, int feather)
{
    if (!unw || nrow < 1 || ncol < 1) return fail(CUPHU_ERR_INVALID, "bad arguments");
    int dev = 0;
    CUPHU_TRY_CUDA(cudaGetDevice(&dev));
    cudaStream_t s = lib_stream(dev);
    const size_t n = (size_t)nrow * ncol;
    float *d_u = dev_alloc_async<float>(n, s);
    unsigned char *d_m = mask ? dev_alloc_async<unsigned char>(n, s) : nullptr;
    int rc = (!d_u || (mask && !d_m)) ? fail(CUPHU_ERR_ALLOC, "device allocation failed") : 0;
    if (!rc) rc = copy_async(d_u, unw, 4 * n, cudaMemcpyHostToDevice, s, "H2D unw");
    if (!rc && mask) rc = copy_async(d_m, mask, n, cudaMemcpyHostToDevice, s, "H2D mask");
    if (!rc) rc = postpass_device(which, d_u, d_m, nrow, ncol, ntr, ntc, rovl, covl, feather, s);
    if (!rc) rc = copy_async(unw, d_u, 4 * n, cudaMemcpyDeviceToHost, s, "D2H unw");
    cudaError_t e = cudaStreamSynchronize(s);
    if (d_u) cudaFreeAsync(d_u, s);
    if (d_m) cudaFreeAsync(d_m, s);
    cudaStreamSynchronize(s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "post-pass");
    return rc;
}

int cuphu_fix_cycle_spikes_device(float *d_unw, const unsigned char *d_mask, int nrow, int ncol,
                                  void *stream)
{
    return postpass_device(0, d_unw, d_mask, nrow, ncol, 1, 1, 0, 0, 0, (cudaStream_t)stream);
}

int cuphu_laplace_neighbor_feedback_device(float *d_unw, const unsigned char *d_mask, int nrow,
                                           int ncol, int ntr, int ntc, int row_ovrlp,
                                           int col_ovrlp, int feather_px, void *stream)
{
    return postpass_device(1, d_unw, d_mask, nrow, ncol, ntr, ntc, row_ovrlp, col_ovrlp,
                           feather_px, (cudaStream_t)stream);
}

int cuphu_fix_cycle_spikes_test(float *unw, const unsigned char *mask, int nrow, int ncol)
{
    return postpass_host(0, unw, mask, nrow, ncol, 1, 1, 0, 0, 0);
}

int cuphu_laplace_neighbor_feedback_test(float *unw, const unsigned char *mask, int nrow, int ncol,
                                         int ntr, int ntc, int row_ovrlp, int col_ovrlp,
                                         int feather_px)
{
    return postpass_host(1, unw, mask, nrow, ncol, ntr, ntc, row_ovrlp, col_ovrlp, feather_px);
}

int cuphu_phase_gpu(const float *d_igram_c64, long long n, float *d_phase, void *stream)
{
    if (!d_igram_c64 || !d_phase || n < 0) return fail(CUPHU_ERR_INVALID, "bad arguments");
    return launch_phase(reinterpret_cast<const float2 *>(d_igram_c64), d_phase, n,
                        (cudaStream_t)stream);
}

int cuphu_residues_gpu(const float *d_phase, int nrow, int ncol, signed char *d_res, void *stream)
{
    if (!d_phase || !d_res || nrow < 1 || ncol < 1) return fail(CUPHU_ERR_INVALID, "bad arguments");
    return launch_residues(d_phase, nrow, ncol, d_res, (cudaStream_t)stream);
}

int cuphu_build_costs_device(const float *d_phase, const float *d_corr, const short *d_weights,
                             int nrow, int ncol, int mode, const CuPhuParams *params,
                             void *d_costs, signed char *d_residues, void *stream)
{
    int rc = check_common((CuPhuCostMode)mode, params);
    if (rc) return rc;
    if (!d_phase || !d_corr || !d_costs || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    return launch_costs(d_phase, d_corr, d_weights, nrow, ncol, mode, *params, d_costs, d_residues,
                        (cudaStream_t)stream);
}

static int build_costs_launcher(const float *d_phase, const float *d_corr, const short *d_roww,
                                const short *d_colw, int nrow, int ncol, const CuPhuParams *params,
                                int kperp, int kpar, void **d_costs_out, void *stream, int mode)
{
    if (!d_costs_out) return fail(CUPHU_ERR_INVALID, "d_costs_out must not be NULL");
    *d_costs_out = nullptr;
    if (!params || !d_phase || !d_corr || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    if ((d_roww == nullptr) != (d_colw == nullptr))
        return fail(CUPHU_ERR_INVALID, "row and column weights must both be given or both NULL");
    cudaStream_t s = (cudaStream_t)stream;
    size_t nra = (size_t)(nrow - 1) * ncol, nca = (size_t)nrow * (ncol - 1);
    size_t es = mode ? 8 : 4;
    void *out = nullptr;
    CUPHU_TRY_CUDA(cudaMallocAsync(&out, (nra + nca) * es + 8, s));
    short *w = nullptr;
    if (d_roww) {
        /* the launcher interface passes two weight arrays; the kernel reads
         * one flat array, so gather them once */
        CUPHU_TRY_CUDA(cudaMallocAsync((void **)&w, (nra + nca) * sizeof(short) + 8, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(w, d_roww, nra * sizeof(short), cudaMemcpyDeviceToDevice, s));
        CUPHU_TRY_CUDA(cudaMemcpyAsync(w + nra, d_colw, nca * sizeof(short), cudaMemcpyDeviceToDevice, s));
    }
    CuPhuParams p = *params;
    p.kperpdpsi = kperp;
    p.kpardpsi = kpar;
    int rc = launch_costs(d_phase, d_corr, w, nrow, ncol, mode, p, out, nullptr, s);
    if (w) cudaFreeAsync(w, s);
    if (rc) {
        cudaFreeAsync(out, s);
        return rc;
    }
    *d_costs_out = out;
    return 0;
}

int cuphu_build_smooth_costs_gpu(const float *d_phase, const float *d_corr, const short *d_roww,
                                 const short *d_colw, int nrow, int ncol,
                                 const CuPhuParams *params, int kperpdpsi, int kpardpsi,
                                 void **d_costs_out, void *stream)
{
    return build_costs_launcher(d_phase, d_corr, d_roww, d_colw, nrow, ncol, params, kperpdpsi,
                                kpardpsi, d_costs_out, stream, 0);
}

int cuphu_build_defo_costs_gpu(const float *d_phase, const float *d_corr, const short *d_roww,
                               const short *d_colw, int nrow, int ncol, const CuPhuParams *params,
                               int kperpdpsi, int kpardpsi, void **d_costs_out, void *stream)
{
    return build_costs_launcher(d_phase, d_corr, d_roww, d_colw, nrow, ncol, params, kperpdpsi,
                                kpardpsi, d_costs_out, stream, 1);
}

int cuphu_build_costs_gpu(const float *igram_r, const float *igram_i, const float *corr,
                          const float *mag, const short *weights, int nrow, int ncol,
                          CuPhuCostMode cost_mode, const CuPhuParams *params, int gpu_id,
                          void **costs_out, size_t *cost_elem_sz)
{
    (void)mag;
    if (!costs_out || !cost_elem_sz) return fail(CUPHU_ERR_INVALID, "output pointers must not be NULL");
    *costs_out = nullptr;
    *cost_elem_sz = 0;
    int rc = check_common(cost_mode, params);
    if (rc) return rc;
    if (!igram_r || !igram_i || !corr || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    cudaStream_t s = lib_stream(gpu_id);
    size_t n = (size_t)nrow * ncol;
    size_t narcs = (size_t)(nrow - 1) * ncol + (size_t)nrow * (ncol - 1);
    size_t es = cost_mode == CUPHU_COST_SMOOTH ? 4 : 8;
    float *d_corr = dev_alloc_async<float>(n, s), *d_ph = dev_alloc_async<float>(n, s);
    short *d_w = weights ? dev_alloc_async<short>(narcs, s) : nullptr;
    char *d_c = dev_alloc_async<char>(narcs * es + 8, s);
    void *h = std::malloc(narcs * es + 8);
    if (!d_corr || !d_ph || !d_c || (weights && !d_w) || !h)
        rc = fail(CUPHU_ERR_ALLOC, "allocation failed");
    if (!rc) {
        /* the phase as the reference takes it: host atan2 (cuphu_solver.cpp:2120-2126) */
        rc = upload_host_phase(nullptr, igram_r, igram_i, n, d_ph, gpu_id, s);
        if (!rc) rc = copy_async(d_corr, corr, 4 * n, cudaMemcpyHostToDevice, s, "H2D corr");
        if (!rc && weights)
            rc = copy_async(d_w, weights, 2 * narcs, cudaMemcpyHostToDevice, s, "H2D weights");
    }
    if (!rc)
        rc = launch_costs(d_ph, d_corr, d_w, nrow, ncol, cost_mode == CUPHU_COST_SMOOTH ? 0 : 1,
                          *params, d_c, nullptr, s);
    if (!rc) rc = copy_async(h, d_c, narcs * es, cudaMemcpyDeviceToHost, s, "D2H costs");
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_corr, s);
    cudaFreeAsync(d_ph, s); cudaFreeAsync(d_c, s);
    if (d_w) cudaFreeAsync(d_w, s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cuphu_build_costs_gpu");
    if (rc) {
        std::free(h);
        return rc;
    }
    *costs_out = h;
    *cost_elem_sz = es;
    return (int)es;
}

int cuphu_laplace_solve_device(const void *d_costs, int cost_stride_shorts, const float *d_phase,
                               int nrow, int ncol, const CuPhuSolveOptions *opts, float *d_unw,
                               int32_t *d_cycles, float *d_cont, CuPhuSolveStats *stats,
                               void *stream)
{
    if (!d_costs || !d_phase || !d_unw || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    if (cost_stride_shorts != 2 && cost_stride_shorts != 4)
        return fail(CUPHU_ERR_INVALID, "cost stride must be 2 (smooth) or 4 (defo) shorts");
    CuPhuParams p;
    cuphu_default_params(&p);
    CuPhuSolveOptions so;
    if (opts) so = *opts; else default_solve_options(&so);
    SceneIn in;
    in.ph_in = d_phase;
    in.corr = d_phase;   /* not read: weights come from the cost array */
    in.nrow = nrow;
    in.ncol = ncol;
    in.unw = d_unw;
    in.nlooks = p.ncorrlooks;
    in.ref_row = so.ref_row;
    in.ref_col = so.ref_col;
    std::vector<SceneIn> S(1, in);
    JobOpts jo;
    jo.fp64 = so.precision == CUPHU_PREC_FP64;
    jo.so = so;
    jo.want_cc = false;
    jo.want_cyc = d_cycles != nullptr;
    jo.cycles_out = d_cycles;
    jo.costs = (const short *)d_costs;
    jo.cost_stride = cost_stride_shorts;
    jo.cont_out = d_cont;
    return run_job(S, p, jo, (cudaStream_t)stream, stats);
}

int cuphu_wls_solve_device(const float *d_gd, const float *d_gr, const float *d_rhs,
                           const float *d_wd, const float *d_wr, const double *d_u0, int nrow,
                           int ncol, const CuPhuSolveOptions *opts, double *d_u,
                           CuPhuSolveStats *stats, void *stream)
{
    if (!d_wd || !d_wr || !d_u || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    const bool have_g = d_gd != nullptr || d_gr != nullptr;
    if (have_g == (d_rhs != nullptr))
        return fail(CUPHU_ERR_INVALID, "give either the arc targets (gd, gr) or a right-hand side");
    if (have_g && (!d_gd || !d_gr))
        return fail(CUPHU_ERR_INVALID, "gd and gr are both required");
    CuPhuParams p;
    cuphu_default_params(&p);
    CuPhuSolveOptions so;
    if (opts) so = *opts; else default_solve_options(&so);
    SceneIn in;
    in.ph_in = have_g ? d_gd : d_rhs;   /* any nrow x ncol plane: the phase is not read */
    in.corr = d_wd;
    in.nrow = nrow;
    in.ncol = ncol;
    in.nlooks = p.ncorrlooks;
    std::vector<SceneIn> S(1, in);
    JobOpts jo;
    jo.fp64 = so.precision == CUPHU_PREC_FP64;
    jo.so = so;
    jo.so.n_irls = 0;
    jo.want_cc = false;
    jo.wls = true;
    jo.wls_gd = d_gd;
    jo.wls_gr = d_gr;
    jo.wls_rhs = d_rhs;
    jo.wls_wd = d_wd;
    jo.wls_wr = d_wr;
    jo.wls_u0 = d_u0;
    jo.wls_u = d_u;
    return run_job(S, p, jo, (cudaStream_t)stream, stats);
}

int cuphu_wls_grad_device(const double *d_lambda, const double *d_u, const float *d_gd,
                          const float *d_gr, const float *d_wd, const float *d_wr, int nrow,
                          int ncol, double *d_ggd, double *d_ggr, double *d_gwd, double *d_gwr,
                          void *stream)
{
    if (!d_lambda || !d_u || !d_gd || !d_gr || !d_wd || !d_wr || !d_ggd || !d_ggr || !d_gwd ||
        !d_gwr || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    return launch_wls_grad(d_lambda, d_u, d_gd, d_gr, d_wd, d_wr, nrow, ncol, d_ggd, d_ggr, d_gwd,
                           d_gwr, (cudaStream_t)stream);
}

int cuphu_laplace_unwrap_gpu(const void *d_smooth_costs, const float *d_phase, int nrow, int ncol,
                             double nshortcycle, int max_iter, float tol, int verbose, float *d_unw,
                             void *stream)
{
    (void)nshortcycle;
    (void)verbose;
    CuPhuSolveOptions so;
    default_solve_options(&so);
    so.max_iter = max_iter;
    so.tol = tol;
    return cuphu_laplace_solve_device(d_smooth_costs, 2, d_phase, nrow, ncol, &so, d_unw, nullptr,
                                      nullptr, nullptr, stream);
}

int cuphu_integrate_phase_gpu(const float *wrapped_phase, const short *hflows, const short *vflows,
                              int nrow, int ncol, int gpu_id, float *unw_out)
{
    if (!wrapped_phase || !hflows || !vflows || !unw_out || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    cudaStream_t s = lib_stream(gpu_id);
    float *rowoff = dev_alloc_async<float>(nrow, s);
    if (!rowoff) return fail(CUPHU_ERR_ALLOC, "device allocation failed");
    int rc = launch_integrate(wrapped_phase, hflows, vflows, nrow, ncol, rowoff, unw_out, s);
    cudaFreeAsync(rowoff, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cuphu_integrate_phase_gpu");
    return rc;
}

static int conncomp_scene(const float *unw, const float *corr, const unsigned char *mask, int nrow,
                          int ncol, const short *poscost, const short *negcost, float corr_thresh,
                          long conncompthresh, double minfrac, long maxncomps, uint32_t *labels_out,
                          cudaStream_t s)
{
    TileDesc T = {};
    T.ph = unw;
    T.corr = corr;
    T.mask = mask;
    T.ph_pitch = ncol;
    T.nr = nrow;
    T.nc = ncol;
    T.pitch = (ncol + 3) & ~3;
    T.nbx = (ncol + kItemBx - 1) / kItemBx;
    T.nitems = T.nbx * ((nrow + kItemBy - 1) / kItemBy);
    size_t np = (size_t)nrow * T.pitch;
    char *buf = dev_alloc_async<char>(np * 12 + sizeof(TileDesc) + (size_t)T.nitems * 4 +
                                          (size_t)nrow * 8 + 4096, s);
    if (!buf) return fail(CUPHU_ERR_ALLOC, "device allocation failed");
    Bump b(buf);
    SolverPlanes P = {};
    P.unw = b.take<float>(np);
    P.cc = b.take<uint32_t>(np);
    P.aux = b.take<uint32_t>(np);
    TileDesc *d_t = b.take<TileDesc>(1);
    int *d_item = b.take<int>(T.nitems);
    int *d_row = b.take<int>(2 * (size_t)nrow);
    int *d_nlab = b.take<int>(1);
    std::vector<int> zeros(std::max(T.nitems, nrow), 0);
    int rc = 0;
    cudaMemcpyAsync(d_t, &T, sizeof(T), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_item, zeros.data(), T.nitems * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_row + nrow, zeros.data(), (size_t)nrow * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpy2DAsync(P.unw, (size_t)T.pitch * 4, unw, (size_t)ncol * 4, (size_t)ncol * 4, nrow,
                      cudaMemcpyDeviceToDevice, s);
    CcArgs ca;
    ca.poscost = poscost;
    ca.negcost = negcost;
    ca.corr_thresh = corr_thresh;
    ca.conncompthresh = conncompthresh;
    ca.minfrac = minfrac;
    ca.maxncomps = (int)std::min<long>(maxncomps, 0x7fffffffL);
    rc = launch_conncomp(d_t, 1, nrow, d_item, T.nitems, P, ca, d_row, d_nlab, s);
    if (!rc)
        cudaMemcpy2DAsync(labels_out, (size_t)ncol * 4, P.cc, (size_t)T.pitch * 4, (size_t)ncol * 4,
                          nrow, cudaMemcpyDeviceToDevice, s);
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFreeAsync(buf, s);
    cudaStreamSynchronize(s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "conncomp");
    return rc;
}

int cuphu_conncomp_gpu(const float *unw, const float *corr, const unsigned char *mask, int nrow,
                       int ncol, const short *poscost, const short *negcost,
                       const CuPhuParams *params, int gpu_id, uint32_t *labels_out)
{
    if (!unw || !corr || !labels_out || !params || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    if ((poscost == nullptr) != (negcost == nullptr))
        return fail(CUPHU_ERR_INVALID, "poscost and negcost must both be given or both NULL");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    return conncomp_scene(unw, corr, mask, nrow, ncol, poscost, negcost, 0.05f,
                          params->conncompthresh, params->minconncompfrac, params->maxncomps,
                          labels_out, lib_stream(gpu_id));
}

int cuphu_conncomp_ex(const float *unw, const float *corr, const unsigned char *mask, int nrow,
                      int ncol, float corr_thresh, double minfrac, long maxncomps, int gpu_id,
                      uint32_t *labels_out)
{
    if (!unw || !corr || !labels_out || nrow < 1 || ncol < 1)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    CUPHU_TRY_CUDA(cudaSetDevice(gpu_id));
    cudaStream_t s = lib_stream(gpu_id);
    size_t n = (size_t)nrow * ncol;
    float *du = dev_alloc_async<float>(n, s), *dc = dev_alloc_async<float>(n, s);
    unsigned char *dm = mask ? dev_alloc_async<unsigned char>(n, s) : nullptr;
    uint32_t *dl = dev_alloc_async<uint32_t>(n, s);
    int rc = 0;
    if (!du || !dc || !dl || (mask && !dm)) rc = fail(CUPHU_ERR_ALLOC, "device allocation failed");
    if (!rc) {
        rc = copy_async(du, unw, 4 * n, cudaMemcpyHostToDevice, s, "H2D unw");
        if (!rc) rc = copy_async(dc, corr, 4 * n, cudaMemcpyHostToDevice, s, "H2D corr");
        if (!rc && mask) rc = copy_async(dm, mask, n, cudaMemcpyHostToDevice, s, "H2D mask");
    }
    if (!rc) {
        rc = conncomp_scene(du, dc, dm, nrow, ncol, nullptr, nullptr, corr_thresh, 0, minfrac,
                            maxncomps, dl, s);
    }
    if (!rc) rc = copy_async(labels_out, dl, 4 * n, cudaMemcpyDeviceToHost, s, "D2H labels");
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFreeAsync(du, s); cudaFreeAsync(dc, s); cudaFreeAsync(dl, s);
    if (dm) cudaFreeAsync(dm, s);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "cuphu_conncomp_ex");
    return rc;
}

int cuphu_incrcost_early_exit(const void *d_costs_flat, const short *d_flows_flat, int narcs,
                              long nshortcycle, int nflow, short *d_poscost, short *d_negcost,
                              int *d_scratch)
{
    if (!d_costs_flat || !d_flows_flat || !d_poscost || !d_negcost || !d_scratch || narcs < 0)
        return fail(CUPHU_ERR_INVALID, "bad arguments");
    if (nflow < 1) return fail(CUPHU_ERR_INVALID, "nflow must be >= 1");
    int rc = launch_incrcost((const short *)d_costs_flat, d_flows_flat, narcs, nshortcycle, nflow,
                             d_poscost, d_negcost, d_scratch, 0);
    if (rc) return rc;
    int h[2];
    CUPHU_TRY_CUDA(cudaMemcpy(h, d_scratch, sizeof(h), cudaMemcpyDeviceToHost));
    return (h[0] >= 0 && h[1] >= 0) ? 1 : 0;
}

int cuphu_gpu_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int cuphu_gpu_name(int device, char *buf, int len)
{
    cudaDeviceProp p;
    CUPHU_TRY_CUDA(cudaGetDeviceProperties(&p, device));
    if (buf && len > 0) {
        std::strncpy(buf, p.name, (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return 0;
}

int cuphu_gpu_info(int device, long long *total_memory, int *sm_count, int *cc_major, int *cc_minor)
{
    cudaDeviceProp p;
    CUPHU_TRY_CUDA(cudaGetDeviceProperties(&p, device));
    if (total_memory) *total_memory = (long long)p.totalGlobalMem;
    if (sm_count) *sm_count = p.multiProcessorCount;
    if (cc_major) *cc_major = p.major;
    if (cc_minor) *cc_minor = p.minor;
    return 0;
}

int cuphu_last_status(int gpu_id)
{
    if (gpu_id < 0 || gpu_id >= 64) return fail(CUPHU_ERR_INVALID, "device index out of range");
    return device_status(gpu_id);
}

int cuphu_release_workspace(int gpu_id)
{
    if (gpu_id < 0 || gpu_id >= 64) return fail(CUPHU_ERR_INVALID, "device index out of range");
    Workspace &W = g_ws[gpu_id];
    std::lock_guard<std::mutex> lock(W.mu);
    /* the caller's current device is restored on return */
    int prev = -1;
    CUPHU_TRY_CUDA(cudaGetDevice(&prev));
    int rc = cuda_fail(cudaSetDevice(gpu_id), "cudaSetDevice");
    if (!rc) rc = cuda_fail(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    if (!rc) {
        if (W.dev) cudaFree(W.dev);
        if (W.host) cudaFreeHost(W.host);
        W.dev = nullptr;
        W.host = nullptr;
        W.dev_size = W.host_size = 0;
    }
    cudaSetDevice(prev);
    return rc;
}

}  /* extern "C" */
