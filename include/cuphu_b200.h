/*
 * cuphu_b200.h -- C ABI of the B200-native cuPHU unwrapping path.
 *
 * Drop-in for the reference's C interface (src/cxx/cuphu/cuphu.h).  Structs
 * and enums keep the reference's field order and values so a caller built
 * against the reference header links against libcuphu_b200.so unchanged.
 * Every entry point returns an int status (0 = success, negative =
 * cuphu_status_t) instead of throwing across the ABI (the reference throws
 * std::runtime_error from CUDA_CHECK, cuphu.h:432-440); the message of the
 * last failure on the calling thread is available from cuphu_last_error().
 *
 * Streams are passed as void* (a cudaStream_t; NULL = legacy default stream).
 * "Device" pointers must be device-accessible memory on the selected GPU.
 */
#ifndef CUPHU_B200_H
#define CUPHU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ── status codes (new; the reference throws instead) ──────────────────── */
typedef enum {
    CUPHU_OK                 =  0,
    CUPHU_ERR_ALLOC          = -1,  /* host or device allocation failed (ref: -1) */
    CUPHU_ERR_INVALID        = -2,  /* bad argument (shape, pointer, mode)         */
    CUPHU_ERR_CUDA           = -3,  /* CUDA runtime error                          */
    CUPHU_ERR_UNSUPPORTED    = -4,  /* feature outside this build (MCF/MST, bridge)*/
    CUPHU_ERR_TIMEOUT        = -5,  /* a device-side wait hit its spin limit       */
    CUPHU_ERR_NOT_CONVERGED  = -6   /* reserved: a loop hit its iteration cap      */
} cuphu_status_t;

/* ref cuphu.h:19-23 */
typedef enum {
    CUPHU_COST_SMOOTH = 0,
    CUPHU_COST_DEFO   = 1,
    CUPHU_COST_TOPO   = 2
} CuPhuCostMode;

/* ref cuphu.h:26-30 */
typedef enum {
    CUPHU_INIT_MST     = 0,
    CUPHU_INIT_MCF     = 1,
    CUPHU_INIT_LAPLACE = 2
} CuPhuInitMethod;

/* ref cuphu.h:33-92 -- identical layout */
typedef struct CuPhuParams {
    double nlooks, ncorrlooks, defothreshfactor, rhosconst1, rhosconst2;
    double cstd1, cstd2, cstd3;
    double sigsqcorr, costscale, nshortcycle;
    long   sigsqshortmin;
    double orbitradius, altitude, earthradius, baseline, baselineangle, bperp;
    int    transmitmode;
    long   nlooksrange, nlooksaz, nlooksother, ncorrlooksrange, ncorrlooksaz;
    double nearrange, dr, da, rangeres, azres, lambda;
    double kds, specularexp, dzrcritfactor;
    int    shadow;
    double dzeimin;
    long   laywidth;
    double layminei, sloperatiofactor, sigsqei;
    double dzlaypeak, azdzfactor, dzeifactor, dzeiweight;
    double dzlayfactor, layconst, layfalloffconst, sigsqlayfactor;
    double defoazdzfactor, defomax, defolayconst;
    int    kperpdpsi, kpardpsi;
    double p, maxcost, costscaleambight, dnomincangle;
    double initdzr, initdzstep, threshold;
    long   initmaxflow, arcmaxflowconst, maxflow, nshortcycleL;
    long   cs2scalefactor;
    double minconncompfrac;
    long   conncompthresh;
    long   maxncomps;
} CuPhuParams;

/* ref cuphu.h:95-138 -- identical layout */
typedef struct CuPhuTileParams {
    int ntilerow, ntilecol;
    int rowovrlp, colovrlp;
    int tilecostthresh;
    int minregionsize;
    int nproc;
    int ngpustreams;
    int single_tile_reoptimize;
    int laplace_neighbor_feedback;
    int laplace_neighbor_feedback_feather;
    int fix_cycle_spikes;
} CuPhuTileParams;

/* ref cuphu.h:142-162 -- identical layout; enabled != 0 runs phase
 * bridging as the last stage of cuphu_unwrap */
typedef enum {
    CUPHU_RAMP_NONE = 0, CUPHU_RAMP_LINEAR, CUPHU_RAMP_QUADRATIC,
    CUPHU_RAMP_LINEAR_RANGE, CUPHU_RAMP_LINEAR_AZIMUTH,
    CUPHU_RAMP_QUADRATIC_RANGE, CUPHU_RAMP_QUADRATIC_AZIMUTH
} CuPhuRampType;

typedef struct CuPhuBridgeParams {
    int enabled, radius, min_num_pixel, erosion_size, max_boundary_samples;
    CuPhuRampType ramp_type;
    int ramp_max_num_sample;
} CuPhuBridgeParams;

/* ref cuphu.h:165-169; unw/conncomp are malloc'd by the callee, caller frees */
typedef struct CuPhuResult {
    float    *unw;
    uint32_t *conncomp;
    int       nrow, ncol;
} CuPhuResult;

/* ── solver options (new; no reference counterpart -- the reference reads
 *    the same knobs from CUPHU_N_IRLS, CUPHU_IRLS_DELTA_MAX/MIN,
 *    CUPHU_LAPLACE_MAX_ITER and CUPHU_LAPLACE_TOL, cuphu_laplace.cu:385-390
 *    and cuphu_solver.cpp:468-472, which cuphu_default_solve_options honours) */
typedef enum {
    CUPHU_PREC_MIXED = 0,   /* FP32 stencil/vectors, FP64 dots + residual replacement */
    CUPHU_PREC_FP64  = 1    /* FP64 vectors and dots ("plain FP64 PCG")              */
} CuPhuPrecision;

typedef struct CuPhuSolveOptions {
    int   precision;          /* CuPhuPrecision                                  */
    int   n_irls;             /* IRLS re-solves after the first (default 16)     */
    float irls_delta_max;     /* 0.5                                             */
    float irls_delta_min;     /* 0.01                                            */
    int   max_iter;           /* PCG matvecs per solve (1000)                    */
    float tol;                /* stop when rz < tol^2 rz0 (1e-3)                 */
    int   replace_every;      /* mixed: true-residual replacement period (50)    */
    int   ref_row, ref_col;   /* reference pixel; -1 disables the 2pi shift      */
    int   timeout_ms;         /* device spin limit per grid barrier (5000)       */
    int   device_phase;       /* host-buffer entry points: 0 = wrapped phase from
                                 the host C library's float atan2, as the reference
                                 computes it (bit-exact downstream; default),
                                 1 = the device's correctly rounded angle        */
    int   merge_conncomp;     /* multi-tile scenes: 0 = per-tile label spaces
                                 offset tile by tile, as the reference merges
                                 them (default); 1 = one labelling of the whole
                                 stitched scene, so components that cross tile
                                 seams get one label                            */
} CuPhuSolveOptions;

/* per-call statistics (new) */
typedef struct CuPhuSolveStats {
    int    ntiles;
    int    total_iters;       /* sum over passes of the max PCG iterations      */
    int    max_iters_pass;    /* largest per-pass iteration count                */
    double solve_ms;          /* device time of the persistent solve            */
    double total_ms;          /* device time of the whole GPU pipeline          */
    double px_iters;          /* sum over tiles and passes of iterations x pixels */
} CuPhuSolveStats;

/* ── defaults (ref cuphu.h:177-179) ─────────────────────────────────────── */
void cuphu_default_params(CuPhuParams *p);
void cuphu_default_tile_params(CuPhuTileParams *tp);
void cuphu_default_bridge_params(CuPhuBridgeParams *bp);
void cuphu_default_solve_options(CuPhuSolveOptions *o);          /* new */

const char *cuphu_last_error(void);                               /* new */

/* ── full pipeline (ref cuphu.h:218-234, cuphu_solver.cpp:1675) ─────────────
 * Host pointers.  init_meth must be CUPHU_INIT_LAPLACE; MST/MCF need SNAPHU's
 * CPU network-flow solver, which is outside this build
 * (CUPHU_ERR_UNSUPPORTED).  mag is accepted and unused, as in the
 * reference's Laplace branch. */
int cuphu_unwrap(const float *igram_r, const float *igram_i, const float *corr,
                 const float *mag, const unsigned char *mask, int nrow, int ncol,
                 CuPhuCostMode cost_mode, CuPhuInitMethod init_meth,
                 const CuPhuParams *params, const CuPhuTileParams *tile,
                 const CuPhuBridgeParams *bridge, const unsigned char *orig_mask,
                 int gpu_id, CuPhuResult *result);

/* new: interleaved complex64 igram, caller-owned outputs, solver options and
 * statistics.  Host pointers; igram = 2*nrow*ncol floats (re, im). */
int cuphu_unwrap_ex(const float *igram_c64, const float *corr, const unsigned char *mask,
                    const unsigned char *orig_mask, int nrow, int ncol,
                    CuPhuCostMode cost_mode, const CuPhuParams *params,
                    const CuPhuTileParams *tile, const CuPhuSolveOptions *opts,
                    int gpu_id, float *unw_out, uint32_t *conncomp_out,
                    CuPhuSolveStats *stats);

/* new: the same pipeline on device-resident data, asynchronous on `stream`
 * (returns after enqueueing; stats are filled after a stream sync inside
 * the call only when stats != NULL).  phase_in may replace igram_c64: when
 * igram_c64 is NULL the wrapped phase (radians) is read from phase_in.  The
 * optional cycles_out receives the integer cycle map k (int32, nrow*ncol) with
 * unw = phi + 2*pi*k before tile stitching and the reference-pixel shift
 * (single-tile scenes only; NULL otherwise). */
int cuphu_unwrap_device(const float *igram_c64, const float *phase_in, const float *corr,
                        const unsigned char *mask, const unsigned char *orig_mask,
                        int nrow, int ncol, CuPhuCostMode cost_mode,
                        const CuPhuParams *params, const CuPhuTileParams *tile,
                        const CuPhuSolveOptions *opts, float *unw_out,
                        uint32_t *conncomp_out, int32_t *cycles_out,
                        CuPhuSolveStats *stats, void *stream);

/* new: batched solve of many independent scenes in one persistent launch
 * (device pointers; tiles of every scene share one solver launch). */
typedef struct CuPhuScene {
    const float         *igram_c64;   /* device, or NULL with phase      */
    const float         *phase;       /* device wrapped phase, or NULL   */
    const float         *corr;        /* device                          */
    const unsigned char *mask;        /* device or NULL                  */
    const unsigned char *orig_mask;   /* device or NULL                  */
    int                  nrow, ncol;
    int                  ntilerow, ntilecol, rowovrlp, colovrlp;
    double               nlooks;
    float               *unw_out;     /* device                          */
    uint32_t            *conncomp_out;/* device                          */
} CuPhuScene;

int cuphu_unwrap_batch_device(const CuPhuScene *scenes, int nscenes,
                              CuPhuCostMode cost_mode, const CuPhuParams *params,
                              const CuPhuSolveOptions *opts, CuPhuSolveStats *stats,
                              void *stream);

/* ── cost build (ref cuphu.h:243-256, cuphu_solver.cpp:2104-2171) ─────────
 * Host pointers.  Returns the element size (4 smooth, 8 defo/topo) or a
 * negative status; *costs_out is malloc'd (row arcs then col arcs). */
int cuphu_build_costs_gpu(const float *igram_r, const float *igram_i, const float *corr,
                          const float *mag, const short *weights, int nrow, int ncol,
                          CuPhuCostMode cost_mode, const CuPhuParams *params, int gpu_id,
                          void **costs_out, size_t *cost_elem_sz);

/* launcher level, device pointers (ref cuphu_cost.cu:339-411, 418-479).
 * *d_costs_out is allocated with cudaMallocAsync on `stream`; free it with
 * cudaFree / cudaFreeAsync.  d_roww/d_colw may be NULL (all weights 1). */
int cuphu_build_smooth_costs_gpu(const float *d_phase, const float *d_corr,
                                 const short *d_roww, const short *d_colw, int nrow, int ncol,
                                 const CuPhuParams *params, int kperpdpsi, int kpardpsi,
                                 void **d_costs_out, void *stream);
int cuphu_build_defo_costs_gpu(const float *d_phase, const float *d_corr,
                               const short *d_roww, const short *d_colw, int nrow, int ncol,
                               const CuPhuParams *params, int kperpdpsi, int kpardpsi,
                               void **d_costs_out, void *stream);

/* new: costs into a caller buffer (device), optional residues
 * ((nrow-1)*(ncol-1) int8, device or NULL).  mode: CuPhuCostMode. */
int cuphu_build_costs_device(const float *d_phase, const float *d_corr,
                             const short *d_weights, int nrow, int ncol, int mode,
                             const CuPhuParams *params, void *d_costs,
                             signed char *d_residues, void *stream);

/* new: residues of a wrapped phase (device; (nrow-1)*(ncol-1) int8) */
int cuphu_residues_gpu(const float *d_phase, int nrow, int ncol, signed char *d_res,
                       void *stream);

/* new: wrapped phase in [0,2pi) from an interleaved complex64 igram (device) */
int cuphu_phase_gpu(const float *d_igram_c64, long long n, float *d_phase, void *stream);

/* ── Laplace solve, launcher level (ref cuphu_laplace.cu:352-552) ─────────
 * d_smooth_costs: smoothcostT (offset, sigsq int16 pairs) in the flat
 * row-then-col layout; d_phase wrapped phase; d_unw output.  Uses the
 * default solve options with max_iter/tol overridden; verbose is ignored. */
int cuphu_laplace_unwrap_gpu(const void *d_smooth_costs, const float *d_phase, int nrow,
                             int ncol, double nshortcycle, int max_iter, float tol,
                             int verbose, float *d_unw, void *stream);

/* new: same with options, any cost element stride (2 = smooth, 4 = defo
 * shorts per arc), an optional int32 cycle-map output k (unw = phi + 2 pi k)
 * and an optional float output of the anchored continuous solution before
 * the congruence projection */
int cuphu_laplace_solve_device(const void *d_costs, int cost_stride_shorts,
                               const float *d_phase, int nrow, int ncol,
                               const CuPhuSolveOptions *opts, float *d_unw,
                               int32_t *d_cycles, float *d_cont, CuPhuSolveStats *stats,
                               void *stream);

/* ── launch-shape autotuner (new) ─────────────────────────────────────────
 * Times, on the caller's scene (host pointers, uploaded here), the cost
 * kernel at 3 and 4 blocks per SM and the persistent solver in each of its
 * launch shapes (stages of the per-block shared-memory ring x resident
 * blocks per SM; mixed precision: 3x2, 2x2, 6x1) with a 20-iteration probe
 * of the given tiling, and stores the fastest choice per device and
 * job-size class (floor(log2) of the arc or work-item count) for all later
 * calls.  choices (optional, int[2]) receives {cost variant 0|1, solver
 * shape index}.  Results are identical for every choice: the per-item and
 * per-tile reductions do not depend on the launch shape.  CUPHU_TUNE=0 in
 * the environment ignores stored choices. */
int cuphu_autotune(const float *igram_c64, const float *corr, int nrow, int ncol,
                   CuPhuCostMode cost_mode, const CuPhuParams *params,
                   const CuPhuTileParams *tile, int gpu_id, int *choices);

/* ── batched pipeline as a CUDA graph (new) ─────────────────────────────────
 * Plans the batch once into a workspace owned by the graph object, uploads
 * its descriptors and captures the whole device pipeline (state resets,
 * phase, weights, the persistent solve, conncomp, stitching, merge) into a
 * CUDA graph on the current device.  Every launch re-runs that pipeline on
 * the same device buffers named in `scenes` (refill the inputs in place
 * between launches).  Launches of one graph must not overlap each other on
 * the GPU.  Destroy synchronises the device and frees the workspace. */
int cuphu_batch_graph_create(const CuPhuScene *scenes, int nscenes, CuPhuCostMode cost_mode,
                             const CuPhuParams *params, const CuPhuSolveOptions *opts,
                             void **graph_out);
int cuphu_batch_graph_launch(void *graph, void *stream);
int cuphu_batch_graph_destroy(void *graph);

/* ── weighted least-squares solve and its adjoint (new; the differentiable
 *    core of the Laplace path, cuphu_laplace.cu:88-190 with explicit inputs)
 * u = argmin_u sum_a w_a ((D u)_a - g_a)^2 + eps |u|^2 on one nrow x ncol
 * grid, i.e. (D^T W D + eps I) u = D^T W g with eps = 1e-12 (the Laplace
 * solver's operator).  Planes are nrow x ncol, row-major, device memory:
 * d_gd/d_wd hold arc (r,c)->(r+1,c) (last row ignored), d_gr/d_wr arc
 * (r,c)->(r,c+1) (last column ignored); (D u)_a = u(head) - u(tail).
 * Give either d_gd and d_gr, or d_rhs (nrow x ncol) to solve
 * (D^T W D + eps I) u = rhs -- the adjoint solve.  d_u0: optional FP64
 * warm start.  d_u: FP64 solution (no anchoring).  opts: precision,
 * max_iter, tol, replace_every, timeout_ms (n_irls is ignored). */
int cuphu_wls_solve_device(const float *d_gd, const float *d_gr, const float *d_rhs,
                           const float *d_wd, const float *d_wr, const double *d_u0, int nrow,
                           int ncol, const CuPhuSolveOptions *opts, double *d_u,
                           CuPhuSolveStats *stats, void *stream);

/* gradients of the WLS solve from the adjoint state lambda = (D^T W D +
 * eps I)^-1 ubar and the forward solution u: d_ggd/d_ggr = w (D lambda),
 * d_gwd/d_gwr = (D lambda)(g - D u); nrow x ncol FP64 planes laid out like
 * the inputs (unused last row / column written 0) */
int cuphu_wls_grad_device(const double *d_lambda, const double *d_u, const float *d_gd,
                          const float *d_gr, const float *d_wd, const float *d_wr, int nrow,
                          int ncol, double *d_ggd, double *d_ggr, double *d_gwd, double *d_gwr,
                          void *stream);

/* ── integration of MCF flows (ref cuphu.h:261-270, cuphu_phase.cu:110-144) */
int cuphu_integrate_phase_gpu(const float *wrapped_phase, const short *hflows,
                              const short *vflows, int nrow, int ncol, int gpu_id,
                              float *unw_out);

/* ── integration without device allocation.  No counterpart in the
 *    reference.
 * Same result as cuphu_integrate_phase_gpu, for callers that cannot
 * allocate device memory (a host framework whose caching allocator holds
 * the device's memory, a real-time processor that forbids allocation after
 * start-up).  Device pointers; enqueued on `stream` of the current device,
 * no synchronisation.  The per-row scratch comes from a fixed array inside
 * the library (CUPHU_NOALLOC_MAX_ROWS floats, held by every GPU that loads
 * the library until exit), so nrow above CUPHU_NOALLOC_MAX_ROWS returns
 * CUPHU_ERR_INVALID.  The first call on a device looks up the array's
 * device address: make it before any stream capture.  The address is kept
 * for the life of the process and does not survive cudaDeviceReset.  All
 * calls on a device share the array, so calls that overlap on the GPU race;
 * order them on one stream or with events. */
#define CUPHU_NOALLOC_MAX_ROWS 65536
int cuphu_integrate_phase_noalloc(const float *wrapped_phase, const short *hflows,
                                  const short *vflows, int nrow, int ncol, float *unw_out,
                                  void *stream);

/* ── a scene fed band by band (new; the reference reads its inputs whole,
 *    _unwrap.py:515-523).  create: device planes for an nrow x ncol scene
 *    on gpu_id; flags say which masks the bands carry.  put_rows: host
 *    buffers of rows [row0, row0+nrows) (igram as interleaved complex64);
 *    the reference's host phase of the band is computed on the calling
 *    thread and the band is copied into one of two pinned staging slots and
 *    uploaded asynchronously, so the caller can read the next band while this
 *    one is in flight (the caller's buffers may be reused on return).
 *    unwrap: once every row has been put, the pipeline of cuphu_unwrap_device
 *    on the resident scene (synchronous).  get_rows: rows of the outputs into
 *    host buffers (either may be NULL).  destroy: frees the handle. */
#define CUPHU_STREAM_MASK      1   /* bands carry the solve mask           */
#define CUPHU_STREAM_ORIG_MASK 2   /* bands carry the original mask        */
int cuphu_stream_create(int nrow, int ncol, int flags, int gpu_id, void **handle);
int cuphu_stream_put_rows(void *handle, int row0, int nrows, const float *igram_c64,
                          const float *corr, const unsigned char *mask,
                          const unsigned char *orig_mask);
int cuphu_stream_unwrap(void *handle, CuPhuCostMode cost_mode, const CuPhuParams *params,
                        const CuPhuTileParams *tile, const CuPhuSolveOptions *opts,
                        CuPhuSolveStats *stats);
int cuphu_stream_get_rows(void *handle, int row0, int nrows, float *unw_out,
                          uint32_t *conncomp_out);
int cuphu_stream_destroy(void *handle);

/* ── inputs of the CPU network-flow front end, computed on the GPU (new;
 *    the reference computes them on the host, cuphu_solver.cpp:513-633).
 * cuphu_mst_costs_device: initial-flow arc weights of SMOOTH costs (device
 * smoothcostT pairs, flat row-then-col layout): SNAPHU's incremental cost of
 * a +-1 flow from flow 0, w = clip(min(pos, neg), 1, maxcost).
 * cuphu_mcf_inputs: host buffers; the reference's host phase, the cost
 * arrays (costs_out: 2 shorts per arc for SMOOTH, 4 for DEFO/TOPO), their
 * initial-flow weights (mst_costs_out, narcs shorts, SMOOTH only; NULL to
 * skip) and the residues (residues_out, (nrow-1)*(ncol-1), NULL to skip),
 * one host-to-device copy in and one device-to-host copy per output. */
int cuphu_mst_costs_device(const void *d_smooth_costs, long long narcs, long nshortcycle,
                           long maxcost, short *d_out, void *stream);
int cuphu_mcf_inputs(const float *igram_r, const float *igram_i, const float *corr,
                     const short *weights, int nrow, int ncol, CuPhuCostMode cost_mode,
                     const CuPhuParams *params, int gpu_id, short *costs_out,
                     short *mst_costs_out, signed char *residues_out);

/* ── phase bridging (ref cuphu_solver.cpp:996-1352, cuphu_bridge_gpu.cu):
 * whole-cycle offsets between the 8-connected regions of nonzero, unmasked
 * pixels (regions under min_num_pixel or without an erosion survivor
 * dropped) are reconciled along the minimum spanning tree of their nearest
 * boundary points from the largest region, by window medians of radius
 * `radius`, with an optional ramp (ramp_type) removed over the largest
 * region first.  conncomp is overwritten with the region labels.  Some
 * stages synchronise the stream.  Nothing changes when fewer than two
 * regions remain.
 * ref cuphu.h:381-389 (void there): host buffers, gpu_id selects the device */
int cuphu_bridge_apply_test(float *unw, uint32_t *conncomp, int nrow, int ncol,
                            const CuPhuBridgeParams *bridge, const unsigned char *mask,
                            int gpu_id);
/* new: device buffers on `stream` of the current device */
int cuphu_bridge_device(float *d_unw, uint32_t *d_conncomp, const unsigned char *d_mask, int nrow,
                        int ncol, const CuPhuBridgeParams *bridge, void *stream);

/* ── optional post-passes on a stitched scene (ref cuphu_solver.cpp
 *    :1385-1441, 1469-1656).  The pipeline runs them after the tile merge
 *    of a multi-tile scene when CuPhuTileParams.laplace_neighbor_feedback /
 *    fix_cycle_spikes are set (feedback first), before the reference-pixel
 *    shift.  mask (0 = invalid) may be NULL.  */
/* ref cuphu.h:397-409 (void there); host buffers, unw updated in place */
int cuphu_laplace_neighbor_feedback_test(float *unw, const unsigned char *mask, int nrow,
                                         int ncol, int ntr, int ntc, int row_ovrlp,
                                         int col_ovrlp, int feather_px);
/* ref cuphu.h:415-420 (void there); host buffers, unw updated in place */
int cuphu_fix_cycle_spikes_test(float *unw, const unsigned char *mask, int nrow, int ncol);
/* new: the same on device buffers, asynchronous on `stream` */
int cuphu_laplace_neighbor_feedback_device(float *d_unw, const unsigned char *d_mask, int nrow,
                                           int ncol, int ntr, int ntc, int row_ovrlp,
                                           int col_ovrlp, int feather_px, void *stream);
int cuphu_fix_cycle_spikes_device(float *d_unw, const unsigned char *d_mask, int nrow, int ncol,
                                  void *stream);

/* ── connected components (ref cuphu.h:275-289, cuphu_conncomp.cu:290-428) */
int cuphu_conncomp_gpu(const float *unw, const float *corr, const unsigned char *mask,
                       int nrow, int ncol, const short *poscost, const short *negcost,
                       const CuPhuParams *params, int gpu_id, uint32_t *labels_out);

/* new: host pointers, explicit coherence floor (regrow_conncomp semantics,
 * ref _conncomp.py:12-66: valid = corr >= corr_thresh && mask) */
int cuphu_conncomp_ex(const float *unw, const float *corr, const unsigned char *mask, int nrow,
                      int ncol, float corr_thresh, double minfrac, long maxncomps, int gpu_id,
                      uint32_t *labels_out);

/* ── incremental costs (ref cuphu_incrcost.cu:157-191); returns 1 when no
 *    negative incremental cost exists, 0 otherwise, negative on error */
int cuphu_incrcost_early_exit(const void *d_costs_flat, const short *d_flows_flat,
                              int narcs, long nshortcycle, int nflow, short *d_poscost,
                              short *d_negcost, int *d_scratch);

/* ── GPU queries (ref cuphu_py.cu:435-456) ─────────────────────────────── */
int cuphu_gpu_count(void);
int cuphu_gpu_name(int device, char *buf, int len);
int cuphu_gpu_info(int device, long long *total_memory, int *sm_count, int *cc_major,
                   int *cc_minor);

/* test hook (new): the next persistent solve launched on gpu_id runs with
 * block `block` not arriving at its first grid barrier, so every block's
 * bounded wait runs out after CuPhuSolveOptions.timeout_ms and the call's
 * device status becomes CUPHU_ERR_TIMEOUT (read by cuphu_last_status, or
 * returned by calls that wait).  One-shot: later launches are normal. */
int cuphu_test_skip_barrier_once(int gpu_id, int block);

/* test hook (new): solves launched later from the calling thread use launch
 * shape `shape` of the persistent solver (the index of cuphu_autotune's
 * choices[1]; an index beyond the precision's shapes selects shape 0),
 * overriding stored autotuner choices; -1 restores the normal choice. */
int cuphu_test_force_solve_shape(int shape);

/* wait for the last pipeline enqueued on a device and return its device-side
 * status (CUPHU_ERR_TIMEOUT when a grid barrier gave up) (new) */
int cuphu_last_status(int gpu_id);

/* release the cached per-device workspace (new) */
int cuphu_release_workspace(int gpu_id);

#ifdef __cplusplus
}
#endif
#endif /* CUPHU_B200_H */
