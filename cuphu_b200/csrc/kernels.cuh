/*
 * kernels.cuh -- device data structures shared by the kernels and the host
 * orchestrator, and the launcher declarations.
 *
 * HBM layout: the tiles of every scene of a job are stacked row-wise into
 * one 2-D array per plane with a common pitch (the widest tile rounded up to
 * 4 elements, so every row starts 16-byte aligned); one TMA tensor map per
 * plane then addresses every tile.  Arc weights live in two planes: wd[r][c] is
 * the down arc (r,c)->(r+1,c) (the reference's row arc, cuphu_laplace.cu:85)
 * and wr[r][c] the right arc (r,c)->(r,c+1) (col arc, :86); the last row of
 * wd and the last column of wr are zero.  Scene-level arrays (phase, corr,
 * mask, outputs) stay in the caller's row-major layout and tiles address them
 * through origin pointers.
 */
#pragma once

#include "common.cuh"

namespace cuphu {

struct TileDesc {
    const float *ph;            /* wrapped phase at the tile origin (scene layout) */
    const float *corr;          /* coherence at the tile origin                    */
    const unsigned char *mask;  /* solve mask at the tile origin, or NULL          */
    const unsigned char *conf;  /* stitching confidence mask, or NULL              */
    int ph_pitch;               /* scene row pitch (ncol)                          */
    int scene;
    int nr, nc, pitch;          /* tile shape and plane pitch                      */
    int r0, c0;                 /* origin in the scene                             */
    int tr, tc;                 /* position in the scene's tile grid               */
    long long pix;              /* plane offset of this tile (elements)            */
    int item0, nbx, nitems;     /* solver work items                               */
    int row0;                   /* offset of this tile's rows in per-row arrays   */
};

struct SolverPlanes {
    float *w0d, *w0r;           /* data weights 1/sigsq                  */
    float *wd, *wr;             /* current IRLS weights                  */
    double *x;                  /* solution, FP64 in both precisions     */
    double *bvec;               /* mixed: right-hand side of the current IRLS
                                   pass, stored by its assembly for the
                                   true-residual replacements (else NULL) */
    float *dx;                  /* mixed: FP32 increment since the last fold */
    void *r, *p0, *p1;          /* PCG vectors, float or double; p is    */
    void *q, *diag;             /* double-buffered across iterations     */
    void *z;                    /* z = r / diag (mixed: first z buffer; r is the second) */
    float *q1;                  /* mixed: second q buffer                */
    float *unw;                 /* congruent unwrapped phase per tile    */
    int32_t *cyc;               /* optional cycle map per tile           */
    float *cont;                /* optional anchored continuous solution */
    uint32_t *cc;               /* union-find parents, then labels       */
    uint32_t *aux;              /* component sizes, then root labels     */
    const float *gd, *gr;       /* WLS mode: per-arc targets in place of the
                                   wrapped phase differences (optional) */
    const float *rhs;           /* WLS mode: explicit right-hand side (optional) */
};

/* FP64 partial sums per solver work item: the mixed pass reduces r.z, p.q,
 * z.q and q.(q/diag) together; every other phase uses the first component */
constexpr int kNComp = 4;

/* per-tile PCG scalars, double-buffered by iteration parity: every block
 * touching a tile derives the same values from the same partials */
struct TileState {
    double rz, rz0, thr, alpha, beta;
    int active, iter;
};

struct SolverCtl {
    unsigned bar_count, bar_gen;
    int err, n_active, snap;
    int total_iters, max_pass_iters;
    int pass_max;                  /* largest iteration count of the current pass (mixed) */
    unsigned long long px_iters;   /* sum over tiles and passes of iterations x pixels */
};

struct SolveParams {
    int n_irls, max_iter, replace_every;
    float tol;
    const float *deltas;        /* per-pass IRLS delta (host powf schedule) */
    int *pass_iters;            /* [n_irls+1] iterations per pass (out)     */
    long long timeout_ns;       /* grid-barrier wait limit                   */
    int wls = 0;                /* raw solve: no anchor / congruence phase   */
    int warm = 0;               /* keep the caller's initial x on pass 0     */
    int skip_block = -1;        /* failure test: this block does not arrive at
                                   the first grid barrier (-1: none)         */
};

/* laplace.cu: arm the failure test for the next solver launch on a device */
void solver_skip_barrier_once(int dev, int block);

struct ScenePlan {
    float *unw_out;
    uint32_t *cc_out;
    const float *ph;            /* scene wrapped phase */
    int nrow, ncol;
    int ntr, ntc, rovl, covl;
    int tile0;                  /* first tile index */
    int pair0;                  /* first stitching pair (horizontal then vertical) */
    const int *rowmap, *colmap; /* merge maps: scene row/col -> tile row/col */
    int ref_row, ref_col;
    int maxncomps;
    double minfrac;
    int single;
};

struct PairDesc {
    int a, b, dir;              /* tiles; dir 0 = a left of b, 1 = a above b */
    int ov;
};

struct SceneOut {               /* filled by k_stitch_finalize */
    float shift;
    int do_shift;
};

/* cost.cu */
int launch_phase(const float2 *ig, float *ph, long long n, cudaStream_t s);
int launch_phase_split(const float *re, const float *im, float *ph, long long n, cudaStream_t s);
int launch_costs(const float *ph, const float *corr, const short *weights, int nrow, int ncol,
                 int mode, const CuPhuParams &p, void *costs, signed char *res, cudaStream_t s);
int launch_residues(const float *ph, int nrow, int ncol, signed char *res, cudaStream_t s);
int launch_w0(const TileDesc *tiles, const int *item_tile, int nitems, const CostConsts *sk,
              const SolverPlanes &P, cudaStream_t s);
int launch_w0_from_costs(const short *costs, int stride, int nrow, int ncol, int pitch,
                         const SolverPlanes &P, cudaStream_t s);

/* host_phase.cu: the reference's host phase of an interleaved (c64) or split
 * (re, im) host interferogram, uploaded into d_ph on stream s */
int upload_host_phase(const float *c64, const float *re, const float *im, size_t n, float *d_ph,
                      int dev, cudaStream_t s);
/* the same phase into host memory, computed by the host thread pool */
void compute_host_phase(const float *c64, const float *re, const float *im, size_t n, float *out);

/* laplace.cu */
int launch_solve(bool fp64, const TileDesc *tiles, const int *item_tile, int nitems,
                 int ntiles, const SolverPlanes &P, int plane_pitch, int plane_rows,
                 TileState *st, double *part, SolverCtl *ctl, const SolveParams &sp,
                 int device, cudaStream_t s);
/* the solver's launch shapes (ring stages, blocks per SM) the autotuner
 * chooses among, per precision; shape v of solve_shape_count(fp64) */
int solve_shape_count(bool fp64);
void solve_shape_of(bool fp64, int v, int *stages, int *blocks_per_sm);

/* conncomp.cu */
struct CcArgs {
    const short *poscost, *negcost;   /* flat arc layout of a single scene, or NULL */
    float corr_thresh;                /* validity floor, 0.05 (cuphu_conncomp.cu:324-325) */
    long conncompthresh;
    double minfrac;
    int maxncomps;
};
int launch_conncomp(const TileDesc *tiles, int ntiles, int total_rows, const int *item_tile,
                    int nitems, const SolverPlanes &P, const CcArgs &a, int *rowcnt,
                    int *ntile_labels, cudaStream_t s);

/* stitch.cu */
int launch_stitch(const ScenePlan *scenes, int nscenes, const TileDesc *tiles,
                  const PairDesc *pairs, int npairs, const SolverPlanes &P,
                  const int *ntile_labels, double *pair_k, double *tile_k,
                  unsigned *comp_off, SceneOut *sout, cudaStream_t s);
int launch_merge(const ScenePlan *scenes, const ScenePlan *h_scenes, int nscenes,
                 const TileDesc *tiles, const SolverPlanes &P, const double *tile_k,
                 const unsigned *comp_off, const SceneOut *sout, cudaStream_t s);

/* postpass.cu: the reference's optional post-passes on a stitched scene
 * (scene layout, device memory); scratch of postpass_scratch_bytes */
size_t postpass_scratch_bytes(int nrow, int ncol);
int launch_fix_cycle_spikes(float *unw, const unsigned char *mask, int nrow, int ncol,
                            void *scratch, cudaStream_t s);
int launch_neighbor_feedback(float *unw, const unsigned char *mask, int nrow, int ncol, int ntr,
                             int ntc, int rovl, int covl, int feather, void *scratch,
                             cudaStream_t s);
/* bridge.cu: phase bridging of a stitched scene (device unw and conncomp,
 * scene layout); synchronises the stream for its region-scale steps */
int run_bridge(float *unw, uint32_t *cc, const unsigned char *mask, int nrow, int ncol,
               const CuPhuBridgeParams &bp, cudaStream_t s);
/* stitch.cu: the reference-pixel shift of a merged scene (_unwrap.py:605-617) */
int launch_ref_shift(float *unw, const float *ph, int nrow, int ncol, int ref_row, int ref_col,
                     SceneOut *tmp, cudaStream_t s);

/* tune.cu: kind 0 = cost-kernel variant (0: 3 blocks/SM, 1: 4 blocks/SM),
 * kind 1 = persistent-solver blocks per SM; -1 = no stored choice */
int tune_class(long long n);
int tune_get(int dev, int kind, long long n);
void tune_set(int dev, int kind, long long n, int v);
void tune_force(int kind, int v);
void tune_note_items(long long n);   /* solver job size of the last launch */
long long tune_probe_items();

/* adjoint.cu */
int launch_wls_grad(const double *lam, const double *u, const float *gd, const float *gr,
                    const float *wd, const float *wr, int nrow, int ncol, double *ggd, double *ggr,
                    double *gwd, double *gwr, cudaStream_t s);

/* integrate.cu */
int launch_integrate(const float *ph, const short *hflows, const short *vflows, int nrow,
                     int ncol, float *rowoff, float *unw, cudaStream_t s);
int launch_incrcost(const short *costs, const short *flows, int narcs, long nsc, int nflow,
                    short *pos, short *neg, int *scratch, cudaStream_t s);
int launch_mst_costs(const short *costs, long long narcs, long nsc, long maxcost, short *out,
                     cudaStream_t s);

}  // namespace cuphu
