/*
 * cuphu_oracle.h -- CPU restatement of cuPHU's data-parallel unwrapping path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, as the checker.
 *
 * Every function cites the reference file:line whose arithmetic it restates.
 * Floating-point expressions that the CUDA compiler contracts into a fused
 * multiply-add in the reference kernels are written with fma()/fmaf() here,
 * and the file is compiled with -ffp-contract=off so that no other
 * contraction happens.
 */
#ifndef CUPHU_ORACLE_H
#define CUPHU_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* statistical-cost parameters (subset of CuPhuParams, cuphu.h:33-92) */
typedef struct {
    double ncorrlooks, defothreshfactor, rhosconst1, rhosconst2;
    double cstd1, cstd2, cstd3, sigsqcorr, costscale, nshortcycle;
    long   sigsqshortmin;
    double defomax;
} orc_cost_params;

/* Laplace solve options (cuphu_laplace.cu:385-390, cuphu_solver.cpp:468-469) */
typedef struct {
    int   n_irls;          /* IRLS re-solves after the first (reference 16) */
    float delta_max;       /* 0.5  */
    float delta_min;       /* 0.01 */
    int   max_iter;        /* 1000 */
    float tol;             /* 1e-3 */
    /* canonical reduction geometry shared with the GPU solver */
    int   item_tx, item_vx, item_by;
} orc_lap_opts;

void orc_phase_from_igram(const float *re, const float *im, long n, float *phase);
void orc_phase_from_c64(const float *c64, long n, float *phase);
void orc_wrap_phase(float *p, long n);
void orc_phase_diffs(const float *phase, int nrow, int ncol, float *rng, float *az);
void orc_boxcar2d(const float *src, float *dst, int nrow, int ncol, int kr, int kc);
void orc_cost_constants(const orc_cost_params *p, double out[9]);
void orc_arc_weights_from_mask(const unsigned char *mask, int nrow, int ncol, short *w);
int  orc_build_costs(const float *phase, const float *corr, const short *weights,
                     int nrow, int ncol, int mode, const orc_cost_params *p,
                     int kperp, int kpar, short *out);
void orc_residues(const float *phase, int nrow, int ncol, signed char *out);

int  orc_laplace_f64(const short *costs, int cost_stride, const float *phase,
                     int nrow, int ncol, const orc_lap_opts *o,
                     double *x_out, int *k_out, float *unw_out, int *iters_out);

int  orc_conncomp(const float *unw, const float *corr, const unsigned char *mask,
                  int nrow, int ncol, const short *poscost, const short *negcost,
                  double minfrac, long maxncomps, long conncompthresh,
                  unsigned *labels);

void orc_integrate_phase(const float *phase, const short *hflows, const short *vflows,
                         int nrow, int ncol, float *unw);

int  orc_incrcost(const short *costs, const short *flows, long narcs, long nsc,
                  int nflow, short *pos, short *neg);

void orc_tile_bounds(int n, int nt, int ovl, int t, int *first, int *len);

int  orc_unwrap_tiled(const float *phase, const float *corr, const unsigned char *mask,
                      const unsigned char *conf_mask, int nrow, int ncol, int mode,
                      const orc_cost_params *p, int kperp, int kpar,
                      const orc_lap_opts *o, int ntr, int ntc, int rovl, int covl,
                      double minfrac, long maxncomps, long conncompthresh,
                      float *unw, unsigned *cc, double *tile_k_out);

double orc_dot_canonical(const double *a, const double *b, int nrow, int ncol,
                         int tx, int vx, int by);

/* cuphu_oracle_post.c: the optional post-passes on a stitched scene */
void orc_fix_cycle_spikes(float *unw, const unsigned char *mask, int nrow, int ncol);
void orc_neighbor_feedback(float *unw, const unsigned char *mask, int nrow, int ncol, int ntr,
                           int ntc, int rovl, int covl, int feather);

/* cuphu_oracle_bridge.c: phase bridging; returns the number of regions
 * bridged (0 when there was nothing to bridge and nothing was changed) */
int orc_bridge(float *unw, uint32_t *conncomp, int nrow, int ncol, const unsigned char *mask,
               int radius, int min_num_pixel, int erosion_size, int max_boundary_samples,
               int ramp_type, int ramp_max_num_sample);

#ifdef __cplusplus
}
#endif
#endif
