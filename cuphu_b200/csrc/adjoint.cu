/*
 * adjoint.cu -- gradient assembly of the weighted least-squares solve.
 *
 * The WLS solve u = argmin_u sum_a w_a ((D u)_a - g_a)^2 + eps |u|^2 has the
 * self-adjoint operator L = D^T W D + eps I (the Laplace solver's operator,
 * cuphu_laplace.cu:156-190), so for a loss l(u) with ubar = dl/du the
 * adjoint state is lambda = L^-1 ubar -- one more PCG solve, done by the
 * solver in WLS mode -- and
 *     dl/dg_a = w_a (D lambda)_a,   dl/dw_a = (D lambda)_a (g_a - (D u)_a),
 * where (D x)_a = x(head) - x(tail) for arc a.  This kernel forms both
 * gradients per arc from lambda and the forward solution.  Planes are
 * nrow x ncol row-major: arc (r,c)->(r+1,c) in the "d" planes (last row
 * unused, written 0), arc (r,c)->(r,c+1) in the "r" planes (last column 0).
 */
#include "kernels.cuh"

namespace cuphu {

__global__ void __launch_bounds__(256) k_wls_grad(const double *__restrict__ lam,
                                                  const double *__restrict__ u,
                                                  const float *__restrict__ gd,
                                                  const float *__restrict__ gr,
                                                  const float *__restrict__ wd,
                                                  const float *__restrict__ wr, int nrow,
                                                  int ncol, double *__restrict__ ggd,
                                                  double *__restrict__ ggr,
                                                  double *__restrict__ gwd,
                                                  double *__restrict__ gwr)
{
    const long long n = (long long)nrow * ncol;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / ncol), c = (int)(i - (long long)r * ncol);
        double a_gd = 0.0, a_wd = 0.0, a_gr = 0.0, a_wr = 0.0;
        if (r < nrow - 1) {
            const double dl = lam[i + ncol] - lam[i];
            const double e = (double)gd[i] - (u[i + ncol] - u[i]);
            a_gd = (double)wd[i] * dl;
            a_wd = dl * e;
        }
        if (c < ncol - 1) {
            const double dl = lam[i + 1] - lam[i];
            const double e = (double)gr[i] - (u[i + 1] - u[i]);
            a_gr = (double)wr[i] * dl;
            a_wr = dl * e;
        }
        ggd[i] = a_gd;
        gwd[i] = a_wd;
        ggr[i] = a_gr;
        gwr[i] = a_wr;
    }
}

int launch_wls_grad(const double *lam, const double *u, const float *gd, const float *gr,
                    const float *wd, const float *wr, int nrow, int ncol, double *ggd, double *ggr,
                    double *gwd, double *gwr, cudaStream_t s)
{
    long long n = (long long)nrow * ncol;
    if (n <= 0) return 0;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    k_wls_grad<<<blocks, 256, 0, s>>>(lam, u, gd, gr, wd, wr, nrow, ncol, ggd, ggr, gwd, gwr);
    return cuda_fail(cudaGetLastError(), "k_wls_grad");
}

}  // namespace cuphu
