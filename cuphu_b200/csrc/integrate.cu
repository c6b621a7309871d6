/*
 * integrate.cu -- integration of network-flow cycle counts into unwrapped
 * phase (A15) and SNAPHU smooth-cost incremental costs (A18).
 *
 * Integration restates cuphu_integrate_phase_gpu (cuphu_phase.cu:42-144):
 * a float cumulative sum down column 0 (subtracting 2*pi*hflow), then per
 * row a float cumulative sum along the row (adding 2*pi*vflow), combined as
 * (phi00 + rowoff) + coloff.  The sums are order dependent, so each row keeps
 * the reference's sequential order; the B200 change is the memory access:
 * the reference runs one thread per row over strided global memory
 * (<<<nrow,1>>>) and a <<<1,1>>> column pass plus a separate apply kernel,
 * here a warp owns 32 rows and stages 32x32 chunks of phase and flows through
 * shared memory with coalesced loads and stores, writing unw directly.
 */
#include "kernels.cuh"

namespace cuphu {

__global__ void k_int_rowoff(const float *__restrict__ ph, const short *__restrict__ hflows,
                             int nrow, int ncol, float *rowoff)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    float cs = 0.0f;
    rowoff[0] = 0.0f;
    for (int r = 1; r < nrow; ++r) {
        float d = ph[(size_t)r * ncol] - ph[(size_t)(r - 1) * ncol];
        cs = __fadd_rn(cs, __fmaf_rn(-kTwoPiF, (float)hflows[(size_t)(r - 1) * ncol], wrap_angle(d)));
        rowoff[r] = cs;
    }
}

constexpr int kIntRowsPerWarp = 32;

__global__ void __launch_bounds__(128) k_int_rows(const float *__restrict__ ph,
                                                  const short *__restrict__ vflows,
                                                  const float *__restrict__ rowoff, int nrow,
                                                  int ncol, float *__restrict__ unw)
{
    __shared__ float sp[4][32][33];
    __shared__ float sv[4][32][33];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int r0 = (blockIdx.x * 4 + w) * kIntRowsPerWarp;
    if (r0 >= nrow) return;
    float ref = ph[0];
    int myr = r0 + lane;
    float base = myr < nrow ? __fadd_rn(ref, rowoff[myr]) : 0.0f;
    float cum = 0.0f, prev = 0.0f;
    for (int c0 = 0; c0 < ncol; c0 += 32) {
        for (int i = 0; i < 32; ++i) {
            int r = r0 + i, c = c0 + lane;
            if (r < nrow && c < ncol) {
                sp[w][i][lane] = ph[(size_t)r * ncol + c];
                sv[w][i][lane] = c > 0 ? (float)vflows[(size_t)r * (ncol - 1) + c - 1] : 0.0f;
            }
        }
        __syncwarp();
        if (myr < nrow) {
            for (int j = 0; j < 32 && c0 + j < ncol; ++j) {
                int c = c0 + j;
                float p = sp[w][lane][j];
                if (c > 0) {
                    float d = p - prev;
                    cum = __fadd_rn(cum, __fmaf_rn(kTwoPiF, sv[w][lane][j], wrap_angle(d)));
                }
                prev = p;
                sp[w][lane][j] = __fadd_rn(base, cum);
            }
        }
        __syncwarp();
        for (int i = 0; i < 32; ++i) {
            int r = r0 + i, c = c0 + lane;
            if (r < nrow && c < ncol) unw[(size_t)r * ncol + c] = sp[w][i][lane];
        }
        __syncwarp();
    }
}

int launch_integrate(const float *ph, const short *hflows, const short *vflows, int nrow,
                     int ncol, float *rowoff, float *unw, cudaStream_t s)
{
    if (nrow < 1 || ncol < 1) return 0;
    k_int_rowoff<<<1, 32, 0, s>>>(ph, hflows, nrow, ncol, rowoff);
    int warps = (nrow + kIntRowsPerWarp - 1) / kIntRowsPerWarp;
    k_int_rows<<<(warps + 3) / 4, 128, 0, s>>>(ph, vflows, rowoff, nrow, ncol, unw);
    return cuda_fail(cudaGetLastError(), "integrate kernels");
}

/* ── A18: cuphu_incrcost.cu:55-98 (exact 64-bit integer arithmetic) ────── */
__device__ __forceinline__ long long ceil_div(long long a, long long b)
{
    return a > 0 ? (a + b - 1) / b : a / b;
}
__device__ __forceinline__ long long floor_div(long long a, long long b)
{
    return a >= 0 ? a / b : (a - b + 1) / b;
}

__global__ void __launch_bounds__(256) k_incrcost(const short2 *__restrict__ costs,
                                                  const short *__restrict__ flows, int narcs,
                                                  long long nsc, int nflow, short *pos,
                                                  short *neg, int *mins)
{
    __shared__ int sp[8], sn[8];
    int mp = 32000, mn = 32000;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < narcs; i += gridDim.x * blockDim.x) {
        short2 c = costs[i];
        short pc_s, nc_s;
        if (c.y == 32000) {
            pc_s = 0; nc_s = 0;
        } else {
            long long flow = flows[i], off = c.x, sg = c.y, nf = nflow;
            long long i1 = llabs(flow * nsc + off);
            long long ip = llabs((flow + nf) * nsc + off);
            long long in = llabs((flow - nf) * nsc + off);
            long long c1 = (i1 * i1) / sg;
            long long pr = (ip * ip) / sg - c1;
            long long nr = (in * in) / sg - c1;
            long long nfsq = nf * nf;
            long long pc = pr > 0 ? ceil_div(pr, nfsq) : floor_div(pr, nfsq);
            long long nc = nr > 0 ? ceil_div(nr, nfsq) : floor_div(nr, nfsq);
            pc = max(-32000LL, min(32000LL, pc));
            nc = max(-32000LL, min(32000LL, nc));
            pc_s = (short)pc; nc_s = (short)nc;
        }
        pos[i] = pc_s;
        neg[i] = nc_s;
        mp = min(mp, (int)pc_s);
        mn = min(mn, (int)nc_s);
    }
    for (int off = 16; off > 0; off >>= 1) {
        mp = min(mp, __shfl_down_sync(0xffffffffu, mp, off));
        mn = min(mn, __shfl_down_sync(0xffffffffu, mn, off));
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sp[w] = mp; sn[w] = mn; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) { mp = min(mp, sp[k]); mn = min(mn, sn[k]); }
        atomicMin(mins, mp);
        atomicMin(mins + 1, mn);
    }
}

__global__ void k_init_mins(int *m)
{
    m[0] = 32000;
    m[1] = 32000;
}

/* Initial-flow arc weights of the network-flow front end
 * (cuphu_solver.cpp:607-633): SNAPHU's smooth incremental costs of a +-1
 * flow from flow 0 (the arithmetic of k_incrcost with flow 0, nflow 1, in
 * 64-bit integers), w = clip(min(pos, neg), 1, maxcost).  Arcs with
 * sigsq = LARGESHORT have no cost preference (pos = neg = 0) and get 1. */
__global__ void __launch_bounds__(256) k_mst_costs(const short2 *__restrict__ costs,
                                                   long long narcs, long long nsc,
                                                   long long maxcost, short *out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < narcs;
         i += (long long)gridDim.x * blockDim.x) {
        const short2 c = costs[i];
        long long m = 0;
        if (c.y != 32000) {
            const long long off = c.x, sg = c.y;
            const long long i1 = llabs(off), ip = llabs(nsc + off), in = llabs(off - nsc);
            const long long c1 = (i1 * i1) / sg;
            m = min((ip * ip) / sg - c1, (in * in) / sg - c1);
        }
        out[i] = (short)max(1LL, min(maxcost, m));
    }
}

int launch_mst_costs(const short *costs, long long narcs, long nsc, long maxcost, short *out,
                     cudaStream_t s)
{
    if (narcs > 0) {
        int blocks = (int)std::min<long long>((narcs + 255) / 256, 148LL * 8);
        k_mst_costs<<<blocks, 256, 0, s>>>(reinterpret_cast<const short2 *>(costs), narcs,
                                           (long long)nsc, (long long)maxcost, out);
    }
    return cuda_fail(cudaGetLastError(), "k_mst_costs");
}

int launch_incrcost(const short *costs, const short *flows, int narcs, long nsc, int nflow,
                    short *pos, short *neg, int *scratch, cudaStream_t s)
{
    k_init_mins<<<1, 1, 0, s>>>(scratch);
    if (narcs > 0) {
        int blocks = std::min((narcs + 255) / 256, 148 * 8);
        k_incrcost<<<blocks, 256, 0, s>>>(reinterpret_cast<const short2 *>(costs), flows, narcs,
                                          (long long)nsc, nflow, pos, neg, scratch);
    }
    return cuda_fail(cudaGetLastError(), "k_incrcost");
}

}  // namespace cuphu
