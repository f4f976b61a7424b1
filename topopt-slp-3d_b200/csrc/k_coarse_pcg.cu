// PCG on the coarsest grid (mg.opchol = 1): eH = pcg(A_c, rH, tolPCG,
// maxiterPCG, M) of I/VCycle.m:28-35 / I/FMVCycle.m:24-33, taken when the
// coarsest system is too large for the direct solve and no further grid is
// possible (I/StartStrSLP.m:122-132), or when the caller asks for it.
//
// One cooperative kernel per coarse solve, FP64 throughout: the coarsest
// Galerkin operator as a node-major 27-point stencil (one warp per node, the
// arithmetic of k_stencil_warp), the Jacobi preconditioner z = D^-1 r, and the
// CG recurrences of MATLAB's pcg from a zero iterate: stop once
// ||r|| <= tol ||b|| or after maxit iterations (the iterate is returned
// either way; the reference discards pcg's flag).  Each iteration has three
// grid-wide phases separated by the bounded grid barrier:
//   A  q = A p and the block partials of p'q;
//   B  alpha = rho / p'q; x += alpha p; r -= alpha q; partials of r'D^-1 r, r'r;
//   C  the convergence test; beta = rho_new / rho; p = D^-1 r + beta p.
// Every block sums the partials itself, in block order, so all blocks hold the
// same scalars and take the same branch.  The right-hand side and the result
// are in the cycle precision T; the iteration count is written to *iters.
#include "grid_sync.cuh"
#include "tosp_internal.h"

namespace tosp {

namespace {

constexpr int CPCG_THREADS = 256;
constexpr uint32_t CPCG_WAIT_LIMIT = 1u << 21;   // polls of 64 ns or more per barrier: > 0.1 s

__device__ __forceinline__ double block_sum_d(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
    return s;   // valid in thread 0
}

// Sum of the blocks' partials part[0 .. nb-1], returned to every thread.  The
// same fixed reduction tree runs in every block, so all blocks get the same
// value.
__device__ __forceinline__ double sum_blocks(const double *part, int nb, double *sh) {
    __shared__ double s_tot;
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v += __ldcg(part + i);
    v = block_sum_d(v, sh);
    if (threadIdx.x == 0) s_tot = v;
    __syncthreads();
    const double t = s_tot;
    __syncthreads();
    return t;
}

}  // namespace

template <typename T>
__global__ void __launch_bounds__(CPCG_THREADS)
k_coarse_pcg(const double *__restrict__ st, const double *__restrict__ invd, const T *__restrict__ b,
             T *__restrict__ xout, Grid g, double *x, double *r, double *p, double *q, double *part,
             GridBarrier *bar, double tol, int maxit, int *iters) {
    __shared__ double sh[32];
    const unsigned nb = gridDim.x;
    const uint32_t limit = bar->limit ? bar->limit : CPCG_WAIT_LIMIT;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nthr = (int64_t)nb * blockDim.x;
    const int lane = threadIdx.x & 31;
    const int64_t warp = tid >> 5, nwarps = nthr >> 5;
    const int64_t nd = g.ndof;
    double *pA = part, *pB0 = part + nb, *pB1 = part + 2 * nb;

    // x = 0, r = b, p = D^-1 r; partials of r'p and b'b
    double s0 = 0.0, s1 = 0.0;
    for (int64_t i = tid; i < nd; i += nthr) {
        const double bi = (double)b[i];
        const double zi = invd[i] * bi;
        x[i] = 0.0;
        r[i] = bi;
        p[i] = zi;
        s0 += bi * zi;
        s1 += bi * bi;
    }
    s0 = block_sum_d(s0, sh);
    s1 = block_sum_d(s1, sh);
    if (threadIdx.x == 0) {
        pB0[blockIdx.x] = s0;
        pB1[blockIdx.x] = s1;
    }
    if (!grid_barrier(bar, nb, limit, false)) return;
    double rho = sum_blocks(pB0, nb, sh);
    const double bb = sum_blocks(pB1, nb, sh);
    int it = 0;
    bool done = !(bb > 0.0) || !(sqrt(bb) > 0.0);
    while (!done && it < maxit) {
        // A: q = A p (warp per node) and p'q
        double pq = 0.0;
        for (int64_t I = warp; I < g.nnodes; I += nwarps) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0;
            if (lane < 27) {
                const int i = (int)I, qy = i / g.ny;
                const int yy = i - qy * g.ny, zz = qy / g.nx, xx = qy - zz * g.nx;
                const int oy = lane % 3 - 1, ox = (lane / 3) % 3 - 1, oz = lane / 9 - 1;
                const int jx = xx + ox, jy = yy + oy, jz = zz + oz;
                if (jx >= 0 && jx < g.nx && jy >= 0 && jy < g.ny && jz >= 0 && jz < g.nz) {
                    const int64_t J = I + ((int64_t)oz * g.nx + ox) * g.ny + oy;
                    const double x0 = __ldcg(p + 3 * J), x1 = __ldcg(p + 3 * J + 1), x2 = __ldcg(p + 3 * J + 2);
                    const double *sv = st + I * STENCIL_VALS + lane * 9;
                    a0 = __ldg(sv + 0) * x0 + __ldg(sv + 1) * x1 + __ldg(sv + 2) * x2;
                    a1 = __ldg(sv + 3) * x0 + __ldg(sv + 4) * x1 + __ldg(sv + 5) * x2;
                    a2 = __ldg(sv + 6) * x0 + __ldg(sv + 7) * x1 + __ldg(sv + 8) * x2;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                a0 += __shfl_xor_sync(0xffffffffu, a0, o);
                a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                a2 += __shfl_xor_sync(0xffffffffu, a2, o);
            }
            if (lane < 3) {
                const double a = lane == 0 ? a0 : (lane == 1 ? a1 : a2);
                const int64_t d = 3 * I + lane;
                q[d] = a;
                pq += __ldcg(p + d) * a;
            }
        }
        pq = block_sum_d(pq, sh);
        if (threadIdx.x == 0) pA[blockIdx.x] = pq;
        if (!grid_barrier(bar, nb, limit, false)) return;
        // B: the updates of x and r, and the partials of r'D^-1 r and r'r
        const double alpha = rho / sum_blocks(pA, nb, sh);
        s0 = 0.0;
        s1 = 0.0;
        for (int64_t i = tid; i < nd; i += nthr) {
            x[i] += alpha * __ldcg(p + i);
            const double ri = __ldcg(r + i) - alpha * __ldcg(q + i);
            r[i] = ri;
            s0 += ri * invd[i] * ri;
            s1 += ri * ri;
        }
        s0 = block_sum_d(s0, sh);
        s1 = block_sum_d(s1, sh);
        if (threadIdx.x == 0) {
            pB0[blockIdx.x] = s0;
            pB1[blockIdx.x] = s1;
        }
        if (!grid_barrier(bar, nb, limit, false)) return;
        // C: convergence test and the next direction
        const double rho_new = sum_blocks(pB0, nb, sh);
        const double rr = sum_blocks(pB1, nb, sh);
        ++it;
        if (sqrt(rr) <= tol * sqrt(bb) || !(rho_new == rho_new)) break;
        const double beta = rho_new / rho;
        rho = rho_new;
        for (int64_t i = tid; i < nd; i += nthr) p[i] = invd[i] * __ldcg(r + i) + beta * __ldcg(p + i);
        if (!grid_barrier(bar, nb, limit, false)) return;
    }
    for (int64_t i = tid; i < nd; i += nthr) xout[i] = (T)__ldcg(x + i);
    if (tid == 0) *iters = it;
}

template <typename T>
int coarse_pcg_blocks() {
    static int blocks = 0;
    if (!blocks) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_coarse_pcg<T>, CPCG_THREADS, 0);
        blocks = sms * (per < 1 ? 1 : (per > 2 ? 2 : per));
    }
    return blocks;
}

template <typename T>
void launch_coarse_pcg(const double *st, const double *invd, const T *b, T *x, const Grid &g, CoarsePcgWork &w,
                       double tol, int maxit, cudaStream_t stream) {
    int nblocks = coarse_pcg_blocks<T>();
    const int64_t warps_needed = g.nnodes;                       // one warp per node is enough parallelism
    const int64_t want = (warps_needed * 32 + CPCG_THREADS - 1) / CPCG_THREADS;
    if (want < nblocks) nblocks = (int)(want < 1 ? 1 : want);
    if (nblocks > w.max_blocks) nblocks = w.max_blocks;
    void *args[] = {(void *)&st, (void *)&invd, (void *)&b,     (void *)&x,     (void *)&g,
                    (void *)&w.x, (void *)&w.r, (void *)&w.p,   (void *)&w.q,   (void *)&w.part,
                    (void *)&w.bar, (void *)&tol, (void *)&maxit, (void *)&w.iters};
    cudaLaunchCooperativeKernel((const void *)k_coarse_pcg<T>, dim3(nblocks), dim3(CPCG_THREADS), args, 0, stream);
    count_launch();
}

template void launch_coarse_pcg<float>(const double *, const double *, const float *, float *, const Grid &,
                                       CoarsePcgWork &, double, int, cudaStream_t);
template void launch_coarse_pcg<double>(const double *, const double *, const double *, double *, const Grid &,
                                        CoarsePcgWork &, double, int, cudaStream_t);

int coarse_pcg_max_blocks() { return coarse_pcg_blocks<double>() > coarse_pcg_blocks<float>()
                                         ? coarse_pcg_blocks<double>() : coarse_pcg_blocks<float>(); }

}  // namespace tosp
